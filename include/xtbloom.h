/*
 * xtbloom_b200 public C ABI.
 *
 * This is the drop-in boundary of the batched GFN2-xTB / GFN1-xTB single-point
 * path.  Every structure layout, enum value and entry point below is the one
 * the reference library exports in its public header
 * (include/xtbloom/xtbloom.h in the reference project; line numbers cited per
 * declaration), so bindings written against the reference (its ctypes package
 * python/xtbloom/library.py:417-650, its torch extension, C consumers) load
 * this library unchanged through XTBLOOM_LIBRARY.  Only plain pointers, sizes
 * and int32 tags cross the boundary.  The caller owns all memory.
 */
#ifndef XTBLOOM_B200_XTBLOOM_H
#define XTBLOOM_B200_XTBLOOM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__) || defined(__clang__)
#define XTBLOOM_API __attribute__((visibility("default")))
#else
#define XTBLOOM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* xtbloom.h:28 */
#define XTBLOOM_API_VERSION 1u
/* k_B*T conversion used by the pinned xTB/tblite convention, xtbloom.h:31-35. */
#define XTBLOOM_KELVIN_TO_HARTREE 3.166808578545117e-6
#define XTBLOOM_DEFAULT_ELECTRONIC_TEMPERATURE (300.0 * XTBLOOM_KELVIN_TO_HARTREE)

typedef struct xtbloom_context xtbloom_context_t;
typedef struct xtbloom_plan xtbloom_plan_t;
typedef struct xtbloom_request xtbloom_request_t;

/* All tags are int32_t (xtbloom.h:59-205). */
typedef int32_t xtbloom_status_t;
enum {
  XTBLOOM_STATUS_SUCCESS = 0,
  XTBLOOM_STATUS_INVALID_ARGUMENT = 1,
  XTBLOOM_STATUS_BACKEND_UNAVAILABLE = 2,
  XTBLOOM_STATUS_NOT_SUPPORTED = 3,
  XTBLOOM_STATUS_ALLOCATION_FAILED = 4,
  XTBLOOM_STATUS_NOT_IMPLEMENTED = 5,
  XTBLOOM_STATUS_INTERNAL_ERROR = 6,
  XTBLOOM_STATUS_SCC_NOT_CONVERGED = 7,
  XTBLOOM_STATUS_EIGENSOLVER_FAILED = 8
};
typedef int32_t xtbloom_request_state_t;
enum { XTBLOOM_REQUEST_IDLE = 0, XTBLOOM_REQUEST_PENDING = 1, XTBLOOM_REQUEST_COMPLETE = 2 };
typedef int32_t xtbloom_backend_t;
enum {
  XTBLOOM_BACKEND_AUTO = 0,
  XTBLOOM_BACKEND_CPU = 1,
  XTBLOOM_BACKEND_CUDA = 2,
  XTBLOOM_BACKEND_ROCM = 3
};
typedef int32_t xtbloom_memory_space_t;
enum { XTBLOOM_MEMORY_HOST = 0, XTBLOOM_MEMORY_CUDA_DEVICE = 1, XTBLOOM_MEMORY_ROCM_DEVICE = 2 };
typedef int32_t xtbloom_model_t;
enum { XTBLOOM_MODEL_GFN1_XTB = 1, XTBLOOM_MODEL_GFN2_XTB = 2 };
typedef int32_t xtbloom_scc_start_mode_t;
enum { XTBLOOM_SCC_START_FRESH = 1, XTBLOOM_SCC_START_WARM = 2 };
typedef int32_t xtbloom_scc_mixer_t;
enum { XTBLOOM_SCC_MIXER_MODIFIED_BROYDEN = 1 };
typedef int32_t xtbloom_determinism_t;
enum { XTBLOOM_DETERMINISM_DEFAULT = 0, XTBLOOM_DETERMINISM_REPRODUCIBLE = 1 };
enum {
  XTBLOOM_COMPUTE_ENERGY = 1 << 0,
  XTBLOOM_COMPUTE_FORCES = 1 << 1,
  XTBLOOM_COMPUTE_ATOMIC_CHARGES = 1 << 2,
  XTBLOOM_COMPUTE_POINT_CHARGE_FORCES = 1 << 3,
  XTBLOOM_COMPUTE_DIPOLE_MOMENTS = 1 << 4
};
enum {
  XTBLOOM_RESULT_FORCES_EXCLUDE_EXTERNAL_OPERATOR_DERIVATIVES = 1 << 0,
  XTBLOOM_RESULT_DIPOLE_MOMENTS = 1 << 4
};
typedef int32_t xtbloom_interaction_type_t;
enum { XTBLOOM_INTERACTION_NONE = 0, XTBLOOM_INTERACTION_ELECTRIC_FIELD = 0x0101 };
typedef int32_t xtbloom_periodic_axes_t;
enum { XTBLOOM_PERIODIC_AXES_NONE = 0, XTBLOOM_PERIODIC_AXES_XYZ = 7 };

/* xtbloom.h:243-252 */
typedef struct xtbloom_interaction {
  xtbloom_interaction_type_t type;
  uint32_t flags;
  int64_t system_index;
  uint64_t payload_offset;
  uint64_t payload_size;
} xtbloom_interaction_t;

/* xtbloom.h:284-294 */
typedef struct xtbloom_context_options {
  uint32_t struct_size;
  uint32_t api_version;
  xtbloom_backend_t backend;
  int32_t device_id;
  int32_t cpu_threads;
  uint32_t reserved;
  void* stream;
} xtbloom_context_options_t;

/* xtbloom.h:299-313 */
typedef struct xtbloom_const_buffer {
  const void* data;
  size_t size_bytes;
  xtbloom_memory_space_t memory_space;
  uint32_t reserved;
} xtbloom_const_buffer_t;
typedef struct xtbloom_buffer {
  void* data;
  size_t size_bytes;
  xtbloom_memory_space_t memory_space;
  uint32_t reserved;
} xtbloom_buffer_t;

/* Ragged molecular batch, xtbloom.h:437-487. */
typedef struct xtbloom_batch {
  uint32_t struct_size;
  uint32_t api_version;
  int64_t batch_size;
  int64_t total_atoms;
  int64_t total_point_charges;
  int64_t total_charge_response_elements;
  xtbloom_const_buffer_t atom_offsets;
  xtbloom_const_buffer_t atomic_numbers;
  xtbloom_const_buffer_t positions;
  xtbloom_const_buffer_t molecular_charges;
  xtbloom_const_buffer_t unpaired_electrons;
  xtbloom_const_buffer_t point_charge_offsets;
  xtbloom_const_buffer_t point_charge_positions;
  xtbloom_const_buffer_t point_charge_values;
  xtbloom_const_buffer_t point_charge_gammas;
  xtbloom_const_buffer_t atomic_potential_shifts;
  xtbloom_const_buffer_t charge_response_offsets;
  xtbloom_const_buffer_t charge_response_matrix;
  xtbloom_const_buffer_t spin_channels;
  int64_t total_interactions;
  xtbloom_const_buffer_t interaction_descriptors;
  xtbloom_const_buffer_t interaction_payload;
  xtbloom_const_buffer_t cell_matrices;
  xtbloom_const_buffer_t periodic_axes;
} xtbloom_batch_t;

/* xtbloom.h:525-552 */
typedef struct xtbloom_compute_options {
  uint32_t struct_size;
  uint32_t api_version;
  xtbloom_model_t model;
  uint32_t flags;
  int32_t max_scc_iterations;
  uint32_t reserved;
  double charge_tolerance;
  double energy_tolerance;
  double electronic_temperature;
  xtbloom_scc_start_mode_t scc_start_mode;
  uint32_t reserved_v2;
  xtbloom_scc_mixer_t scc_mixer;
  int32_t scc_mixer_history;
  double scc_mixer_damping;
  xtbloom_determinism_t determinism;
  uint32_t reserved_v3;
} xtbloom_compute_options_t;

/* xtbloom.h:664-687 */
typedef struct xtbloom_batch_result {
  uint32_t struct_size;
  uint32_t api_version;
  uint32_t flags;
  uint32_t reserved;
  xtbloom_buffer_t energies;
  xtbloom_buffer_t forces;
  xtbloom_buffer_t atomic_charges;
  xtbloom_buffer_t point_charge_forces;
  xtbloom_buffer_t scc_iterations;
  xtbloom_buffer_t scc_converged;
  xtbloom_buffer_t per_system_status;
  xtbloom_buffer_t dipole_moments;
  xtbloom_buffer_t quadrupole_moments;
  xtbloom_buffer_t wiberg_orders;
  xtbloom_buffer_t spin_populations;
} xtbloom_batch_result_t;

/* xtbloom.h:727-740 */
typedef struct xtbloom_workspace_query {
  uint32_t struct_size;
  uint32_t api_version;
  uint32_t compute_flags;
  uint32_t reserved;
  uint64_t host_required_bytes;
  uint32_t host_required_alignment;
  uint64_t device_required_bytes;
  uint32_t device_required_alignment;
  uint32_t reserved_v2;
} xtbloom_workspace_query_t;

/* xtbloom.h:766-775 */
typedef struct xtbloom_request_info {
  uint32_t struct_size;
  uint32_t api_version;
  xtbloom_request_state_t state;
  xtbloom_status_t completion_status;
  uint32_t result_flags;
  uint32_t reserved;
} xtbloom_request_info_t;

#define XTBLOOM_CONTEXT_OPTIONS_V1_SIZE (offsetof(xtbloom_context_options_t, stream) + sizeof(void*))
#define XTBLOOM_BATCH_V1_SIZE \
  (offsetof(xtbloom_batch_t, charge_response_matrix) + sizeof(xtbloom_const_buffer_t))
#define XTBLOOM_BATCH_V2_SIZE (offsetof(xtbloom_batch_t, spin_channels) + sizeof(xtbloom_const_buffer_t))
#define XTBLOOM_BATCH_V3_SIZE \
  (offsetof(xtbloom_batch_t, interaction_payload) + sizeof(xtbloom_const_buffer_t))
#define XTBLOOM_BATCH_V4_SIZE (offsetof(xtbloom_batch_t, periodic_axes) + sizeof(xtbloom_const_buffer_t))
#define XTBLOOM_COMPUTE_OPTIONS_V1_SIZE \
  (offsetof(xtbloom_compute_options_t, electronic_temperature) + sizeof(double))
#define XTBLOOM_COMPUTE_OPTIONS_V2_SIZE (offsetof(xtbloom_compute_options_t, reserved_v2) + sizeof(uint32_t))
#define XTBLOOM_COMPUTE_OPTIONS_V3_SIZE (offsetof(xtbloom_compute_options_t, reserved_v3) + sizeof(uint32_t))
#define XTBLOOM_BATCH_RESULT_V1_SIZE \
  (offsetof(xtbloom_batch_result_t, per_system_status) + sizeof(xtbloom_buffer_t))
#define XTBLOOM_BATCH_RESULT_V2_SIZE \
  (offsetof(xtbloom_batch_result_t, spin_populations) + sizeof(xtbloom_buffer_t))

/* Version and diagnostics: xtbloom.h:821-825 (thread-local last error, src/api.cpp:45-50). */
XTBLOOM_API const char* xtbloom_version_string(void);
XTBLOOM_API const char* xtbloom_status_string(xtbloom_status_t status);
XTBLOOM_API const char* xtbloom_get_last_error(void);

/* Size-prefixed initialisers: xtbloom.h:827-837. */
XTBLOOM_API xtbloom_status_t xtbloom_context_options_init(xtbloom_context_options_t* options,
                                                          size_t struct_size);
XTBLOOM_API xtbloom_status_t xtbloom_batch_init(xtbloom_batch_t* batch, size_t struct_size);
XTBLOOM_API xtbloom_status_t xtbloom_compute_options_init(xtbloom_compute_options_t* options,
                                                          size_t struct_size);
XTBLOOM_API xtbloom_status_t xtbloom_batch_result_init(xtbloom_batch_result_t* result,
                                                       size_t struct_size);
XTBLOOM_API xtbloom_status_t xtbloom_workspace_query_init(xtbloom_workspace_query_t* query,
                                                          size_t struct_size);
XTBLOOM_API xtbloom_status_t xtbloom_request_info_init(xtbloom_request_info_t* info,
                                                       size_t struct_size);

/* Context lifecycle: xtbloom.h:839-843.  This library implements the CUDA
 * backend only (AUTO resolves to CUDA); a CPU request returns
 * BACKEND_UNAVAILABLE, there is no CPU fallback. */
XTBLOOM_API xtbloom_status_t xtbloom_context_create(const xtbloom_context_options_t* options,
                                                    xtbloom_context_t** context);
XTBLOOM_API void xtbloom_context_destroy(xtbloom_context_t* context);
XTBLOOM_API xtbloom_backend_t xtbloom_context_get_backend(const xtbloom_context_t* context);
XTBLOOM_API int32_t xtbloom_context_get_device_id(const xtbloom_context_t* context);

/* Requests: xtbloom.h:850-878. */
XTBLOOM_API xtbloom_status_t xtbloom_request_create(xtbloom_context_t* context,
                                                    xtbloom_request_t** request);
XTBLOOM_API xtbloom_status_t xtbloom_request_query(xtbloom_request_t* request,
                                                   xtbloom_request_info_t* info);
XTBLOOM_API xtbloom_status_t xtbloom_request_wait(xtbloom_request_t* request,
                                                  xtbloom_request_info_t* info);
XTBLOOM_API const char* xtbloom_request_get_error(const xtbloom_request_t* request);
XTBLOOM_API void xtbloom_request_destroy(xtbloom_request_t* request);

/* The batched single point: xtbloom.h:896-899 (synchronous) and 933-937 (enqueue). */
XTBLOOM_API xtbloom_status_t xtbloom_compute(xtbloom_context_t* context,
                                             const xtbloom_batch_t* batch,
                                             const xtbloom_compute_options_t* options,
                                             xtbloom_batch_result_t* result);
XTBLOOM_API xtbloom_status_t xtbloom_compute_enqueue(xtbloom_context_t* context,
                                                     const xtbloom_batch_t* batch,
                                                     const xtbloom_compute_options_t* options,
                                                     const xtbloom_batch_result_t* result,
                                                     xtbloom_request_t* request);

/* Fixed-topology plans: xtbloom.h:960-1009. */
XTBLOOM_API xtbloom_status_t xtbloom_plan_create(xtbloom_context_t* context,
                                                 const xtbloom_batch_t* batch,
                                                 const xtbloom_compute_options_t* options,
                                                 xtbloom_plan_t** plan);
XTBLOOM_API void xtbloom_plan_destroy(xtbloom_plan_t* plan);
XTBLOOM_API xtbloom_status_t xtbloom_plan_query_workspace(const xtbloom_plan_t* plan,
                                                          xtbloom_workspace_query_t* query);
XTBLOOM_API xtbloom_status_t xtbloom_plan_compute(xtbloom_plan_t* plan,
                                                  const xtbloom_batch_t* batch,
                                                  const xtbloom_compute_options_t* options,
                                                  xtbloom_batch_result_t* result);
XTBLOOM_API xtbloom_status_t xtbloom_plan_compute_enqueue(xtbloom_plan_t* plan,
                                                          const xtbloom_batch_t* batch,
                                                          const xtbloom_compute_options_t* options,
                                                          const xtbloom_batch_result_t* result,
                                                          xtbloom_request_t* request);

/* Result arenas: xtbloom.h:1011-1150.  Host and CUDA arenas, reference
 * counted; a compact row-major slice exports as a DLPack 1.0 managed tensor
 * (version 1: DLManagedTensorVersioned, version 0: legacy DLManagedTensor)
 * that holds one arena reference until its deleter runs. */
typedef struct xtbloom_result_owner xtbloom_result_owner_t;
typedef struct xtbloom_result_owner_options {
  uint32_t struct_size;
  uint32_t api_version;
  xtbloom_memory_space_t memory_space;
  int32_t device_id;
  uint64_t size_bytes;
  uint32_t reserved;
} xtbloom_result_owner_options_t;
typedef struct xtbloom_dlpack_view {
  uint32_t struct_size;
  uint32_t api_version;
  uint64_t byte_offset;
  int32_t dtype_code;
  int32_t dtype_bits;
  int32_t dtype_lanes;
  int32_t ndim;
  uint32_t reserved;
  const int64_t* shape;
} xtbloom_dlpack_view_t;
#define XTBLOOM_DLPACK_MAX_NDIM 8
#define XTBLOOM_DLPACK_VIEW_V1_SIZE \
  (offsetof(xtbloom_dlpack_view_t, shape) + sizeof(const int64_t*))
XTBLOOM_API xtbloom_status_t
xtbloom_result_owner_options_init(xtbloom_result_owner_options_t* options, size_t struct_size);
XTBLOOM_API xtbloom_status_t xtbloom_result_owner_create(
    const xtbloom_result_owner_options_t* options, xtbloom_result_owner_t** owner);
XTBLOOM_API xtbloom_status_t xtbloom_result_owner_buffer(const xtbloom_result_owner_t* owner,
                                                         xtbloom_buffer_t* buffer);
XTBLOOM_API void xtbloom_result_owner_retain(xtbloom_result_owner_t* owner);
XTBLOOM_API void xtbloom_result_owner_release(xtbloom_result_owner_t* owner);
XTBLOOM_API xtbloom_status_t xtbloom_result_owner_export_dltensor(
    const xtbloom_result_owner_t* owner, const xtbloom_dlpack_view_t* view, int version,
    void** out_managed);

/*
 * Diagnostics export (no counterpart in the reference ABI): copies one
 * retained per-system intermediate of the context's most recent compute into
 * host memory, for stage-by-stage parity tests.  name is one of "cn",
 * "overlap", "h0", "density", "eigenvalues", "qsh", "dipoles", "quadrupoles",
 * "energy_terms", "point_charge_potential" (per shell), "point_charge_dq"
 * (dE/dQ per point charge; system -1 returns every charge of the batch).
 * Returns INVALID_ARGUMENT when the name, system or capacity is wrong.
 * *count receives the number of doubles.
 */
XTBLOOM_API xtbloom_status_t xtbloom_b200_debug_fetch(xtbloom_context_t* context, const char* name,
                                                      int64_t system, double* out,
                                                      size_t capacity, size_t* count);

/*
 * Execution form of a CUDA context's later computes (no counterpart in the
 * reference ABI, whose arithmetic is FP64 throughout).
 *   precision 0 (XTBLOOM_B200_PRECISION_FP64, the default): every stage FP64.
 *   precision 1 (XTBLOOM_B200_PRECISION_MIXED): the basis-transform and density
 *     GEMMs of an SCC iteration run as split-precision (3xTF32, FP32
 *     accumulation) tensor-core products while the system's charge residual is
 *     at least switch_residual (0 selects 1e-5); below it the system iterates
 *     in FP64, and it converges only on an FP64 iteration, so energies, forces
 *     and charges are those of the FP64 fixed point.  The eigensolver, the
 *     occupations, the mixer and every energy and force reduction stay FP64.
 *     scc_iterations may differ from the FP64 form by a few iterations.
 *   capture_graphs nonzero: SCC iterations whose active set is unchanged are
 *     replayed from a captured CUDA graph (same kernels and results).
 * Returns INVALID_ARGUMENT for an unknown precision or a negative or
 * non-finite switch_residual, BACKEND_UNAVAILABLE for a CPU context.
 */
#define XTBLOOM_B200_PRECISION_FP64 0
#define XTBLOOM_B200_PRECISION_MIXED 1
XTBLOOM_API xtbloom_status_t xtbloom_b200_context_set_execution(xtbloom_context_t* context,
                                                                int32_t precision,
                                                                double switch_residual,
                                                                int32_t capture_graphs);

/*
 * Allocation-free eigenvectors of one symmetric tridiagonal matrix (no
 * counterpart in the reference ABI).  For callers that may not allocate device
 * memory once set up: cudaMalloc/cudaFree can synchronise the device and fail
 * under a committed memory budget.  Inverse iteration for eigenvectors
 * 0..m-1 of T = tridiag(offdiagonal[n-1], diagonal[n], offdiagonal[n-1]) with
 * ascending eigenvalues[m]; vector j goes to vectors[j*n .. j*n+n), largest
 * component positive.  The eigenvalues must be sorted ascending: with
 * unsorted values every gap looks like a cluster and the vectors returned are
 * undefined (the call cannot detect this and still returns SUCCESS).  All pointers are CUDA device memory of the current
 * device (offdiagonal may be NULL when n == 1); the work is enqueued on
 * cuda_stream (a cudaStream_t, NULL for the default stream) and the call
 * returns without waiting.  cluster_tolerance (0 selects 2e-7, the value the
 * SCC uses for Hamiltonians; the overlap factorisation uses 2e-6) is relative
 * to ||T||_1: eigenvalues closer than that are re-orthogonalised together.
 * An error already pending from earlier asynchronous work is reported as
 * INTERNAL_ERROR with its own message, before anything is launched.
 * Work vectors live in a fixed 1.25 MiB array of the library's device memory,
 * so n is limited to 256 (INVALID_ARGUMENT beyond, before anything runs);
 * nothing in it has to start at zero.  Calls that overlap on one device race
 * on that array: serialise them.  The first call on each device looks the
 * array up (and may load the module), so it belongs in the caller's set-up.
 */
XTBLOOM_API xtbloom_status_t xtbloom_b200_tridiag_eigenvectors_static(
    const double* diagonal, const double* offdiagonal, const double* eigenvalues, int32_t n,
    int32_t m, double* vectors, double cluster_tolerance, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* XTBLOOM_B200_XTBLOOM_H */
