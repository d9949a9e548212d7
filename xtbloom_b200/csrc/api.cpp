// The extern "C" boundary: struct initialisation, validation before any
// output is touched, context/request/plan lifecycles, thread-local error
// text, and dispatch into the CUDA engine.  Semantics follow the reference
// ABI implementation (src/api.cpp:45-1169, runtime/validation.cpp:368-1447):
// call-level failures modify no output; a SUCCESS return means every
// per-system diagnostic was committed, failed systems carrying quiet-NaN
// slices.  Exceptions never cross the boundary.
#include <atomic>
#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "engine.h"
#include "static_eigvec.h"
#include "xtbloom.h"

namespace {

thread_local std::string g_last_error;

xtbloom_status_t fail(xtbloom_status_t st, const std::string& msg) {
  g_last_error = msg;
  return st;
}

template <class T>
xtbloom_status_t init_struct(T* p, size_t size, size_t v1) {
  if (p == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "structure pointer is NULL");
  if (size < v1 || size > UINT32_MAX)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT,
                "structure size is smaller than its ABI-v1 prefix or exceeds uint32_t");
  // Never write past the layout this library knows; the caller's size is
  // recorded as given (a newer caller's larger structure keeps its size), as
  // the reference does (src/api.cpp:66-80).
  const size_t n = size < sizeof(T) ? size : sizeof(T);
  std::memset(static_cast<void*>(p), 0, n);
  p->struct_size = static_cast<uint32_t>(size);
  p->api_version = XTBLOOM_API_VERSION;
  g_last_error.clear();
  return XTBLOOM_STATUS_SUCCESS;
}

template <class T>
bool valid_header(const T* p, size_t v1) {
  return p != nullptr && p->struct_size >= v1 && p->api_version == XTBLOOM_API_VERSION;
}

bool has_field(uint32_t struct_size, size_t end) { return struct_size >= end; }

bool buffer_active(const xtbloom_const_buffer_t& b) { return b.data != nullptr || b.size_bytes != 0; }

bool check_in(const xtbloom_const_buffer_t& b, size_t need, const char* name, std::string& err) {
  if (need == 0) return true;
  if (b.data == nullptr) {
    err = std::string(name) + " must not be NULL";
    return false;
  }
  if (b.size_bytes < need) {
    err = std::string(name) + " is smaller than the batch requires";
    return false;
  }
  if (b.memory_space != XTBLOOM_MEMORY_HOST && b.memory_space != XTBLOOM_MEMORY_CUDA_DEVICE) {
    err = std::string(name) + " uses an unsupported memory space";
    return false;
  }
  if (b.reserved != 0) {
    err = std::string(name) + " reserved field must be zero";
    return false;
  }
  return true;
}

bool check_out(const xtbloom_buffer_t& b, size_t need, bool required, const char* name, std::string& err) {
  if (!required) return true;
  if (b.data == nullptr) {
    err = std::string(name) + " output must not be NULL when requested";
    return false;
  }
  if (b.size_bytes < need) {
    err = std::string(name) + " output is smaller than the batch requires";
    return false;
  }
  if (b.memory_space != XTBLOOM_MEMORY_HOST && b.memory_space != XTBLOOM_MEMORY_CUDA_DEVICE) {
    err = std::string(name) + " output uses an unsupported memory space";
    return false;
  }
  return true;
}

}  // namespace

struct xtbloom_context {
  std::mutex mutex;   // one transaction at a time (synchronous calls and accepted requests)
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::unique_ptr<xtb::Engine> engine;
  // execution form (xtbloom_b200_context_set_execution), applied to the
  // context engine and to the engines of its plans
  int precision = 0;
  double switch_residual = 1e-5;
  bool graphs = false;
};

// A reusable asynchronous request (src/runtime/request.cpp semantics): an
// accepted submission runs on a worker thread that drives the context stream
// under the context's transaction lock, so enqueue returns at once; query
// polls the state, wait blocks until the submission has completed.  The
// descriptors are copied at submission; the buffers they name must stay
// valid until completion.
struct xtbloom_request {
  xtbloom_context_t* context = nullptr;
  std::mutex mu;
  std::condition_variable cv;
  xtbloom_request_state_t state = XTBLOOM_REQUEST_IDLE;
  xtbloom_status_t completion = XTBLOOM_STATUS_SUCCESS;
  uint32_t result_flags = 0;
  std::string error;
  std::mutex join_mu;
  std::thread worker;
  xtbloom_batch_t batch{};
  xtbloom_compute_options_t options{};
  xtbloom_batch_result_t result{};
  xtb::ComputeRequest req;
  void join() {
    std::lock_guard<std::mutex> lock(join_mu);
    if (worker.joinable()) worker.join();
  }
};

// The immutable part of a batch that a fixed-topology plan binds
// (docs/developer-guide/architecture.md "Fixed-topology plans"): atom
// offsets, element numbers, molecular charges, unpaired electrons, spin
// channels, point-charge and charge-response structure.
struct PlanTopology {
  int64_t nsys = 0, natoms = 0, npc = 0;
  std::vector<int64_t> atom_off, pc_off, resp_off;
  std::vector<int32_t> Z, uhf, nch;
  std::vector<double> qmol;
  bool has_nch = false, has_pc = false, has_resp = false;
  bool operator==(const PlanTopology& o) const {
    return nsys == o.nsys && natoms == o.natoms && npc == o.npc && atom_off == o.atom_off &&
           pc_off == o.pc_off && resp_off == o.resp_off && Z == o.Z && uhf == o.uhf && nch == o.nch &&
           qmol == o.qmol && has_nch == o.has_nch && has_pc == o.has_pc && has_resp == o.has_resp;
  }
};

// The compute policy a plan binds: model, requested properties, SCC
// tolerances, iteration limit, electronic temperature, mixer, determinism
// (FRESH or WARM stays a per-call choice).
struct PlanPolicy {
  int32_t model = 0, max_iter = 0, memory = 0, determinism = 0;
  uint32_t flags = 0;
  double ctol = 0, etol = 0, kt = 0, damping = 0;
  bool operator==(const PlanPolicy& o) const {
    return model == o.model && max_iter == o.max_iter && memory == o.memory &&
           determinism == o.determinism && flags == o.flags && ctol == o.ctol && etol == o.etol &&
           kt == o.kt && damping == o.damping;
  }
};

struct xtbloom_plan {
  xtbloom_context_t* context = nullptr;
  std::unique_ptr<xtb::Engine> engine;   // plan-owned execution cache
  PlanTopology topo;
  PlanPolicy policy;
};

struct xtbloom_result_owner {
  std::atomic<int> refs{1};   // exported tensors may be released from any thread
  xtbloom_memory_space_t space = XTBLOOM_MEMORY_HOST;
  int device = -1;
  void* data = nullptr;
  uint64_t bytes = 0;
};

namespace {

xtbloom_status_t validate_and_normalise(const xtbloom_batch_t* batch,
                                        const xtbloom_compute_options_t* options,
                                        const xtbloom_batch_result_t* result, xtb::ComputeRequest& req,
                                        std::string& err) {
  if (!valid_header(batch, XTBLOOM_BATCH_V1_SIZE)) {
    err = "batch is NULL, too small, or uses an unsupported API version";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (!valid_header(options, XTBLOOM_COMPUTE_OPTIONS_V1_SIZE)) {
    err = "compute options are NULL, too small, or use an unsupported API version";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (!valid_header(result, XTBLOOM_BATCH_RESULT_V1_SIZE)) {
    err = "batch result is NULL, too small, or uses an unsupported API version";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (batch->batch_size <= 0) {
    err = "batch_size must be positive";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (batch->total_atoms < batch->batch_size) {
    err = "total_atoms must permit at least one atom in every batch item";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (batch->total_point_charges < 0 || batch->total_charge_response_elements < 0) {
    err = "point-charge and response counts must be nonnegative";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  const size_t B = static_cast<size_t>(batch->batch_size);
  const size_t N = static_cast<size_t>(batch->total_atoms);
  if (!check_in(batch->atom_offsets, (B + 1) * 8, "atom_offsets", err) ||
      !check_in(batch->atomic_numbers, N * 4, "atomic_numbers", err) ||
      !check_in(batch->positions, N * 24, "positions", err) ||
      !check_in(batch->molecular_charges, B * 8, "molecular_charges", err)) {
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (buffer_active(batch->unpaired_electrons) &&
      !check_in(batch->unpaired_electrons, B * 4, "unpaired_electrons", err)) {
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (has_field(batch->struct_size, XTBLOOM_BATCH_V2_SIZE) && buffer_active(batch->spin_channels)) {
    if (!check_in(batch->spin_channels, B * 4, "spin_channels", err)) return XTBLOOM_STATUS_INVALID_ARGUMENT;
    std::unique_ptr<int32_t[]> sc(new int32_t[B]);
    if (batch->spin_channels.memory_space == XTBLOOM_MEMORY_HOST) {
      std::memcpy(sc.get(), batch->spin_channels.data, B * 4);
    } else if (cudaMemcpy(sc.get(), batch->spin_channels.data, B * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
      err = "failed to read spin_channels";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    for (size_t i = 0; i < B; ++i) {
      if (sc[i] != 1 && sc[i] != 2) {
        err = "spin_channels values must be one or two";
        return XTBLOOM_STATUS_INVALID_ARGUMENT;
      }
    }
    req.spin_channels = true;
  }
  const size_t P = static_cast<size_t>(batch->total_point_charges);
  if (P != 0 || buffer_active(batch->point_charge_offsets)) {
    if (!check_in(batch->point_charge_offsets, (B + 1) * 8, "point_charge_offsets", err))
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (P != 0 && (!check_in(batch->point_charge_positions, P * 24, "point_charge_positions", err) ||
                 !check_in(batch->point_charge_values, P * 8, "point_charge_values", err) ||
                 !check_in(batch->point_charge_gammas, P * 8, "point_charge_gammas", err))) {
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  // Charge response b + A q for periodic QM/MM coupling (reference
  // include/xtbloom/xtbloom.h:429-436): per-atom shifts b, per-system
  // row-major symmetric A packed at charge_response_offsets.
  req.have_response = false;
  if (batch->total_charge_response_elements != 0 || buffer_active(batch->atomic_potential_shifts) ||
      buffer_active(batch->charge_response_offsets) || buffer_active(batch->charge_response_matrix)) {
    const int64_t E = batch->total_charge_response_elements;
    if (E < 0) {
      err = "total_charge_response_elements must be nonnegative";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    if (!check_in(batch->atomic_potential_shifts, N * 8, "atomic_potential_shifts", err) ||
        !check_in(batch->charge_response_offsets, (B + 1) * 8, "charge_response_offsets", err) ||
        !check_in(batch->charge_response_matrix, static_cast<size_t>(E) * 8, "charge_response_matrix", err))
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    req.resp_b.resize(N);
    req.resp_off.resize(B + 1);
    req.resp_A.resize(static_cast<size_t>(E));
    auto fetch_in = [&](const xtbloom_const_buffer_t& b, void* dst, size_t bytes) {
      if (bytes == 0) return true;
      if (b.memory_space == XTBLOOM_MEMORY_HOST) {
        std::memcpy(dst, b.data, bytes);
        return true;
      }
      return cudaMemcpy(dst, b.data, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
    };
    if (!fetch_in(batch->atomic_potential_shifts, req.resp_b.data(), N * 8) ||
        !fetch_in(batch->charge_response_offsets, req.resp_off.data(), (B + 1) * 8) ||
        !fetch_in(batch->charge_response_matrix, req.resp_A.data(), static_cast<size_t>(E) * 8)) {
      err = "failed to read the charge-response inputs";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    std::vector<int64_t> aoff(B + 1);
    if (!fetch_in(batch->atom_offsets, aoff.data(), (B + 1) * 8)) {
      err = "failed to read atom_offsets";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    if (req.resp_off[0] != 0 || req.resp_off[B] != E) {
      err = "charge_response_offsets must start at zero and end at total_charge_response_elements";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    for (size_t i = 0; i < B; ++i) {
      const int64_t na = aoff[i + 1] - aoff[i];
      if (na < 0 || req.resp_off[i + 1] - req.resp_off[i] != na * na) {
        err = "charge_response_offsets must delimit one atoms x atoms block per system";
        return XTBLOOM_STATUS_INVALID_ARGUMENT;
      }
      const double* A = req.resp_A.data() + req.resp_off[i];
      for (int64_t r = 0; r < na; ++r)
        for (int64_t c = 0; c < na; ++c) {
          if (!std::isfinite(A[r * na + c])) {
            err = "charge_response_matrix contains NaN or infinity";
            return XTBLOOM_STATUS_INVALID_ARGUMENT;
          }
          if (A[r * na + c] != A[c * na + r]) {
            err = "charge_response_matrix must be exactly symmetric per system";
            return XTBLOOM_STATUS_INVALID_ARGUMENT;
          }
        }
    }
    for (size_t a = 0; a < N; ++a)
      if (!std::isfinite(req.resp_b[a])) {
        err = "atomic_potential_shifts contains NaN or infinity";
        return XTBLOOM_STATUS_INVALID_ARGUMENT;
      }
    req.have_response = true;
  }
  // External interaction attachments (src/runtime/validation.cpp:916-1000,
  // 1104-1135 of the reference): the uniform electric field is executed, every
  // other known tag is refused as not implemented.
  req.field_attached.assign(B, 0);
  req.field.assign(3 * B, 0.0);
  if (has_field(batch->struct_size, XTBLOOM_BATCH_V3_SIZE) &&
      (batch->total_interactions != 0 || buffer_active(batch->interaction_descriptors))) {
    if (batch->total_interactions < 0) {
      err = "total_interactions must be nonnegative";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    const size_t K = static_cast<size_t>(batch->total_interactions);
    if (K > 0) {
      if (!check_in(batch->interaction_descriptors, K * sizeof(xtbloom_interaction_t),
                    "interaction_descriptors", err))
        return XTBLOOM_STATUS_INVALID_ARGUMENT;
      if (!buffer_active(batch->interaction_payload)) {
        err = "interaction_payload is required when interactions are present";
        return XTBLOOM_STATUS_INVALID_ARGUMENT;
      }
      auto stage = [&](const xtbloom_const_buffer_t& b, size_t bytes, std::vector<unsigned char>& out) {
        out.resize(bytes);
        if (bytes == 0) return true;
        if (b.memory_space == XTBLOOM_MEMORY_HOST) {
          std::memcpy(out.data(), b.data, bytes);
          return true;
        }
        return cudaMemcpy(out.data(), b.data, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
      };
      std::vector<unsigned char> desc, payload;
      const size_t pbytes = batch->interaction_payload.size_bytes;
      if (!stage(batch->interaction_descriptors, K * sizeof(xtbloom_interaction_t), desc) ||
          !stage(batch->interaction_payload, pbytes, payload)) {
        err = "failed to read the interaction attachments";
        return XTBLOOM_STATUS_INVALID_ARGUMENT;
      }
      bool other_tag = false;
      for (size_t k = 0; k < K; ++k) {
        xtbloom_interaction_t it;
        std::memcpy(&it, desc.data() + k * sizeof(xtbloom_interaction_t), sizeof(it));
        const bool known = (it.type >= 0x0101 && it.type <= 0x0104) ||
                           (it.type >= 0x0201 && it.type <= 0x0205) || it.type == 0x0301 ||
                           it.type == 0x0302 || it.type == 0x0401;
        if (it.flags != 0u) {
          err = "interaction descriptor flags must be zero";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
        if (!known) {
          err = "an interaction descriptor uses an unknown or NONE type tag";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
        if (it.system_index < 0 || static_cast<size_t>(it.system_index) >= B) {
          err = "an interaction system_index lies outside the batch";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
        if (it.payload_offset > pbytes || it.payload_size > pbytes - it.payload_offset) {
          err = "an interaction payload block extends past interaction_payload";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
        const uintptr_t addr = reinterpret_cast<uintptr_t>(batch->interaction_payload.data) +
                               static_cast<uintptr_t>(it.payload_offset);
        if (it.type != XTBLOOM_INTERACTION_ELECTRIC_FIELD) {
          if (it.payload_size < sizeof(int32_t) || addr % alignof(int32_t) != 0u) {
            err = "an interaction payload block must contain an aligned block_version";
            return XTBLOOM_STATUS_INVALID_ARGUMENT;
          }
          other_tag = true;
          continue;
        }
        // block_version 1: int32 version, int32 reserved, three doubles (8-byte aligned)
        if (it.payload_size < 32u || addr % alignof(double) != 0u) {
          err = "an electric-field interaction payload block is undersized or misaligned";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
        if (it.payload_size > 32u) {
          err = "an electric-field interaction payload block exceeds the released contract";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
        int32_t version = 0, reserved = 0;
        double e[3];
        const unsigned char* blk = payload.data() + it.payload_offset;
        std::memcpy(&version, blk, 4);
        std::memcpy(&reserved, blk + 4, 4);
        std::memcpy(e, blk + 8, 24);
        if (version != 1) {
          err = "an electric-field interaction uses an unsupported block_version";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
        if (reserved != 0) {
          err = "an electric-field interaction reserved payload field must be zero";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
        if (!std::isfinite(e[0]) || !std::isfinite(e[1]) || !std::isfinite(e[2])) {
          err = "an electric-field interaction contains NaN or infinity";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
        const size_t si = static_cast<size_t>(it.system_index);
        if (req.field_attached[si]) {
          err = "a batch item carries more than one electric-field attachment";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
        req.field_attached[si] = 1;
        for (int c = 0; c < 3; ++c) req.field[3 * si + c] = e[c];
      }
      if (other_tag) {
        err = "an interaction attachment uses a tag whose execution is not implemented";
        return XTBLOOM_STATUS_NOT_IMPLEMENTED;
      }
    }
  }
  if (has_field(batch->struct_size, XTBLOOM_BATCH_V4_SIZE) &&
      (buffer_active(batch->cell_matrices) || buffer_active(batch->periodic_axes))) {
    err = "native periodic cells are not implemented";
    return XTBLOOM_STATUS_NOT_IMPLEMENTED;
  }
  // options
  if (options->model != XTBLOOM_MODEL_GFN2_XTB && options->model != XTBLOOM_MODEL_GFN1_XTB) {
    err = "unknown model";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (options->model == XTBLOOM_MODEL_GFN1_XTB) {
    // as the reference (src/runtime/validation.cpp:1425-1437): GFN1 takes
    // point charges and charge response, but neither interaction attachments
    // (fields) nor the dipole publication
    bool field = false;
    for (uint8_t v : req.field_attached) field = field || v != 0;
    if ((options->flags & XTBLOOM_COMPUTE_DIPOLE_MOMENTS) != 0u) {
      err = "GFN1-xTB molecular dipole publication is not implemented";
      return XTBLOOM_STATUS_NOT_IMPLEMENTED;
    }
    if (field || (has_field(batch->struct_size, XTBLOOM_BATCH_V3_SIZE) && batch->total_interactions != 0)) {
      err = "GFN1-xTB interaction attachments are not implemented";
      return XTBLOOM_STATUS_NOT_IMPLEMENTED;
    }
  }
  req.model = options->model;
  const uint32_t known = XTBLOOM_COMPUTE_ENERGY | XTBLOOM_COMPUTE_FORCES |
                         XTBLOOM_COMPUTE_ATOMIC_CHARGES | XTBLOOM_COMPUTE_POINT_CHARGE_FORCES |
                         XTBLOOM_COMPUTE_DIPOLE_MOMENTS;
  if ((options->flags & ~known) != 0 || options->reserved != 0) {
    err = "compute flags contain reserved bits";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (options->max_scc_iterations <= 0) {
    err = "max_scc_iterations must be positive";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (!(options->charge_tolerance > 0.0) || !std::isfinite(options->charge_tolerance) ||
      !(options->energy_tolerance > 0.0) || !std::isfinite(options->energy_tolerance) ||
      !(options->electronic_temperature >= 0.0) || !std::isfinite(options->electronic_temperature)) {
    err = "tolerances must be finite and positive and the electronic temperature finite and nonnegative";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  req.flags = options->flags;
  req.max_iter = options->max_scc_iterations;
  req.ctol = options->charge_tolerance;
  req.etol = options->energy_tolerance;
  req.kt = options->electronic_temperature;
  req.memory = 8;
  req.damping = 0.4;
  if (has_field(options->struct_size, XTBLOOM_COMPUTE_OPTIONS_V2_SIZE)) {
    if (options->scc_start_mode != XTBLOOM_SCC_START_FRESH &&
        options->scc_start_mode != XTBLOOM_SCC_START_WARM && options->scc_start_mode != 0) {
      err = "unknown SCC start mode";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
  }
  req.warm = has_field(options->struct_size, XTBLOOM_COMPUTE_OPTIONS_V2_SIZE) &&
             options->scc_start_mode == XTBLOOM_SCC_START_WARM;
  if (has_field(options->struct_size, XTBLOOM_COMPUTE_OPTIONS_V3_SIZE)) {
    if (options->scc_mixer != XTBLOOM_SCC_MIXER_MODIFIED_BROYDEN || options->scc_mixer_history < 1 ||
        options->scc_mixer_history > 64 || !(options->scc_mixer_damping > 0.0) ||
        !(options->scc_mixer_damping <= 1.0) ||
        (options->determinism != XTBLOOM_DETERMINISM_DEFAULT &&
         options->determinism != XTBLOOM_DETERMINISM_REPRODUCIBLE)) {
      err = "invalid SCC mixer or determinism settings";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    if (options->scc_mixer_history > 8) {
      err = "Broyden history deeper than 8 is not supported by this CUDA path";
      return XTBLOOM_STATUS_NOT_SUPPORTED;
    }
    req.memory = options->scc_mixer_history;
    req.damping = options->scc_mixer_damping;
  }
  // result buffers
  const uint32_t f = options->flags;
  if (!check_out(result->energies, B * 8, (f & XTBLOOM_COMPUTE_ENERGY) != 0, "energies", err) ||
      !check_out(result->forces, N * 24, (f & XTBLOOM_COMPUTE_FORCES) != 0, "forces", err) ||
      !check_out(result->atomic_charges, N * 8, (f & XTBLOOM_COMPUTE_ATOMIC_CHARGES) != 0,
                 "atomic_charges", err) ||
      !check_out(result->point_charge_forces, P * 24,
                 (f & XTBLOOM_COMPUTE_POINT_CHARGE_FORCES) != 0 && P != 0, "point_charge_forces", err) ||
      !check_out(result->dipole_moments, B * 24, (f & XTBLOOM_COMPUTE_DIPOLE_MOMENTS) != 0,
                 "dipole_moments", err) ||
      !check_out(result->scc_iterations, B * 4, true, "scc_iterations", err) ||
      !check_out(result->scc_converged, B, true, "scc_converged", err) ||
      !check_out(result->per_system_status, B * 4, true, "per_system_status", err)) {
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  // positions must be finite (host check; device inputs are checked after staging)
  if (batch->positions.memory_space == XTBLOOM_MEMORY_HOST) {
    const double* x = static_cast<const double*>(batch->positions.data);
    for (size_t i = 0; i < 3 * N; ++i) {
      if (!std::isfinite(x[i])) {
        err = "positions contain NaN or infinity";
        return XTBLOOM_STATUS_INVALID_ARGUMENT;
      }
    }
  }
  req.batch = batch;
  req.options = options;
  req.result = result;
  return XTBLOOM_STATUS_SUCCESS;
}

// One transaction on an engine of the context (its own or a plan's): the
// caller holds no lock; the context's transaction lock is taken here.  The
// caller's current device is restored.
xtbloom_status_t execute(xtbloom_context_t* ctx, xtb::Engine* engine, const xtb::ComputeRequest& req,
                         uint32_t* result_flags, std::string& err) {
  std::lock_guard<std::mutex> lock(ctx->mutex);
  int prev = 0;
  cudaGetDevice(&prev);
  xtbloom_status_t st;
  try {
    engine->set_execution(ctx->precision, ctx->switch_residual, ctx->graphs);
    st = engine->compute(req, err);
  } catch (const std::bad_alloc&) {
    st = XTBLOOM_STATUS_ALLOCATION_FAILED;
    err = "host allocation failed";
  } catch (...) {
    st = XTBLOOM_STATUS_INTERNAL_ERROR;
    err = "unexpected exception in the CUDA engine";
  }
  cudaSetDevice(prev);
  if (result_flags) {
    uint32_t rf = 0u;
    if (st == XTBLOOM_STATUS_SUCCESS && (req.flags & XTBLOOM_COMPUTE_DIPOLE_MOMENTS))
      rf |= XTBLOOM_RESULT_DIPOLE_MOMENTS;
    if (st == XTBLOOM_STATUS_SUCCESS && req.have_response)
      rf |= XTBLOOM_RESULT_FORCES_EXCLUDE_EXTERNAL_OPERATOR_DERIVATIVES;
    *result_flags = rf;
  }
  return st;
}

xtbloom_status_t run(xtbloom_context_t* ctx, const xtbloom_batch_t* batch,
                     const xtbloom_compute_options_t* options, const xtbloom_batch_result_t* result,
                     uint32_t* result_flags) {
  if (ctx == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "context is NULL");
  xtb::ComputeRequest req;
  std::string err;
  xtbloom_status_t st = validate_and_normalise(batch, options, result, req, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return fail(st, err);
  st = execute(ctx, ctx->engine.get(), req, result_flags, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return fail(st, err);
  g_last_error.clear();
  return XTBLOOM_STATUS_SUCCESS;
}

// Copies a caller structure of `struct_size` bytes into the library's own
// layout (fields past the caller's size stay zero, fields past the library's
// layout are not read).
template <class T>
void copy_struct(T& dst, const T* src) {
  std::memset(static_cast<void*>(&dst), 0, sizeof(T));
  std::memcpy(static_cast<void*>(&dst), static_cast<const void*>(src),
              std::min<size_t>(src->struct_size, sizeof(T)));
  dst.struct_size = static_cast<uint32_t>(std::min<size_t>(src->struct_size, sizeof(T)));
}

// Accepts a validated submission on `request`: the descriptors are copied,
// the request turns PENDING and a worker thread runs the transaction.
xtbloom_status_t submit(xtbloom_context_t* ctx, xtb::Engine* engine, xtbloom_request_t* r,
                        const xtbloom_batch_t* batch, const xtbloom_compute_options_t* options,
                        const xtbloom_batch_result_t* result, xtb::ComputeRequest&& req) {
  {
    std::lock_guard<std::mutex> lock(r->mu);
    if (r->state == XTBLOOM_REQUEST_PENDING)
      return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "request already has pending work");
  }
  r->join();   // the previous submission's worker has finished; reclaim it
  copy_struct(r->batch, batch);
  copy_struct(r->options, options);
  copy_struct(r->result, result);
  r->req = std::move(req);
  r->req.batch = &r->batch;
  r->req.options = &r->options;
  r->req.result = &r->result;
  {
    std::lock_guard<std::mutex> lock(r->mu);
    r->state = XTBLOOM_REQUEST_PENDING;
    r->completion = XTBLOOM_STATUS_SUCCESS;
    r->result_flags = 0;
    r->error.clear();
  }
  try {
    r->worker = std::thread([ctx, engine, r] {
      std::string err;
      uint32_t flags = 0;
      const xtbloom_status_t st = execute(ctx, engine, r->req, &flags, err);
      {
        std::lock_guard<std::mutex> lock(r->mu);
        r->completion = st;
        r->result_flags = st == XTBLOOM_STATUS_SUCCESS ? flags : 0u;
        r->error = st == XTBLOOM_STATUS_SUCCESS ? std::string() : err;
        r->state = XTBLOOM_REQUEST_COMPLETE;
      }
      r->cv.notify_all();
    });
  } catch (...) {
    std::lock_guard<std::mutex> lock(r->mu);
    r->state = XTBLOOM_REQUEST_IDLE;
    return fail(XTBLOOM_STATUS_ALLOCATION_FAILED, "failed to start the request's worker thread");
  }
  g_last_error.clear();
  return XTBLOOM_STATUS_SUCCESS;
}

bool read_any(const xtbloom_const_buffer_t& b, void* dst, size_t bytes) {
  if (bytes == 0) return true;
  if (b.data == nullptr) return false;
  if (b.memory_space == XTBLOOM_MEMORY_HOST) {
    std::memcpy(dst, b.data, bytes);
    return true;
  }
  return cudaMemcpy(dst, b.data, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
}

// The immutable topology of a validated batch.
xtbloom_status_t capture_topology(const xtbloom_batch_t* b, const xtb::ComputeRequest& req,
                                  PlanTopology& t, std::string& err) {
  t.nsys = b->batch_size;
  t.natoms = b->total_atoms;
  t.npc = b->total_point_charges;
  const size_t B = (size_t)t.nsys, N = (size_t)t.natoms;
  t.atom_off.resize(B + 1);
  t.Z.resize(N);
  t.qmol.resize(B);
  t.uhf.assign(B, 0);
  bool ok = read_any(b->atom_offsets, t.atom_off.data(), (B + 1) * 8) &&
            read_any(b->atomic_numbers, t.Z.data(), N * 4) &&
            read_any(b->molecular_charges, t.qmol.data(), B * 8) &&
            (b->unpaired_electrons.data == nullptr || read_any(b->unpaired_electrons, t.uhf.data(), B * 4));
  t.has_nch = req.spin_channels;
  t.nch.assign(B, 1);
  if (ok && t.has_nch && b->spin_channels.data != nullptr) ok = read_any(b->spin_channels, t.nch.data(), B * 4);
  t.has_pc = t.npc > 0;
  t.pc_off.clear();
  if (ok && t.has_pc) {
    t.pc_off.resize(B + 1);
    ok = read_any(b->point_charge_offsets, t.pc_off.data(), (B + 1) * 8);
  }
  t.has_resp = req.have_response;
  t.resp_off = req.have_response ? req.resp_off : std::vector<int64_t>();
  if (!ok) {
    err = "failed to read the batch topology";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  return XTBLOOM_STATUS_SUCCESS;
}

PlanPolicy capture_policy(const xtbloom_compute_options_t* o, const xtb::ComputeRequest& req) {
  PlanPolicy p;
  p.model = o->model;
  p.flags = req.flags;
  p.max_iter = req.max_iter;
  p.ctol = req.ctol;
  p.etol = req.etol;
  p.kt = req.kt;
  p.memory = req.memory;
  p.damping = req.damping;
  p.determinism = has_field(o->struct_size, XTBLOOM_COMPUTE_OPTIONS_V3_SIZE) ? o->determinism : 0;
  return p;
}

// Validates a plan call: the batch and options on their own, then against
// the plan's bound topology and policy (before any output is touched).
xtbloom_status_t plan_request(const xtbloom_plan_t* plan, const xtbloom_batch_t* batch,
                              const xtbloom_compute_options_t* options,
                              const xtbloom_batch_result_t* result, xtb::ComputeRequest& req,
                              std::string& err) {
  xtbloom_status_t st = validate_and_normalise(batch, options, result, req, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return st;
  PlanTopology t;
  st = capture_topology(batch, req, t, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return st;
  if (!(t == plan->topo)) {
    err = "batch topology (atom offsets, elements, charges, spin, point-charge or charge-response "
          "structure) differs from the plan";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (!(capture_policy(options, req) == plan->policy)) {
    err = "compute policy (model, properties, SCC settings, mixer, determinism) differs from the plan";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  return XTBLOOM_STATUS_SUCCESS;
}

}  // namespace

extern "C" {

const char* xtbloom_version_string(void) { return "0.1.0+b200"; }

const char* xtbloom_status_string(xtbloom_status_t status) {
  switch (status) {
    case XTBLOOM_STATUS_SUCCESS: return "success";
    case XTBLOOM_STATUS_INVALID_ARGUMENT: return "invalid argument";
    case XTBLOOM_STATUS_BACKEND_UNAVAILABLE: return "backend unavailable";
    case XTBLOOM_STATUS_NOT_SUPPORTED: return "not supported";
    case XTBLOOM_STATUS_ALLOCATION_FAILED: return "allocation failed";
    case XTBLOOM_STATUS_NOT_IMPLEMENTED: return "not implemented";
    case XTBLOOM_STATUS_INTERNAL_ERROR: return "internal error";
    case XTBLOOM_STATUS_SCC_NOT_CONVERGED: return "SCC not converged";
    case XTBLOOM_STATUS_EIGENSOLVER_FAILED: return "eigensolver failed";
  }
  return "unknown status";
}

const char* xtbloom_get_last_error(void) { return g_last_error.c_str(); }

xtbloom_status_t xtbloom_context_options_init(xtbloom_context_options_t* o, size_t size) {
  const xtbloom_status_t st = init_struct(o, size, XTBLOOM_CONTEXT_OPTIONS_V1_SIZE);
  if (st != XTBLOOM_STATUS_SUCCESS) return st;
  o->backend = XTBLOOM_BACKEND_AUTO;
  o->device_id = -1;
  return XTBLOOM_STATUS_SUCCESS;
}

xtbloom_status_t xtbloom_batch_init(xtbloom_batch_t* b, size_t size) {
  return init_struct(b, size, XTBLOOM_BATCH_V1_SIZE);
}

xtbloom_status_t xtbloom_compute_options_init(xtbloom_compute_options_t* o, size_t size) {
  const xtbloom_status_t st = init_struct(o, size, XTBLOOM_COMPUTE_OPTIONS_V1_SIZE);
  if (st != XTBLOOM_STATUS_SUCCESS) return st;
  o->model = XTBLOOM_MODEL_GFN2_XTB;
  o->flags = XTBLOOM_COMPUTE_ENERGY | XTBLOOM_COMPUTE_FORCES;
  o->max_scc_iterations = 250;
  o->charge_tolerance = 1.0e-6;
  o->energy_tolerance = 1.0e-8;
  o->electronic_temperature = XTBLOOM_DEFAULT_ELECTRONIC_TEMPERATURE;
  if (size >= XTBLOOM_COMPUTE_OPTIONS_V2_SIZE) o->scc_start_mode = XTBLOOM_SCC_START_FRESH;
  if (size >= XTBLOOM_COMPUTE_OPTIONS_V3_SIZE) {
    o->scc_mixer = XTBLOOM_SCC_MIXER_MODIFIED_BROYDEN;
    o->scc_mixer_history = 8;
    o->scc_mixer_damping = 0.4;
    o->determinism = XTBLOOM_DETERMINISM_DEFAULT;
  }
  return XTBLOOM_STATUS_SUCCESS;
}

xtbloom_status_t xtbloom_batch_result_init(xtbloom_batch_result_t* r, size_t size) {
  return init_struct(r, size, XTBLOOM_BATCH_RESULT_V1_SIZE);
}

xtbloom_status_t xtbloom_workspace_query_init(xtbloom_workspace_query_t* q, size_t size) {
  return init_struct(q, size, offsetof(xtbloom_workspace_query_t, reserved_v2) + sizeof(uint32_t));
}

xtbloom_status_t xtbloom_request_info_init(xtbloom_request_info_t* i, size_t size) {
  return init_struct(i, size, offsetof(xtbloom_request_info_t, reserved) + sizeof(uint32_t));
}

xtbloom_status_t xtbloom_context_create(const xtbloom_context_options_t* options,
                                        xtbloom_context_t** context) {
  if (context == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "context output pointer is NULL");
  *context = nullptr;
  if (!valid_header(options, XTBLOOM_CONTEXT_OPTIONS_V1_SIZE))
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT,
                "context options are NULL, too small, or use an unsupported API version");
  if (options->reserved != 0) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "context options reserved field must be zero");
  if (options->backend == XTBLOOM_BACKEND_CPU || options->backend == XTBLOOM_BACKEND_ROCM)
    return fail(XTBLOOM_STATUS_BACKEND_UNAVAILABLE, "this library implements the CUDA backend only");
  if (options->backend != XTBLOOM_BACKEND_AUTO && options->backend != XTBLOOM_BACKEND_CUDA)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "unknown backend");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    return fail(XTBLOOM_STATUS_BACKEND_UNAVAILABLE, "no CUDA device is available");
  }
  int dev = options->device_id;
  if (dev < 0) {
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  }
  if (dev >= ndev) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "device_id is out of range");
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, dev);
  if (prop.major != 10) return fail(XTBLOOM_STATUS_BACKEND_UNAVAILABLE, "this library is built for sm_100a (B200) devices only");
  try {
    auto* ctx = new xtbloom_context;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(dev);
    ctx->device = dev;
    if (options->stream != nullptr) {
      ctx->stream = static_cast<cudaStream_t>(options->stream);
    } else {
      cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
      ctx->own_stream = true;
    }
    ctx->engine.reset(new xtb::Engine(dev, ctx->stream));
    cudaSetDevice(prev);
    *context = ctx;
    g_last_error.clear();
    return XTBLOOM_STATUS_SUCCESS;
  } catch (...) {
    return fail(XTBLOOM_STATUS_ALLOCATION_FAILED, "failed to create the context");
  }
}

void xtbloom_context_destroy(xtbloom_context_t* context) {
  if (context == nullptr) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(context->device);
  {
    std::lock_guard<std::mutex> lock(context->mutex);   // no transaction in flight
    context->engine.reset();
  }
  if (context->own_stream && context->stream) cudaStreamDestroy(context->stream);
  cudaSetDevice(prev);
  delete context;
}

xtbloom_backend_t xtbloom_context_get_backend(const xtbloom_context_t* context) {
  return context == nullptr ? XTBLOOM_BACKEND_AUTO : XTBLOOM_BACKEND_CUDA;
}

int32_t xtbloom_context_get_device_id(const xtbloom_context_t* context) {
  return context == nullptr ? -1 : context->device;
}

xtbloom_status_t xtbloom_compute(xtbloom_context_t* context, const xtbloom_batch_t* batch,
                                 const xtbloom_compute_options_t* options,
                                 xtbloom_batch_result_t* result) {
  uint32_t flags = 0;
  const xtbloom_status_t st = run(context, batch, options, result, &flags);
  if (st == XTBLOOM_STATUS_SUCCESS && result != nullptr) result->flags = flags;
  return st;
}

xtbloom_status_t xtbloom_request_create(xtbloom_context_t* context, xtbloom_request_t** request) {
  if (request != nullptr) *request = nullptr;
  if (context == nullptr || request == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "NULL argument");
  auto* r = new (std::nothrow) xtbloom_request;
  if (r == nullptr) return fail(XTBLOOM_STATUS_ALLOCATION_FAILED, "failed to allocate a request");
  r->context = context;
  *request = r;
  g_last_error.clear();
  return XTBLOOM_STATUS_SUCCESS;
}

// Validation happens before admission (a rejected submission changes neither
// the request nor any output); an accepted one returns at once with the
// request PENDING, and its transaction runs on the context stream behind any
// earlier one (src/api.cpp:375).
xtbloom_status_t xtbloom_compute_enqueue(xtbloom_context_t* context, const xtbloom_batch_t* batch,
                                         const xtbloom_compute_options_t* options,
                                         const xtbloom_batch_result_t* result,
                                         xtbloom_request_t* request) {
  if (context == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "context is NULL");
  if (request == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "request is NULL");
  if (request->context != context)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "request was created by a different context");
  xtb::ComputeRequest req;
  std::string err;
  const xtbloom_status_t st = validate_and_normalise(batch, options, result, req, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return fail(st, err);
  return submit(context, context->engine.get(), request, batch, options, result, std::move(req));
}

xtbloom_status_t xtbloom_request_query(xtbloom_request_t* request, xtbloom_request_info_t* info) {
  if (request == nullptr || !valid_header(info, offsetof(xtbloom_request_info_t, reserved) + sizeof(uint32_t)))
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "invalid request or info");
  std::lock_guard<std::mutex> lock(request->mu);
  info->state = request->state;
  info->completion_status = request->completion;
  info->result_flags = request->result_flags;
  g_last_error.clear();
  return XTBLOOM_STATUS_SUCCESS;
}

xtbloom_status_t xtbloom_request_wait(xtbloom_request_t* request, xtbloom_request_info_t* info) {
  if (request == nullptr || !valid_header(info, offsetof(xtbloom_request_info_t, reserved) + sizeof(uint32_t)))
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "invalid request or info");
  {
    std::unique_lock<std::mutex> lock(request->mu);
    request->cv.wait(lock, [&] { return request->state != XTBLOOM_REQUEST_PENDING; });
    info->state = request->state;
    info->completion_status = request->completion;
    info->result_flags = request->result_flags;
  }
  request->join();
  g_last_error.clear();
  return XTBLOOM_STATUS_SUCCESS;
}

const char* xtbloom_request_get_error(const xtbloom_request_t* request) {
  if (request == nullptr) return "";
  auto* r = const_cast<xtbloom_request_t*>(request);
  std::lock_guard<std::mutex> lock(r->mu);
  return r->error.c_str();
}

// A pending submission is waited for: its worker must not outlive the request.
void xtbloom_request_destroy(xtbloom_request_t* request) {
  if (request == nullptr) return;
  request->join();
  delete request;
}

// A plan binds the batch's immutable topology and the compute policy, and
// owns its engine (its execution cache): creation validates the request and
// runs it once (FRESH, into scratch outputs) so that every device buffer,
// pinned staging buffer and tuned launch choice of the topology exists
// before the first plan_compute; later plan computes of the same topology
// allocate nothing.  The set-up run leaves no WARM checkpoint.
// (docs/developer-guide/architecture.md "Fixed-topology plans", src/api.cpp:636-770.)
xtbloom_status_t xtbloom_plan_create(xtbloom_context_t* context, const xtbloom_batch_t* batch,
                                     const xtbloom_compute_options_t* options, xtbloom_plan_t** plan) {
  if (plan == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "plan output pointer is NULL");
  *plan = nullptr;
  if (context == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "context is NULL");
  if (batch == nullptr || options == nullptr)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "batch or compute options is NULL");
  if (!valid_header(batch, XTBLOOM_BATCH_V1_SIZE) || !valid_header(options, XTBLOOM_COMPUTE_OPTIONS_V1_SIZE))
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT,
                "batch or compute options are too small or use an unsupported API version");
  if (batch->batch_size <= 0 || batch->total_atoms <= 0 || batch->total_point_charges < 0)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "batch sizes must be positive");
  const size_t B = (size_t)batch->batch_size, N = (size_t)batch->total_atoms;
  const size_t P = (size_t)batch->total_point_charges;
  // scratch outputs of the set-up run (device memory of the context's device)
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(context->device);
  void* scratch = nullptr;
  const size_t bytes = B * 8 + N * 24 + N * 8 + P * 24 + B * 24 + B * 4 + B + B * 4 + 64;
  if (cudaMalloc(&scratch, bytes) != cudaSuccess) {
    cudaGetLastError();
    cudaSetDevice(prev);
    return fail(XTBLOOM_STATUS_ALLOCATION_FAILED, "failed to allocate the plan's set-up outputs");
  }
  cudaSetDevice(prev);
  struct Free {
    void* p;
    int dev;
    ~Free() {
      int d = 0;
      cudaGetDevice(&d);
      cudaSetDevice(dev);
      cudaFree(p);
      cudaSetDevice(d);
    }
  } free_scratch{scratch, context->device};
  char* q = static_cast<char*>(scratch);
  xtbloom_batch_result_t res;
  xtbloom_batch_result_init(&res, sizeof(res));
  auto out = [&](xtbloom_buffer_t& b, size_t n) {
    b.data = n ? q : nullptr;
    b.size_bytes = n;
    b.memory_space = XTBLOOM_MEMORY_CUDA_DEVICE;
    q += (n + 7) & ~size_t(7);
  };
  const uint32_t f = options->flags;
  out(res.energies, (f & XTBLOOM_COMPUTE_ENERGY) ? B * 8 : 0);
  out(res.forces, (f & XTBLOOM_COMPUTE_FORCES) ? N * 24 : 0);
  out(res.atomic_charges, (f & XTBLOOM_COMPUTE_ATOMIC_CHARGES) ? N * 8 : 0);
  out(res.point_charge_forces, (f & XTBLOOM_COMPUTE_POINT_CHARGE_FORCES) ? P * 24 : 0);
  out(res.dipole_moments, (f & XTBLOOM_COMPUTE_DIPOLE_MOMENTS) ? B * 24 : 0);
  out(res.scc_iterations, B * 4);
  out(res.scc_converged, B);
  out(res.per_system_status, B * 4);
  xtb::ComputeRequest req;
  std::string err;
  xtbloom_status_t st = validate_and_normalise(batch, options, &res, req, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return fail(st, err);
  req.warm = false;   // the set-up run starts FRESH whatever the options say
  std::unique_ptr<xtbloom_plan_t> p(new (std::nothrow) xtbloom_plan);
  if (!p) return fail(XTBLOOM_STATUS_ALLOCATION_FAILED, "failed to allocate a plan");
  p->context = context;
  st = capture_topology(batch, req, p->topo, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return fail(st, err);
  p->policy = capture_policy(options, req);
  try {
    cudaSetDevice(context->device);
    p->engine.reset(new xtb::Engine(context->device, context->stream));
    cudaSetDevice(prev);
  } catch (...) {
    cudaSetDevice(prev);
    return fail(XTBLOOM_STATUS_ALLOCATION_FAILED, "failed to create the plan's engine");
  }
  st = execute(context, p->engine.get(), req, nullptr, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return fail(st, err);
  p->engine->invalidate_checkpoint();
  *plan = p.release();
  g_last_error.clear();
  return XTBLOOM_STATUS_SUCCESS;
}

void xtbloom_plan_destroy(xtbloom_plan_t* plan) {
  if (plan == nullptr) return;
  if (plan->context != nullptr) {
    std::lock_guard<std::mutex> lock(plan->context->mutex);   // no transaction of it in flight
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(plan->context->device);
    plan->engine.reset();
    cudaSetDevice(prev);
  }
  delete plan;
}

// The bytes the plan keeps alive for its property set: device buffers of its
// engine and its pinned host staging (graph and stream handles are opaque
// and not counted, as in the reference).
xtbloom_status_t xtbloom_plan_query_workspace(const xtbloom_plan_t* plan, xtbloom_workspace_query_t* q) {
  if (plan == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "plan is NULL");
  if (!valid_header(q, offsetof(xtbloom_workspace_query_t, reserved_v2) + sizeof(uint32_t)))
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT,
                "workspace query is NULL, too small, or uses an unsupported API version");
  if (q->compute_flags != plan->policy.flags)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "compute_flags must equal the plan's flags");
  std::lock_guard<std::mutex> lock(plan->context->mutex);
  q->host_required_bytes = plan->engine->host_bytes();
  q->host_required_alignment = 64;
  q->device_required_bytes = plan->engine->device_bytes();
  q->device_required_alignment = 256;
  g_last_error.clear();
  return XTBLOOM_STATUS_SUCCESS;
}

xtbloom_status_t xtbloom_plan_compute(xtbloom_plan_t* plan, const xtbloom_batch_t* batch,
                                      const xtbloom_compute_options_t* options,
                                      xtbloom_batch_result_t* result) {
  if (plan == nullptr || !plan->engine) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "plan is NULL");
  if (batch == nullptr || options == nullptr || result == nullptr)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "batch, compute options, or batch result is NULL");
  xtb::ComputeRequest req;
  std::string err;
  xtbloom_status_t st = plan_request(plan, batch, options, result, req, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return fail(st, err);
  uint32_t flags = 0;
  st = execute(plan->context, plan->engine.get(), req, &flags, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return fail(st, err);
  result->flags = flags;
  g_last_error.clear();
  return XTBLOOM_STATUS_SUCCESS;
}

xtbloom_status_t xtbloom_plan_compute_enqueue(xtbloom_plan_t* plan, const xtbloom_batch_t* batch,
                                              const xtbloom_compute_options_t* options,
                                              const xtbloom_batch_result_t* result,
                                              xtbloom_request_t* request) {
  if (plan == nullptr || !plan->engine) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "plan is NULL");
  if (request == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "request is NULL");
  if (request->context != plan->context)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "request and plan were created by different contexts");
  if (batch == nullptr || options == nullptr || result == nullptr)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "batch, compute options, or batch result is NULL");
  xtb::ComputeRequest req;
  std::string err;
  const xtbloom_status_t st = plan_request(plan, batch, options, result, req, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return fail(st, err);
  return submit(plan->context, plan->engine.get(), request, batch, options, result, std::move(req));
}

xtbloom_status_t xtbloom_result_owner_options_init(xtbloom_result_owner_options_t* o, size_t size) {
  const xtbloom_status_t st = init_struct(o, size, offsetof(xtbloom_result_owner_options_t, reserved) + 4);
  if (st == XTBLOOM_STATUS_SUCCESS) o->device_id = -1;
  return st;
}

xtbloom_status_t xtbloom_result_owner_create(const xtbloom_result_owner_options_t* o,
                                             xtbloom_result_owner_t** owner) {
  if (owner != nullptr) *owner = nullptr;
  if (owner == nullptr || !valid_header(o, offsetof(xtbloom_result_owner_options_t, reserved) + 4) ||
      o->size_bytes == 0 || o->reserved != 0)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "invalid result owner options");
  // host arenas carry the sentinel device -1, CUDA arenas a real ordinal
  if ((o->memory_space == XTBLOOM_MEMORY_HOST && o->device_id != -1) ||
      (o->memory_space == XTBLOOM_MEMORY_CUDA_DEVICE && o->device_id < 0))
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "result owner device id contradicts its memory space");
  auto* r = new (std::nothrow) xtbloom_result_owner;
  if (r == nullptr) return fail(XTBLOOM_STATUS_ALLOCATION_FAILED, "allocation failed");
  r->space = o->memory_space;
  r->bytes = o->size_bytes;
  if (o->memory_space == XTBLOOM_MEMORY_HOST) {
    r->data = std::malloc(o->size_bytes);
  } else if (o->memory_space == XTBLOOM_MEMORY_CUDA_DEVICE) {
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(o->device_id) != cudaSuccess ||
        cudaMalloc(&r->data, o->size_bytes) != cudaSuccess) {
      cudaGetLastError();
      r->data = nullptr;
    }
    cudaSetDevice(prev);
    r->device = o->device_id;
  } else {
    delete r;
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "unsupported memory space");
  }
  if (r->data == nullptr) {
    delete r;
    return fail(XTBLOOM_STATUS_ALLOCATION_FAILED, "arena allocation failed");
  }
  *owner = r;
  return XTBLOOM_STATUS_SUCCESS;
}

xtbloom_status_t xtbloom_result_owner_buffer(const xtbloom_result_owner_t* owner, xtbloom_buffer_t* b) {
  if (owner == nullptr || b == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "NULL argument");
  b->data = owner->data;
  b->size_bytes = owner->bytes;
  b->memory_space = owner->space;
  b->reserved = 0;
  return XTBLOOM_STATUS_SUCCESS;
}

void xtbloom_result_owner_retain(xtbloom_result_owner_t* owner) {
  if (owner) owner->refs.fetch_add(1);
}

void xtbloom_result_owner_release(xtbloom_result_owner_t* owner) {
  if (owner == nullptr || owner->refs.fetch_sub(1) > 1) return;
  if (owner->space == XTBLOOM_MEMORY_HOST) {
    std::free(owner->data);
  } else {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(owner->device);
    cudaFree(owner->data);
    cudaSetDevice(prev);
  }
  delete owner;
}

}  // extern "C"

namespace {

// DLPack 1.0 structures (the public dlpack.h layout, restated; the reference
// pins the same layout in src/runtime/dlpack_layout.hpp).
struct DlDevice {
  int32_t device_type;   // 1 CPU, 2 CUDA
  int32_t device_id;
};
struct DlDataType {
  uint8_t code;
  uint8_t bits;
  uint16_t lanes;
};
struct DlTensor {
  void* data;
  DlDevice device;
  int32_t ndim;
  DlDataType dtype;
  int64_t* shape;
  int64_t* strides;
  uint64_t byte_offset;
};
struct DlManagedTensor {
  DlTensor dl_tensor;
  void* manager_ctx;
  void (*deleter)(DlManagedTensor*);
};
struct DlPackVersion {
  uint32_t major;
  uint32_t minor;
};
struct DlManagedTensorVersioned {
  DlPackVersion version;
  void* manager_ctx;
  void (*deleter)(DlManagedTensorVersioned*);
  uint64_t flags;
  DlTensor dl_tensor;
};
static_assert(sizeof(DlTensor) == 48, "DLTensor layout");
static_assert(sizeof(DlManagedTensor) == 64, "DLManagedTensor layout");
static_assert(sizeof(DlManagedTensorVersioned) == 80, "DLManagedTensorVersioned layout");

// One exported tensor: the managed struct first (its address is the exported
// pointer and the deleter's argument), then the copied shape.  manager_ctx is
// the arena whose reference the tensor holds.
template <class M>
struct Export {
  M managed;
  int64_t shape[XTBLOOM_DLPACK_MAX_NDIM];
};

template <class M>
void export_deleter(M* self) {
  if (self == nullptr) return;
  auto* owner = static_cast<xtbloom_result_owner_t*>(self->manager_ctx);
  delete reinterpret_cast<Export<M>*>(self);
  xtbloom_result_owner_release(owner);   // never calls back into the importer
}

template <class M>
M* make_export(xtbloom_result_owner_t* owner, const xtbloom_dlpack_view_t* v, uint64_t payload) {
  auto* e = new (std::nothrow) Export<M>{};
  if (e == nullptr) return nullptr;
  DlTensor& t = e->managed.dl_tensor;
  // the offset is folded into data; an empty slice publishes NULL data
  t.data = payload == 0 ? nullptr : static_cast<unsigned char*>(owner->data) + v->byte_offset;
  t.device = owner->space == XTBLOOM_MEMORY_HOST ? DlDevice{1, 0} : DlDevice{2, owner->device};
  t.ndim = v->ndim;
  t.dtype = DlDataType{(uint8_t)v->dtype_code, (uint8_t)v->dtype_bits, (uint16_t)v->dtype_lanes};
  for (int i = 0; i < v->ndim; ++i) e->shape[i] = v->shape[i];
  t.shape = e->shape;
  t.strides = nullptr;   // compact row-major
  t.byte_offset = 0;
  e->managed.manager_ctx = owner;
  e->managed.deleter = &export_deleter<M>;
  return &e->managed;
}

}  // namespace

extern "C" {

xtbloom_status_t xtbloom_result_owner_export_dltensor(const xtbloom_result_owner_t* owner,
                                                      const xtbloom_dlpack_view_t* view, int version,
                                                      void** out_managed) {
  // Every failure leaves *out_managed NULL and the arena's count untouched.
  if (out_managed != nullptr) *out_managed = nullptr;
  if (owner == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "result owner is NULL");
  if (version != 0 && version != 1)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT,
                "DLPack export version must be 0 (legacy) or 1 (versioned)");
  if (view == nullptr || out_managed == nullptr)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "DLPack export view or output pointer is NULL");
  if (view->struct_size < XTBLOOM_DLPACK_VIEW_V1_SIZE || view->api_version != XTBLOOM_API_VERSION)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT,
                "DLPack view is too small or uses an unsupported API version");
  if (view->reserved != 0)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "DLPack view reserved field must be zero");
  if (view->ndim < 0 || view->ndim > XTBLOOM_DLPACK_MAX_NDIM)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "DLPack view ndim must lie between 0 and 8");
  if (view->dtype_lanes != 1)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "DLPack view lanes must be 1");
  // int8/16/32/64, uint8, float32/64: the scalar types the header documents
  const int code = view->dtype_code, bits = view->dtype_bits;
  const bool dtype_ok = (code == 0 && (bits == 8 || bits == 16 || bits == 32 || bits == 64)) ||
                        (code == 1 && bits == 8) || (code == 2 && (bits == 32 || bits == 64));
  if (!dtype_ok)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT,
                "DLPack view uses an unsupported dtype code/bits combination");
  if (view->ndim > 0 && view->shape == nullptr)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "DLPack view with ndim > 0 requires a shape");
  const uint64_t esize = static_cast<uint64_t>(bits / 8);
  uint64_t count = 1;
  bool empty = false;
  for (int i = 0; i < view->ndim; ++i) {
    if (view->shape[i] < 0)
      return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "DLPack view has a negative shape extent");
    const uint64_t ext = static_cast<uint64_t>(view->shape[i]);
    if (ext == 0) empty = true;
    if (empty) continue;   // no elements; keep checking signs only
    if (ext > UINT64_MAX / esize / count)
      return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "DLPack view shape overflows uint64_t");
    count *= ext;
  }
  const uint64_t payload = empty ? 0 : count * esize;
  if (view->byte_offset > owner->bytes || payload > owner->bytes - view->byte_offset)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "DLPack view extends past the arena end");
  if (payload != 0 &&
      (reinterpret_cast<uintptr_t>(owner->data) + view->byte_offset) % esize != 0)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT,
                "DLPack view offset does not preserve the dtype alignment");
  auto* o = const_cast<xtbloom_result_owner_t*>(owner);
  void* m = version != 0 ? static_cast<void*>(make_export<DlManagedTensorVersioned>(o, view, payload))
                         : static_cast<void*>(make_export<DlManagedTensor>(o, view, payload));
  if (m == nullptr)
    return fail(XTBLOOM_STATUS_ALLOCATION_FAILED, "failed to allocate a DLPack managed tensor");
  if (version != 0) {
    auto* mv = static_cast<DlManagedTensorVersioned*>(m);
    mv->version = DlPackVersion{1, 0};
    mv->flags = 0;
  }
  o->refs.fetch_add(1);   // the exported tensor's arena reference
  *out_managed = m;
  return XTBLOOM_STATUS_SUCCESS;
}

xtbloom_status_t xtbloom_b200_debug_fetch(xtbloom_context_t* context, const char* name, int64_t system,
                                          double* out, size_t capacity, size_t* count) {
  if (context == nullptr || name == nullptr || out == nullptr || count == nullptr)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "NULL argument");
  std::lock_guard<std::mutex> lock(context->mutex);
  std::string err;
  const xtbloom_status_t st = context->engine->debug_fetch(name, system, out, capacity, count, err);
  if (st != XTBLOOM_STATUS_SUCCESS) return fail(st, err);
  return st;
}

xtbloom_status_t xtbloom_b200_context_set_execution(xtbloom_context_t* context, int32_t precision,
                                                    double switch_residual, int32_t capture_graphs) {
  if (context == nullptr) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "NULL context");
  if (precision != XTBLOOM_B200_PRECISION_FP64 && precision != XTBLOOM_B200_PRECISION_MIXED)
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "precision must be 0 (FP64) or 1 (mixed)");
  if (!(switch_residual >= 0.0) || !std::isfinite(switch_residual))
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "switch_residual must be finite and >= 0");
  std::lock_guard<std::mutex> lock(context->mutex);
  if (!context->engine) return fail(XTBLOOM_STATUS_BACKEND_UNAVAILABLE, "not a CUDA context");
  context->precision = precision;
  context->switch_residual = switch_residual > 0.0 ? switch_residual : 1e-5;
  context->graphs = capture_graphs != 0;
  context->engine->set_execution(context->precision, context->switch_residual, context->graphs);
  return XTBLOOM_STATUS_SUCCESS;
}

xtbloom_status_t xtbloom_b200_tridiag_eigenvectors_static(const double* diagonal,
                                                          const double* offdiagonal,
                                                          const double* eigenvalues, int32_t n,
                                                          int32_t m, double* vectors,
                                                          double cluster_tolerance,
                                                          void* cuda_stream) {
  if (diagonal == nullptr || eigenvalues == nullptr || vectors == nullptr ||
      (offdiagonal == nullptr && n > 1))
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "NULL argument");
  if (!(cluster_tolerance >= 0.0) || !std::isfinite(cluster_tolerance))
    return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, "cluster_tolerance must be finite and >= 0");
  std::string err;
  const int rc = xtb::static_eigvec_run(diagonal, offdiagonal, eigenvalues, n, m, vectors,
                                        cluster_tolerance > 0.0 ? cluster_tolerance : 2e-7,
                                        static_cast<cudaStream_t>(cuda_stream), err);
  if (rc == 1) return fail(XTBLOOM_STATUS_INVALID_ARGUMENT, err);
  if (rc == 2) return fail(XTBLOOM_STATUS_BACKEND_UNAVAILABLE, err);
  if (rc != 0) return fail(XTBLOOM_STATUS_INTERNAL_ERROR, err);
  return XTBLOOM_STATUS_SUCCESS;
}

}  // extern "C"
