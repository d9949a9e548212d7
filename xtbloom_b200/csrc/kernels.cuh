// Kernel argument blocks and host launch entry points of the CUDA path.
#pragma once

#include "common.cuh"

namespace xtb {

struct GemmArgs {
  const int32_t* list;     // active systems (blockIdx.y -> system)
  const int32_t* nao;      // leading dimension of every matrix of a system
  const int32_t* dm;       // rows of C
  const int32_t* dn;       // columns of C
  const int32_t* dk;       // contraction length
  const double* A;
  const int64_t* offA;
  const double* B;
  const int64_t* offB;
  double* C;
  const int64_t* offC;
  const double* w;         // per-k weight (weighted form)
  const int64_t* offW;
  int32_t sym;             // C is symmetric: compute the lower tiles, mirror them
  const uint8_t* prec;     // per system: 0 = split-precision (3xTF32) tile, else FP64; NULL = FP64
  const int32_t* prec_of;  // list entry (channel) -> index into prec; NULL = the entry itself
  const uint8_t* only;     // per list entry id: 0 = skip (its CTAs return at once); NULL = all
  int32_t umma;            // split-precision tiles run in k_gemm_umma: k_gemm skips those systems
  int32_t* fault;          // set to 1 when a tensor-core wait of k_gemm_umma ran out
};

struct EigArgs {
  const int32_t* list;
  const int32_t* nao;
  const int64_t* mat_off;
  const int64_t* ao_off;
  double* A;          // matrix to tridiagonalise (destroyed: holds reflectors)
  double* d;
  double* e;
  double* tau;
  double* eig;        // eigenvalues (ao-indexed)
  double* occ;        // occupations (ao-indexed); Loewdin weights in setup
  double* occ_eps;    // occupation * eigenvalue
  double* entropy;    // per system
  int32_t* nvec;      // per system: number of eigenvectors formed
  double* Z;          // eigenvector-major n x n blocks
  double* scratch;    // inverse-iteration workspace
  const int64_t* scratch_off;
  const double* nel_a;
  const double* nel_b;
  // per channel: 0 = skip (every CTA of the channel returns at once); NULL = all
  const uint8_t* only;
  // nonzero: inverse iteration and the back-transform form all n eigenvectors
  // (nvec still counts the occupied ones the density needs)
  int32_t all_vectors;
};

struct SccArgs {
  DevTopo t;
  const int32_t* list;
  int32_t count;
  // state (mixed input) and raw populations
  double* qsh;        // per shell
  double* dip;        // 3 per atom
  double* qp;         // 6 per atom
  double* pop_sh;     // accumulated sum_mu P S per shell (zeroed each iteration)
  double* pop_dip;
  double* pop_qp;
  double* e_core;     // per system Tr(P H0)
  // potentials
  double* vsh;        // per shell (scalar shell + atomic potential)
  double* vd;
  double* vq;
  // spin polarisation (unrestricted systems): magnetisation m = pop_beta -
  // pop_alpha per shell (mixed input), its potential W m, and the raw
  // magnetisation populations of P_alpha - P_beta
  double* qmag;
  double* vmag;
  double* pop_mag;    // per shell: sum (P_a - P_b) S
  double* pop_mdip;   // 3 per atom
  double* pop_mqp;    // 6 per atom
  const double* Pm;   // P_alpha - P_beta at the system's matrix offset
  // per-channel workspace (the eigensolver's scratch, free after the
  // back-transform): partial column sums of the split Mulliken reduction
  double* work;
  const int64_t* work_off;
  // spin channels: channel c of an active list -> system, sign (0 restricted,
  // +1 alpha, -1 beta), matrix offset of its Hamiltonian
  const int32_t* clist;
  int32_t ccount;
  const int32_t* ch_sys;
  const int32_t* ch_sign;
  const int64_t* ch_mat;
  // geometry caches
  const double* gam;
  const double* mrad;
  const double* cn_d4;
  // matrices
  const double* S;
  const double* D;
  const double* Q;
  const double* H0;
  double* H;
  const double* P;
  int64_t total_mat;
  double* pot_acc;    // per atom: atomic potential between the two potential kernels
  // per system energies / status
  const double* entropy;
  double* free_energy;
  double* terms;      // 8 per system: core, es2, es3, aes2, d4, -kTS, rep, atm
  int32_t* iterations;
  int32_t* status;
  uint8_t* converged;
  // Broyden state
  double* mx_cur;
  double* mx_prev;
  double* mx_res;
  double* mx_df;      // memory x dim per system, at vec_off * memory
  double* mx_u;
  double* mx_omega;   // memory per system
  int32_t memory;
  double damping;
  double ctol, etol, kt;
  int32_t max_iter;
  // precision ladder: prec[s] = 0 while system s iterates with split-precision
  // GEMMs, 1 once it iterates in FP64 (a system converges only on an FP64
  // iteration); it switches when its residual falls below prec_switch.
  // WARM start: the retained converged state (shell charges, dipoles,
  // quadrupoles; magnetisation, its dipoles and quadrupoles) seeds the SCC
  const double* ck_qsh;
  const double* ck_dip;
  const double* ck_qp;
  const double* ck_qmag;
  const double* ck_mdip;
  const double* ck_mqp;
  uint8_t* prec;
  double prec_switch;
  int32_t* split_iters;   // per system: iterations run with split-precision GEMMs
  int32_t* gate_hits;     // per system: FP64 iterations that met the ordinary gate (split form)
  double* last_rms;       // per system: charge residual (rms) of the latest iteration
};

// Split-precision form: FP64 iterations continue until the residual and the
// energy change are this much below the requested tolerances, for at most
// kMixedExtra iterations past the ordinary gate.
constexpr double kMixedTighten = 1e-2;
constexpr int kMixedExtra = 10;
// A system whose residual has not fallen below the precision switch after
// this many split-precision iterations continues in FP64.
constexpr int kMaxSplitIterations = 40;

void launch_setup(const DevTopo& t, const int32_t* list, int count, int max_atoms,
                  int64_t max_pairs, int64_t max_shells, double* cn, double* cn_d4, double* mrad,
                  double* dmrad, double* S, double* D, double* Q, double* H0, double* gam,
                  int64_t total_mat, cudaStream_t stream);

// width 32 or 64 forces the FP64 tile edge; 0 picks 32 when fewer 64-wide
// tiles than SMs.  Both widths form every element identically.
void launch_gemm_umma(const GemmArgs& g, bool transA, bool weighted, int tm, int count,
                      cudaStream_t stream);
void launch_gemm(const GemmArgs& g, bool transA, bool weighted, int max_tiles, int count,
                 cudaStream_t stream, int width = 0);
void launch_tridiag_smem(const EigArgs& g, const int32_t* list, int count, int max_n, cudaStream_t stream);
// Register-resident cluster tridiagonalisation for systems with n <= tridiag_reg_max_n().
int tridiag_reg_max_n();
void launch_tridiag_reg(const EigArgs& g, const int32_t* list, int count, int max_n, cudaStream_t stream);
size_t tridiag_smem_bytes(int nl, int nt);
int sm_count();   // multiprocessors of the current device (cached)
// max_levels: the most eigenvalues a system of the launch needs in the SCC
// (mode 0): its occupied levels and eight above them.
void launch_eigvals(const EigArgs& g, int mode, double kt, int count, int max_n, int max_levels,
                    cudaStream_t stream);
void launch_inverse_iteration(const EigArgs& g, int count, int max_n, int want_m, double ortol_rel,
                              cudaStream_t stream);
void launch_backtransform_rows(const EigArgs& g, int count, int max_n, int want_m, cudaStream_t stream);
// Compact-WY back-transform.  factored: the T factors were formed already by
// launch_wy_factor (which needs only the reflectors, so it can run beside the
// eigenvalues and the inverse iteration); otherwise they are formed first.
void launch_wy_factor(const EigArgs& g, int count, int max_n, cudaStream_t stream);
void launch_backtransform_wy(const EigArgs& g, int count, int max_n, int max_m, int want_m,
                             cudaStream_t stream, bool factored = false);
// Per-channel scratch of the eigensolver, in doubles: the inverse
// iteration's work arrays (5 n per thread of a 128-thread block), then the
// T factors of the compact-WY blocks (32 x 32 per block of 32 reflectors)
// at wy_t_offset(n), apart from them so that both can be live at once.
__host__ __device__ inline int64_t wy_t_offset(int64_t n) { return 128 * 5 * n; }
__host__ __device__ inline int64_t eig_scratch(int64_t n) {
  return wy_t_offset(n) + ((n > 2 ? n - 2 : 0) + 31) / 32 * 32 * 32;
}
size_t backtransform_wy_bytes(int n, int m);
void launch_lowdin_weights(const EigArgs& g, int32_t* status, int count, cudaStream_t stream);

// ---------------------------------------------------------------------------
// Warm-started eigensolver of the SCC (k_refine.cu): from the second SCC
// iteration on, a channel's eigenvector columns V of the previous iteration
// are refined for the new matrix A by the matrix-multiplication iteration of
// Ogita and Aishima, which only needs the products U = A V, S = V^T U and
// G = V^T V and the update V (I + E); see k_refine.cu.
// ---------------------------------------------------------------------------
enum WarmPhase : uint8_t { kWarmCold = 0, kWarmActive = 1, kWarmFinal = 2, kWarmDone = 3, kWarmFailed = 4 };

struct RefineArgs {
  const int32_t* list;     // active channels
  int32_t count;
  const int32_t* nao;
  const int64_t* mat_off;
  const int64_t* ao_off;
  const int32_t* ch_sys;   // channel -> system
  const double* nel_a;     // per channel: electrons of the two Fermi populations
  const double* nel_b;
  double kt;
  const double* Sm;        // V^T A V
  const double* G;         // V^T V
  double* Ep;              // I + E
  double* V;               // eigenvector columns (valid where wstate == 1)
  const double* Vt;        // V (I + E) of the step
  const double* Zrows;     // eigenvector rows of the Householder path
  double* eig;             // Rayleigh quotients of the columns (ao-indexed)
  double* occ;             // occupations, occupation * Rayleigh quotient, count of
  double* occ_eps;         // occupied columns and entropy of refined channels
  int32_t* nvec;
  double* entropy;
  uint8_t* wstate;         // per channel: 1 = V holds the eigenvectors of an earlier iteration
  uint8_t* phase;          // per channel WarmPhase of this iteration
  uint8_t* m_step;         // mask: channels whose U, S, G products run in this step
  uint8_t* m_apply;        // mask: channels whose V (I + E) product runs in this step
  uint8_t* m_cold;         // mask: channels the Householder path solves in this iteration
  uint8_t* m_warm;         // mask: channels refined in this iteration
  unsigned long long* emax;   // per channel: max |E| of the step (bits of a nonnegative double)
  int32_t* fail;           // per channel: failure flag of the step
  int32_t* arrive;         // per channel: CTAs of the step that finished
  double* bounds;          // per channel and part: Gershgorin bounds of the occupation blocks
  int32_t* stats;          // [iteration][8] counters (attempted, done at step 1..3+, failed, unfinished)
  const int32_t* iterations;   // per system: SCC iterations done
  const uint8_t* prec;     // per system split-precision flag (0 = split), NULL = FP64
  const double* last_rms;  // per system: charge residual of the previous SCC iteration
  double final_rms;        // below this residual a system is in its final SCC iterations
  int32_t warm_from;       // first SCC iteration that refines
  int32_t step;            // 0-based step of this SCC iteration
  // convergence thresholds of max |E|: split-precision iterations, FP64
  // iterations on the approach, FP64 iterations near the fixed point
  double theta_split, theta, theta_final;
};

constexpr int kRefineMaxParts = 16;

void launch_warm_begin(const RefineArgs& r, cudaStream_t stream);
void launch_refine_update(const RefineArgs& r, int max_n, int parts, cudaStream_t stream);
void launch_refine_apply(const RefineArgs& r, int max_n, bool last, cudaStream_t stream);
void launch_vectors_from_rows(const RefineArgs& r, int max_n, cudaStream_t stream);

void launch_sad_init(const SccArgs& a, cudaStream_t stream);
void launch_warm_init(const SccArgs& a, cudaStream_t stream);
void launch_potential(const SccArgs& a, const double* qsh, const double* dip, const double* qp,
                      int max_atoms, int max_shells, cudaStream_t stream);
void launch_fock(const SccArgs& a, int max_n, cudaStream_t stream);
void launch_mulliken(const SccArgs& a, int max_n, cudaStream_t stream);
void launch_energy_mixer(const SccArgs& a, int max_atoms, int max_shells, int max_dim,
                         int first_iteration, cudaStream_t stream);
void launch_compact(const int32_t* order, int nsys, const int32_t* status, const uint8_t* converged,
                    const int32_t* iterations, int max_iter, int32_t* list, int32_t* count,
                    cudaStream_t stream);

struct ForceArgs {
  DevTopo t;
  const int32_t* list;
  int32_t count;
  const double* cn;
  const double* cn_d4;
  const double* mrad;
  const double* dmrad;
  const double* S;
  const double* P;
  const double* W;
  const double* vsh;
  const double* vd;
  const double* vq;
  const double* vmag;     // spin potential per shell (unrestricted systems)
  const double* Pm;       // P_alpha - P_beta (unrestricted systems)
  const double* qsh;
  const double* dip;
  const double* qp;
  const double* gam;
  double* grad;       // 3 per atom (dE/dR), accumulated
  double* acn;        // dE/dCN (dexp) per atom, accumulated
  double* acn_d4;     // dE/dCN (D4) per atom, accumulated
  double* terms;      // per-system energy terms (rep, atm written)
  int32_t want_grad;
  // work arrays free once the SCC has ended: the D4 three-body pair tables
  // (n^2 per system at the matrix offsets) and per-system scratch
  double* atm_c6;
  double* atm_dc6;
  double* work;
  const int64_t* work_off;
};

void launch_force_pairs(const ForceArgs& f, int64_t max_pairs, cudaStream_t stream);

// external point charges (k_pc.cu)
void launch_pc_potential(const DevTopo& t, const int32_t* list, int count, double* vpc,
                         cudaStream_t stream);
void launch_pc_forces(const DevTopo& t, const int32_t* list, int count, const double* qsh,
                      double* grad, double* pc_grad, double* pc_dq, cudaStream_t stream);
void launch_pc_publish(const DevTopo& t, const int32_t* status, int nsys, const double* pc_grad,
                       double* out, cudaStream_t stream);
void launch_classical(const ForceArgs& f, int max_atoms, int max_shells, cudaStream_t stream);
void launch_cn_chain(const ForceArgs& f, int max_atoms, cudaStream_t stream);

}  // namespace xtb
