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
};

void launch_setup(const DevTopo& t, const int32_t* list, int count, int max_atoms,
                  int64_t max_pairs, int64_t max_shells, double* cn, double* cn_d4, double* mrad,
                  double* dmrad, double* S, double* D, double* Q, double* H0, double* gam,
                  int64_t total_mat, cudaStream_t stream);

// width 32 or 64 forces the FP64 tile edge; 0 picks 32 when fewer 64-wide
// tiles than SMs.  Both widths form every element identically.
void launch_gemm(const GemmArgs& g, bool transA, bool weighted, int max_tiles, int count,
                 cudaStream_t stream, int width = 0);
void launch_tridiag(const EigArgs& g, int count, int max_n, cudaStream_t stream);
void launch_tridiag_smem(const EigArgs& g, const int32_t* list, int count, int max_n, cudaStream_t stream);
// Register-resident cluster tridiagonalisation for systems with n <= tridiag_reg_max_n().
int tridiag_reg_max_n();
void launch_tridiag_reg(const EigArgs& g, const int32_t* list, int count, int max_n, cudaStream_t stream);
size_t tridiag_smem_bytes(int nl, int nt);
int sm_count();   // multiprocessors of the current device (cached)
void launch_eigvals(const EigArgs& g, int mode, double kt, int count, int max_n, cudaStream_t stream);
void launch_inverse_iteration(const EigArgs& g, int count, int max_n, int want_m, double ortol_rel,
                              cudaStream_t stream);
void launch_backtransform(const EigArgs& g, const int32_t* list, int count, int max_n, int mcap,
                          cudaStream_t stream);
void launch_backtransform_wy(const EigArgs& g, int count, int max_n, int max_m, int want_m,
                             cudaStream_t stream);
size_t backtransform_wy_bytes(int n, int m);
void launch_lowdin_weights(const EigArgs& g, int32_t* status, int count, cudaStream_t stream);

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
