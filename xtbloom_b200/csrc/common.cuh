// Shared device-side definitions of the xtbloom_b200 CUDA path.
//
// Data layout in HBM (all FP64 unless stated; "global" = batch-wide index):
//   per system s : atom/shell/AO ranges, packed matrix offset mat_off[s] = sum n_t^2,
//                  shell-matrix offset gam_off[s] = sum k_t^2, mixer vector offset.
//   per atom     : Z, position (3), element constants gathered at topology time.
//   per shell    : owning atom, l, first AO (system-local), primitive range, level, kcn,
//                  shell polynomial, Slater exponent, hardness, third-order gamma,
//                  reference occupation.
//   per AO       : owning shell and atom (global indices).
//   matrices     : row-major n_s x n_s blocks at mat_off[s]; dipole and quadrupole
//                  integrals are component-major (3 resp. 6 full packed arrays).
#pragma once

#include <cstdint>
#include <map>
#include <mutex>
#include <utility>

#include <cuda_runtime.h>

namespace xtb {

// Lets `func` use as much dynamic shared memory as the current device allows
// beside its static shared memory; returns that limit in bytes.  The
// attribute belongs to the device, so it is set once per (kernel, device)
// and remembered: contexts on several devices of one process each get it.
template <class F>
inline size_t allow_max_dynamic_smem(F func) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  int dev = 0;
  cudaGetDevice(&dev);
  const std::pair<const void*, int> key((const void*)func, dev);
  std::lock_guard<std::mutex> lock(mu);
  const auto it = done.find(key);
  if (it != done.end()) return it->second;
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa{};
  cudaFuncGetAttributes(&fa, func);
  const size_t cap = (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
  cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap);
  done.emplace(key, cap);
  return cap;
}

constexpr int kMaxD4Refs = 7;
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kSqrtPi3 = 5.5683279968317061;   // pi^(3/2)
constexpr double kIntegralCutoff = 25.0;          // Gaussian-product screen

// Model constants shared by all kernels (set once per context).
struct ModelConstants {
  int32_t gfn1;   // 0: GFN2-xTB, 1: GFN1-xTB (the fields below hold that model's values)
  double wexp, enscale, kpol, pair_scale_default;
  double shell_pair_scale[9];
  double rep_kexp, rep_klight;
  double es3_scale[3];
  double mp_kexp, mp_shift, mp_rmax;
  double d4_a1, d4_a2, d4_s6, d4_s8, d4_s9;
  // GFN1: D3(BJ) dispersion, halogen-bond correction, exponential CN
  double d3_a1, d3_a2, d3_s6, d3_s8;
  double xb_damping, xb_radius_scale;
  double cn_steepness;
};

constexpr int kD3MaxRefs = 5;       // D3 reference systems per element
constexpr int kD3Refs = 237;        // all D3 references

struct DevTopo {
  ModelConstants m;
  int32_t nsys;
  int64_t total_atoms, total_shells, total_aos;
  // per system
  const int64_t* atom_off;
  const int64_t* shell_off;
  const int64_t* ao_off;
  const int64_t* mat_off;
  const int64_t* gam_off;
  const int64_t* vec_off;
  const int32_t* nao;
  const double* nel_a;
  const double* nel_b;
  const double* qmol;
  const int32_t* nch;         // spin channels (1 restricted, 2 unrestricted)
  const int32_t* beta_ch;     // channel id of the beta channel (-1 for restricted systems)
  const double* efield;       // 3 per system: uniform electric field; NULL when no system has one
  const double* resp_b;       // per atom: caller potential shift b (charge response); NULL if none
  const double* resp_A;       // per system: row-major symmetric atoms x atoms block A
  const int64_t* resp_off;    // nsys + 1 offsets into resp_A
  // per atom
  const int32_t* Z;
  const int32_t* atom_sh;     // total_atoms + 1
  const double* pos;          // 3 per atom
  const double* at_en;        // GFN2 electronegativity
  const double* at_rad;       // H0 polynomial radius (bohr)
  const double* at_rcov;      // double-exponential CN radius (bohr)
  const double* at_mprad;
  const double* at_mpvcn;
  const double* at_dk;
  const double* at_qk;
  const double* at_rep_sa;    // sqrt(arep)
  const double* at_rep_z;     // repulsion zeff
  const double* d4_rcov;
  const double* d4_en;
  const double* d4_zeff;
  const double* d4_eta;
  const double* d4_r4r2;
  const int32_t* d4_roff;
  const int32_t* d4_rcnt;
  // GFN1: halogen-bond strength per atom, pair scaling of H0 (86 x 86),
  // D3 reference tables (references per element, their offsets and CNs, the
  // C6 of every pair of references, <r^4>/<r^2> per element)
  const double* at_xbond;
  const double* kpair;
  const int32_t* d3_rcnt;
  const int32_t* d3_roff;
  const double* d3_ref_cn;
  const double* d3_c6;
  const double* d3_r4r2;
  // per shell
  const int32_t* sh_val;      // 1 for valence shells (GFN1 H0 pair scaling)
  const int32_t* sh_atom;
  const int32_t* sh_l;
  const int32_t* sh_ao;       // first AO of the shell, system-local
  const int32_t* sh_p0;
  const int32_t* sh_np;
  const double* sh_level;
  const double* sh_kcn;
  const double* sh_shpoly;
  const double* sh_zeta;
  const double* sh_eta;
  const double* sh_g3;
  const double* sh_refocc;
  const double* sh_spinw;     // 3 per shell: spin coupling W(shell, k-th shell of its atom)
  const double* p_alpha;
  const double* p_coeff;
  // per AO (global)
  const int32_t* ao_sh;
  const int32_t* ao_at;
  // D4 reference tables
  const double* ref_cn;
  const double* ref_q;
  const int32_t* ref_ng;
  const double* ref_c6;       // 262 x 262
  int32_t ref_count;
  // external point charges (per system ranges; empty when pc_off is null)
  const int64_t* pc_off;      // nsys + 1
  const double* pc_pos;       // 3 per charge
  const double* pc_q;
  const double* pc_gam;
  const double* vpc;          // per shell: potential of the point charges
};

// Per-system energy terms (terms[kTermCount * s + k]).
enum TermIndex : int {
  kTermCore = 0, kTermEs2 = 1, kTermEs3 = 2, kTermAes2 = 3, kTermD4 = 4, kTermEntropy = 5,
  kTermRep = 6, kTermAtm = 7, kTermPc = 8, kTermSpin = 9, kTermField = 10, kTermResp = 11,
  kTermDisp3 = 12, kTermXb = 13, kTermCount = 14
};

__device__ __forceinline__ double logistic(double x) {
  if (x >= 0.0) {
    const double e = exp(-x);
    return 1.0 / (1.0 + e);
  }
  const double e = exp(x);
  return e / (1.0 + e);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum; all threads receive the result.  scratch needs 33 doubles.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double t = lane < nw ? scratch[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) scratch[32] = t;
  }
  __syncthreads();
  return scratch[32];
}

__device__ __forceinline__ double block_max(double v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double t = lane < nw ? scratch[lane] : -1.7976931348623157e308;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
    if (lane == 0) scratch[32] = t;
  }
  __syncthreads();
  return scratch[32];
}

// Gradient accumulators (dE/dR, dE/dCN and the shared-memory partial sums of
// the force kernels) are 64-bit two's-complement fixed point with 2^-40
// units: every contribution is rounded once to the grid, and the integer
// atomic adds that sum them are associative, so the result does not depend
// on the order in which threads arrive: forces are bitwise reproducible
// from run to run.  The grid (9.1e-13) and range (|sum| < 2^23) are far
// below and above what a gradient needs.
constexpr double kFixOne = 1099511627776.0;   // 2^40
__device__ __forceinline__ void fix_add(double* acc, double v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(acc),
            static_cast<unsigned long long>(__double2ll_rn(v * kFixOne)));
}
// Adds one fixed-point accumulator (a partial sum) to another.
__device__ __forceinline__ void fix_merge(double* acc, const double& part) {
  atomicAdd(reinterpret_cast<unsigned long long*>(acc), *reinterpret_cast<const unsigned long long*>(&part));
}
__device__ __forceinline__ double fix_value(const double& acc) {
  return static_cast<double>(*reinterpret_cast<const long long*>(&acc)) * (1.0 / kFixOne);
}

// Length of a system's charge block in the Broyden vector: shell charges,
// atomic dipoles and quadrupoles (GFN2), shell charges only (GFN1).  An
// unrestricted system carries a magnetisation block of the same length.
__device__ __forceinline__ int charge_block(const DevTopo& t, int ns, int na) {
  return t.m.gfn1 ? ns : ns + 9 * na;
}

// Per-system status codes mirror the public per_system_status values.
enum SysStatus : int32_t { kOk = 0, kNotConverged = 7, kEigenFailed = 8, kInternal = 6 };

}  // namespace xtb
