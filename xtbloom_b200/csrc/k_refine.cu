// Warm-started eigensolver of the SCC: the eigenvectors of the previous SCC
// iteration, refined for the new orthogonalised Hamiltonian A by the
// matrix-multiplication iteration of Ogita and Aishima ("Iterative refinement
// for symmetric eigenvalue decomposition", Japan J. Indust. Appl. Math. 35,
// 1007-1035, 2018).  With V the current eigenvector columns,
//   S = V^T A V,  G = V^T V  (batched GEMMs after U = A V),
//   lambda_i = S_ii / G_ii,
//   E_ij = (S_ij - lambda_j G_ij) / (lambda_j - lambda_i)   (i != j),
//   E_ii = (1 - G_ii) / 2,
//   V <- V (I + E)  (one more GEMM),
// the first-order solution of (I + E)^T G (I + E) = I and (I + E)^T S (I + E)
// diagonal.  What the SCC needs of an iteration's eigenproblem is the density
// P = sum_i f_i c_i c_i^T: it depends on V only through the invariant
// subspaces of equal occupation (doubly, singly and un-occupied levels), and
// their separation is the only part of the iteration that must converge.
// Pairs of columns in different occupation blocks take the step above, whose
// denominators are at least the frontier-orbital gap; pairs inside a block
// take it only where it is small (|E_ij| <= 0.1), and otherwise (near
// degenerate levels, typical of long chains, where a first-order step is not
// a contraction) keep their orthogonality correction alone, -G_ij / 2.  The
// channel is done once max |E| over the cross-block and orthogonality terms
// is below theta (1e-7 in FP64; the separation error left is far smaller).
//
// The occupations of a refined channel are those of the block it sits in,
// which equal the Fermi-Dirac occupations to the last bit when the blocks are
// separated by more than kRefineGapKt k_B T: Gershgorin bounds of each
// block's rows of S check this in every step.  The energy-weighted density of
// the forces needs the eigenpairs themselves, so the engine solves the last
// iteration of a refined system again with the Householder path (the matrix
// A is kept for that).
//
// The reference diagonalises every SCC iteration from scratch (LAPACK dsyevd,
// model/gfn2/eigensolver.cpp:1221-1254; cuSOLVER syevj/syevd on its GPU path,
// backends/cuda/gfn2_eigensolver.cu:2332-2360).  A channel whose refinement
// fails (a cross-block step above kRefineMaxStep, blocks closer than the gap
// bound, fractional electron counts, non-finite values) or does not finish
// within the SCC iteration's steps is solved by the Householder path in the
// same iteration; so is every channel's first iteration.  The kernels here
// keep the per-channel phases and masks that route channels between the two
// paths, so the launch sequence of an SCC iteration does not depend on the
// data and is captured into CUDA graphs whole.
#include <cfloat>

#include "kernels.cuh"

namespace xtb {

constexpr double kRefineMaxStep = 0.25;     // largest cross-block |E_ij| of a step
constexpr double kRefineInBlock = 0.1;      // largest in-block |E_ij| taken as a rotation
constexpr double kRefineTinyGap = 1e-12;    // relative gap below which levels count as equal
constexpr double kRefineGapKt = 100.0;      // block separation that makes occupations exact
constexpr int kStatSlots = 8;

__device__ __forceinline__ void stat_add(const RefineArgs& r, int c, int slot) {
  if (r.stats == nullptr) return;
  const int it = min(r.iterations[r.ch_sys[c]], 255);
  atomicAdd(&r.stats[kStatSlots * it + slot], 1);
}

constexpr int kRefineBoundSlots = 9;

__device__ __forceinline__ void shared_max(double* p, double v) {
  unsigned long long* a = reinterpret_cast<unsigned long long*>(p);
  unsigned long long old = *a, assumed;
  do {
    assumed = old;
    if (__longlong_as_double((long long)assumed) >= v) return;
    old = atomicCAS(a, assumed, (unsigned long long)__double_as_longlong(v));
  } while (old != assumed);
}

__device__ __forceinline__ void shared_min(double* p, double v) {
  unsigned long long* a = reinterpret_cast<unsigned long long*>(p);
  unsigned long long old = *a, assumed;
  do {
    assumed = old;
    if (__longlong_as_double((long long)assumed) <= v) return;
    old = atomicCAS(a, assumed, (unsigned long long)__double_as_longlong(v));
  } while (old != assumed);
}

// Occupation block boundaries of channel c: levels below k1 hold both
// populations, levels k1..k2-1 one of them; false when a count is fractional.
__device__ __forceinline__ bool occupation_blocks(const RefineArgs& r, int c, int n, int& k1, int& k2) {
  const double a = r.nel_a[c], b = r.nel_b[c];
  if (a != floor(a) || b != floor(b) || a < 0.0 || b < 0.0 || a > n || b > n) return false;
  k1 = (int)fmin(a, b);
  k2 = (int)fmax(a, b);
  return true;
}

// Phase of every active channel for this SCC iteration: refine when its V
// holds the eigenvectors of an earlier iteration, else the Householder path.
__global__ void k_warm_begin(RefineArgs r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.count) return;
  const int c = r.list[i];
  int k1 = 0, k2 = 0;
  const bool warm = r.wstate[c] == 1 && r.iterations[r.ch_sys[c]] >= r.warm_from &&
                    occupation_blocks(r, c, r.nao[c], k1, k2);
  r.phase[c] = warm ? kWarmActive : kWarmCold;
  r.m_step[c] = warm ? 1 : 0;
  r.m_apply[c] = 0;
  r.m_cold[c] = warm ? 0 : 1;
  r.m_warm[c] = 0;
  r.emax[c] = 0ull;
  r.fail[c] = 0;
  r.arrive[c] = 0;
  if (warm) stat_add(r, c, 0);
}

// One step's correction I + E of a channel: grid (parts, channels), a warp
// per row, part p taking rows p, p + parts, ...; the last part of a channel
// to finish decides its phase.
__global__ void __launch_bounds__(256) k_refine_update(RefineArgs r, int parts) {
  extern __shared__ double lam[];
  const int c = r.list[blockIdx.y];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  if (r.phase[c] != kWarmActive) {
    // masks of channels that do not refine are cleared here, so that no
    // stale mask of an earlier step selects them in the products that follow
    if (blockIdx.x == 0 && tid == 0) r.m_apply[c] = 0;
    return;
  }
  const int n = r.nao[c];
  int k1 = 0, k2 = 0;
  occupation_blocks(r, c, n, k1, k2);   // checked by k_warm_begin
  const int64_t mo = r.mat_off[c];
  const double* S = r.Sm + mo;
  const double* G = r.G + mo;
  double* Ep = r.Ep + mo;
  __shared__ double red[33];
  // per block b: largest and smallest Rayleigh quotient, sum of squares of
  // the off-diagonal elements of S inside the block (s_max[b], s_min[b], s_ss[b])
  __shared__ double s_max[3], s_min[3], s_ss[3];
  __shared__ int s_bad;
  double amax = 0.0;
  for (int i = tid; i < n; i += blockDim.x) {
    const double l = S[(int64_t)i * n + i] / G[(int64_t)i * n + i];
    lam[i] = l;
    amax = fmax(amax, fabs(l));
  }
  if (tid < 3) {
    s_max[tid] = -DBL_MAX;
    s_min[tid] = DBL_MAX;
    s_ss[tid] = 0.0;
  }
  if (tid == 0) s_bad = 0;
  const double tiny = kRefineTinyGap * fmax(block_max(amax, red), 1.0);   // synchronises
  double emx = 0.0;
  bool bad = false;
  for (int i = blockIdx.x + parts * warp; i < n; i += parts * nw) {
    const int bi = i < k1 ? 0 : (i < k2 ? 1 : 2);
    const double li = lam[i];
    double ss = 0.0;   // sum of S_ij^2 over the other columns of i's block
    for (int j = lane; j < n; j += 32) {
      const int64_t ij = (int64_t)i * n + j;
      const double g = G[ij];
      const int bj = j < k1 ? 0 : (j < k2 ? 1 : 2);
      double e;
      bool counts = true;
      if (i == j) {
        e = 0.5 * (1.0 - g);
      } else {
        const double sij = S[ij];
        const double num = sij - lam[j] * g;
        const double den = lam[j] - li;
        if (bi != bj) {
          if (fabs(den) > tiny) {
            e = num / den;
            if (!(fabs(e) <= kRefineMaxStep)) bad = true;
          } else {
            e = 0.0;
            bad = true;
          }
        } else {
          ss = fma(sij, sij, ss);
          if (fabs(den) > tiny && fabs(num) <= kRefineInBlock * fabs(den)) {
            e = num / den;
            counts = false;   // a rotation inside a block: the density does not see it
          } else {
            e = -0.5 * g;
          }
        }
      }
      if (!isfinite(e)) {
        e = 0.0;
        bad = true;
      }
      if (counts) emx = fmax(emx, fabs(e));
      Ep[ij] = (i == j ? 1.0 : 0.0) + e;
    }
    ss = warp_sum(ss);
    if (lane == 0) {
      atomicAdd(&s_ss[bi], ss);   // the order only moves the bound, not a result
      shared_max(&s_max[bi], li);
      shared_min(&s_min[bi], li);
    }
  }
  if (bad) s_bad = 1;
  emx = block_max(emx, red);   // synchronises (s_bad and the block sums are complete after it)
  if (tid == 0) {
    double* bnd = r.bounds + ((int64_t)c * kRefineMaxParts + blockIdx.x) * kRefineBoundSlots;
    for (int b = 0; b < 3; ++b) {
      bnd[b] = s_max[b];
      bnd[3 + b] = s_min[b];
      bnd[6 + b] = s_ss[b];
    }
    atomicMax(&r.emax[c], (unsigned long long)__double_as_longlong(emx));
    if (s_bad) atomicOr(&r.fail[c], 1);
    __threadfence();
    if (atomicAdd(&r.arrive[c], 1) == parts - 1) {
      __threadfence();
      // Weyl: every eigenvalue of a block's matrix lies within the Frobenius
      // norm of its off-diagonal part of the block's Rayleigh quotients
      const volatile double* vb = r.bounds + (int64_t)c * kRefineMaxParts * kRefineBoundSlots;
      double mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX}, mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
      double sq[3] = {0.0, 0.0, 0.0};
      for (int p = 0; p < parts; ++p)
        for (int b = 0; b < 3; ++b) {
          mx[b] = fmax(mx[b], vb[kRefineBoundSlots * p + b]);
          mn[b] = fmin(mn[b], vb[kRefineBoundSlots * p + 3 + b]);
          sq[b] += vb[kRefineBoundSlots * p + 6 + b];
        }
      const double need = kRefineGapKt * r.kt;
      // consecutive non-empty occupation blocks must be separated
      const int size[3] = {k1, k2 - k1, n - k2};
      bool sep = true;
      int prev = -1;
      for (int b = 0; b < 3; ++b) {
        if (size[b] == 0) continue;
        if (prev >= 0) sep = sep && (mn[b] - sqrt(sq[b])) - (mx[prev] + sqrt(sq[prev])) > need;
        prev = b;
      }
      const double e = __longlong_as_double((long long)atomicAdd(&r.emax[c], 0ull));
      const bool failed = atomicAdd(&r.fail[c], 0) != 0;
      const int sy = r.ch_sys[c];
      const bool split = r.prec != nullptr && r.prec[sy] == 0;
      const double theta = split ? r.theta_split
                                 : (r.last_rms != nullptr && r.last_rms[sy] < r.final_rms ? r.theta_final
                                                                                            : r.theta);
      uint8_t ph = kWarmActive;
      if (failed) ph = kWarmFailed;
      else if (e <= theta) ph = sep ? kWarmFinal : kWarmFailed;
      r.phase[c] = ph;
      r.m_apply[c] = (ph == kWarmActive || ph == kWarmFinal) ? 1 : 0;
      r.emax[c] = 0ull;
      r.fail[c] = 0;
      r.arrive[c] = 0;
      if (ph == kWarmFinal) stat_add(r, c, 1 + min(r.step, 2));
      if (ph == kWarmFailed) stat_add(r, c, sep ? 4 : 6);
      if (ph == kWarmFinal) {
        r.nvec[c] = k2;
        r.entropy[c] = 0.0;
      }
    }
  }
  // occupations and Rayleigh quotients of this part's rows (used only if the
  // channel finishes refined; the Householder path overwrites them otherwise)
  const int64_t ao = r.ao_off[c];
  for (int i = blockIdx.x + parts * tid; i < n; i += parts * blockDim.x) {
    const double f = i < k1 ? 2.0 : (i < k2 ? 1.0 : 0.0);
    r.eig[ao + i] = lam[i];
    r.occ[ao + i] = f;
    r.occ_eps[ao + i] = f * lam[i];
  }
}

// V <- V (I + E) for the channels that applied this step's correction (the
// product went to Vt), then the masks of the next step; after the last step
// of the SCC iteration, the channels that did not finish go to the
// Householder path.
__global__ void __launch_bounds__(256) k_refine_apply(RefineArgs r, int last) {
  const int c = r.list[blockIdx.y];
  const bool apply = r.m_apply[c] != 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    uint8_t ph = r.phase[c];
    if (ph == kWarmFinal) ph = kWarmDone;
    r.phase[c] = ph;
    r.m_step[c] = ph == kWarmActive ? 1 : 0;
    if (last) {
      r.m_cold[c] = ph == kWarmDone ? 0 : 1;
      r.m_warm[c] = ph == kWarmDone ? 1 : 0;
      if (ph == kWarmActive) stat_add(r, c, 5);
    }
  }
  if (!apply) return;
  const int n = r.nao[c];
  const int64_t mo = r.mat_off[c];
  const int64_t nn = (int64_t)n * n;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  // matrix offsets are sums of n^2 and may be odd: vector copies only when
  // both ends are 16-byte aligned
  if ((mo & 1) == 0) {
    const double2* src = reinterpret_cast<const double2*>(r.Vt + mo);
    double2* dst = reinterpret_cast<double2*>(r.V + mo);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nn / 2; k += stride) dst[k] = src[k];
    if ((nn & 1) && blockIdx.x == 0 && threadIdx.x == 0) r.V[mo + nn - 1] = r.Vt[mo + nn - 1];
  } else {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nn; k += stride)
      r.V[mo + k] = r.Vt[mo + k];
  }
}

// V (columns) from the Householder path's eigenvector rows, for the channels
// it solved; every solved channel can refine from the next iteration on.
__global__ void __launch_bounds__(256) k_vectors_from_rows(RefineArgs r) {
  const int c = r.list[blockIdx.y];
  if (r.m_cold[c] == 0) return;
  const int n = r.nao[c];
  const int tn = (n + 31) / 32;
  const int64_t mo = r.mat_off[c];
  __shared__ double tile[32][33];
  if (blockIdx.x == 0 && threadIdx.x == 0) r.wstate[c] = 1;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int t = blockIdx.x; t < tn * tn; t += gridDim.x) {
    const int ti = t / tn, tj = t - (t / tn) * tn;
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
      const int i = ti * 32 + k, j = tj * 32 + tx;   // row i of Z: eigenvector i
      tile[k][tx] = (i < n && j < n) ? r.Zrows[mo + (int64_t)i * n + j] : 0.0;
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
      const int j = tj * 32 + k, i = ti * 32 + tx;   // V[j][i] = Z[i][j]
      if (i < n && j < n) r.V[mo + (int64_t)j * n + i] = tile[tx][k];
    }
  }
}

void launch_warm_begin(const RefineArgs& r, cudaStream_t stream) {
  if (r.count == 0) return;
  k_warm_begin<<<(r.count + 255) / 256, 256, 0, stream>>>(r);
}

void launch_refine_update(const RefineArgs& r, int max_n, int parts, cudaStream_t stream) {
  if (r.count == 0) return;
  parts = std::max(1, std::min(parts, kRefineMaxParts));
  const size_t bytes = (size_t)max_n * sizeof(double);
  const size_t cap = allow_max_dynamic_smem(k_refine_update);
  (void)cap;
  k_refine_update<<<dim3(parts, r.count), 256, bytes, stream>>>(r, parts);
}

void launch_refine_apply(const RefineArgs& r, int max_n, bool last, cudaStream_t stream) {
  if (r.count == 0) return;
  const int64_t nn = (int64_t)max_n * max_n;
  const int parts = (int)std::max<int64_t>(1, std::min<int64_t>(16, (nn + 4095) / 4096));
  k_refine_apply<<<dim3(parts, r.count), 256, 0, stream>>>(r, last ? 1 : 0);
}

void launch_vectors_from_rows(const RefineArgs& r, int max_n, cudaStream_t stream) {
  if (r.count == 0) return;
  const int tn = (max_n + 31) / 32;
  const int parts = std::max(1, std::min(32, tn * tn));
  k_vectors_from_rows<<<dim3(parts, r.count), 256, 0, stream>>>(r);
}

}  // namespace xtb
