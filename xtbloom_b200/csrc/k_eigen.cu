// Batched FP64 generalized symmetric eigensolver for ragged batches.
//
// HC = SCe is reduced with the symmetric (Loewdin) orthogonaliser X = S^-1/2,
// built once per geometry from the eigenpairs of S, so both basis transforms
// are plain GEMMs: A = X H X, C = X Z.  The standard problem A z = e z is
// solved per system by one CTA: Householder tridiagonalisation (lower,
// LAPACK sytd2 order), eigenvalues by Sturm-count bisection, Fermi-Dirac
// occupations by bisection on the chemical potential, eigenvectors of the
// tridiagonal matrix by inverse iteration with partially pivoted LU and
// modified Gram-Schmidt inside eigenvalue clusters, and the Householder
// back-transform.  Only eigenvectors with non-negligible occupation are
// formed, which is all the density and energy-weighted density need.
//
// The reference solves the same problem with Cholesky + dsyevd
// (model/gfn2/eigensolver.cpp:1221-1268) and Fermi smearing at
// eigensolver.cpp:1026-1219; results agree to rounding because the generalized
// eigenpairs are basis independent.
#include "kernels.cuh"

#include <cfloat>

namespace xtb {

// ---------------------------------------------------------------------------
// Ragged batched GEMM.  C = op(A) * diag(w) * B with op(A) = A or A^T.
// Every matrix of system s is row-major with leading dimension nao[s].
// ---------------------------------------------------------------------------
constexpr int GB = 64, GK = 16;

template <bool TA, bool W>
__global__ void __launch_bounds__(256) k_gemm(GemmArgs g) {
  const int s = g.list[blockIdx.y];
  const int M = g.dm[s], N = g.dn[s], K = g.dk[s];
  const int ld = g.nao[s];
  const int tn = (N + GB - 1) / GB;
  const int tm = (M + GB - 1) / GB;
  if ((int)blockIdx.x >= tm * tn) return;
  const int ti = blockIdx.x / tn, tj = blockIdx.x % tn;
  const double* A = g.A + g.offA[s];
  const double* B = g.B + g.offB[s];
  double* C = g.C + g.offC[s];
  const double* w = W ? g.w + g.offW[s] : nullptr;
  __shared__ double As[GK][GB + 1];
  __shared__ double Bs[GK][GB + 1];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  const int i0 = ti * GB, j0 = tj * GB;
  for (int k0 = 0; k0 < K; k0 += GK) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;   // 0..1023
      if (TA) {
        // A^T tile: element (i, k) = A[k][i]; load row k, cols i (coalesced)
        const int kk = e / GB, ii = e % GB;
        const int gk = k0 + kk, gi = i0 + ii;
        As[kk][ii] = (gk < K && gi < M) ? A[(int64_t)gk * ld + gi] : 0.0;
      } else {
        const int ii = e / GK, kk = e % GK;
        const int gk = k0 + kk, gi = i0 + ii;
        As[kk][ii] = (gk < K && gi < M) ? A[(int64_t)gi * ld + gk] : 0.0;
      }
      const int kk = e / GB, jj = e % GB;
      const int gk = k0 + kk, gj = j0 + jj;
      double bv = (gk < K && gj < N) ? B[(int64_t)gk * ld + gj] : 0.0;
      if (W && gk < K) bv *= w[gk];
      Bs[kk][jj] = bv;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gi = i0 + ty + 16 * i;
    if (gi >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gj = j0 + tx + 16 * j;
      if (gj < N) C[(int64_t)gi * ld + gj] = acc[i][j];
    }
  }
}

void launch_gemm(const GemmArgs& g, bool transA, bool weighted, int max_tiles, int count,
                 cudaStream_t stream) {
  if (count == 0) return;
  dim3 grid(max_tiles, count);
  if (transA && weighted) k_gemm<true, true><<<grid, 256, 0, stream>>>(g);
  else if (transA) k_gemm<true, false><<<grid, 256, 0, stream>>>(g);
  else if (weighted) k_gemm<false, true><<<grid, 256, 0, stream>>>(g);
  else k_gemm<false, false><<<grid, 256, 0, stream>>>(g);
}

// ---------------------------------------------------------------------------
// Householder tridiagonalisation of the full symmetric matrix (in place).
// Reflector i (v[0] = 1 at row i+1, v[k] stored in A[i][i+1+k], k >= 1) and
// tau_i; d, e receive the tridiagonal.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_tridiag(EigArgs g) {
  extern __shared__ double sm[];
  const int s = g.list[blockIdx.x];
  const int n = g.nao[s];
  double* a = g.A + g.mat_off[s];
  double* d = g.d + g.ao_off[s];
  double* e = g.e + g.ao_off[s];
  double* tau = g.tau + g.ao_off[s];
  double* v = sm;
  double* p = sm + n;
  double* red = sm + 2 * n;
  const int tid = threadIdx.x, bs = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = bs >> 5;
  for (int i = 0; i + 2 < n; ++i) {
    const int m = n - i - 1;
    double* row = a + (int64_t)i * n + (i + 1);
    double part = 0.0;
    for (int k = tid; k < m; k += bs) {
      const double x = row[k];
      v[k] = x;
      if (k >= 1) part += x * x;
    }
    const double xn2 = block_sum(part, red);   // includes a sync
    const double alpha = v[0];
    double ti = 0.0, beta = alpha;
    if (xn2 > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
      ti = (beta - alpha) / beta;
      const double sc = 1.0 / (alpha - beta);
      for (int k = tid; k < m; k += bs) {
        if (k >= 1) {
          const double vk = v[k] * sc;
          v[k] = vk;
          row[k] = vk;
        }
      }
    }
    __syncthreads();
    if (tid == 0) {
      v[0] = 1.0;
      d[i] = a[(int64_t)i * n + i];
      e[i] = beta;
      tau[i] = ti;
    }
    __syncthreads();
    if (ti == 0.0) continue;
    // p = tau * A22 v   (A22 = rows/cols i+1..n-1), one warp per row
    double* a22 = a + (int64_t)(i + 1) * n + (i + 1);
    for (int r = warp; r < m; r += nw) {
      const double* ar = a22 + (int64_t)r * n;
      double acc = 0.0;
      for (int c = lane; c < m; c += 32) acc = fma(ar[c], v[c], acc);
      acc = warp_sum(acc);
      if (lane == 0) p[r] = ti * acc;
    }
    __syncthreads();
    double pv = 0.0;
    for (int k = tid; k < m; k += bs) pv += p[k] * v[k];
    const double K = 0.5 * ti * block_sum(pv, red);
    for (int k = tid; k < m; k += bs) p[k] -= K * v[k];
    __syncthreads();
    for (int r = warp; r < m; r += nw) {
      double* ar = a22 + (int64_t)r * n;
      const double vr = v[r], wr = p[r];
      for (int c = lane; c < m; c += 32) ar[c] -= vr * p[c] + wr * v[c];
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (n >= 2) {
      d[n - 2] = a[(int64_t)(n - 2) * n + (n - 2)];
      e[n - 2] = a[(int64_t)(n - 2) * n + (n - 1)];
      tau[n - 2] = 0.0;
    }
    d[n - 1] = a[(int64_t)(n - 1) * n + (n - 1)];
    e[n - 1] = 0.0;
    tau[n - 1] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// Eigenvalues (bisection), occupations and the number of needed eigenvectors.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int sturm_count(const double* d, const double* e2, int n, double x,
                                           double pivmin) {
  int c = 0;
  double q = d[0] - x;
  if (fabs(q) <= pivmin) q = -pivmin;
  if (q < 0.0) ++c;
  for (int k = 1; k < n; ++k) {
    q = d[k] - x - e2[k - 1] / q;
    if (fabs(q) <= pivmin) q = -pivmin;
    if (q < 0.0) ++c;
  }
  return c;
}

__device__ __forceinline__ double fermi_f(double de, double kt) {
  // 1 / (1 + exp(de/kt)) without overflow
  const double x = de / kt;
  if (x > 0.0) {
    const double ex = exp(-x);
    return ex / (1.0 + ex);
  }
  return 1.0 / (1.0 + exp(x));
}

// One warp: occupations of one spin channel (model/gfn2/eigensolver.cpp:1026-1219).
__device__ void warp_fermi(const double* eps, int n, double nel, double kt, double* f,
                           double& entropy) {
  const int lane = threadIdx.x & 31;
  entropy = 0.0;
  if (kt == 0.0) {
    const int full = min((int)floor(nel), n);
    for (int j = lane; j < n; j += 32) f[j] = j < full ? 1.0 : (j == full ? nel - full : 0.0);
    __syncwarp();
    return;
  }
  if (nel <= 0.0) {
    for (int j = lane; j < n; j += 32) f[j] = 0.0;
    __syncwarp();
    return;
  }
  if (nel >= (double)n) {
    for (int j = lane; j < n; j += 32) f[j] = 1.0;
    __syncwarp();
    return;
  }
  const bool holes = nel > 0.5 * n;
  const double ref = holes ? eps[n - 1] : eps[0];
  const double target = holes ? (double)n - nel : nel;
  const double span = eps[n - 1] - eps[0];
  const double margin =
      fmax(64.0, -log(target / n) + 8.0) * kt + 64.0 * DBL_EPSILON * fmax(1.0, fabs(span));
  double lo = (eps[0] - ref) - margin, hi = (eps[n - 1] - ref) + margin;
  const double tol = 64.0 * DBL_EPSILON * target;
  for (int it = 0; it < 400; ++it) {
    const double mid = lo + 0.5 * (hi - lo);
    if (mid == lo || mid == hi) break;
    double q = 0.0;
    for (int j = lane; j < n; j += 32) {
      const double de = (eps[j] - ref) - mid;
      q += holes ? fermi_f(-de, kt) : fermi_f(de, kt);
    }
    q = warp_sum(q);
    if (fabs(q - target) <= tol) {
      lo = hi = mid;
      break;
    }
    if ((!holes && q < target) || (holes && q > target)) lo = mid; else hi = mid;
  }
  const double mu = lo + 0.5 * (hi - lo);
  double sacc = 0.0;
  for (int j = lane; j < n; j += 32) {
    const double fj = fermi_f((eps[j] - ref) - mu, kt);
    f[j] = fj;
    if (fj > 0.0 && fj < 1.0) sacc -= fj * log(fj) + (1.0 - fj) * log(1.0 - fj);
  }
  entropy = warp_sum(sacc);
  __syncwarp();
}

// mode 0: SCC (occupations, needed vectors); mode 1: all vectors, no occupations.
__global__ void __launch_bounds__(256) k_tridiag_eigvals(EigArgs g, int mode, double kt) {
  extern __shared__ double sm[];
  const int s = g.list[blockIdx.x];
  const int n = g.nao[s];
  const int64_t o = g.ao_off[s];
  double* d = sm;
  double* e2 = sm + n;
  double* ev = sm + 2 * n;
  double* fa = sm + 3 * n;
  double* fb = sm + 4 * n;
  double* red = sm + 5 * n;
  const int tid = threadIdx.x, bs = blockDim.x;
  double lo_b = DBL_MAX, hi_b = -DBL_MAX, emax = 0.0;
  for (int k = tid; k < n; k += bs) {
    d[k] = g.d[o + k];
    const double ek = (k < n - 1) ? g.e[o + k] : 0.0;
    const double ekm = (k > 0) ? g.e[o + k - 1] : 0.0;
    e2[k] = ek * ek;
    const double r = fabs(ek) + fabs(ekm);
    lo_b = fmin(lo_b, d[k] - r);
    hi_b = fmax(hi_b, d[k] + r);
    emax = fmax(emax, ek * ek);
  }
  const double gl = -block_max(-lo_b, red);
  const double gu = block_max(hi_b, red);
  const double e2max = block_max(emax, red);
  const double pivmin = DBL_MIN * fmax(1.0, e2max);
  const double tnorm = fmax(fabs(gl), fabs(gu));
  const double glo = gl - 2.0 * tnorm * DBL_EPSILON * n - 4.0 * pivmin;
  const double ghi = gu + 2.0 * tnorm * DBL_EPSILON * n + 4.0 * pivmin;
  for (int j = tid; j < n; j += bs) {
    double lo = glo, hi = ghi;
    for (int it = 0; it < 256; ++it) {
      if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + 4.0 * pivmin) break;
      const double mid = 0.5 * (lo + hi);
      if (mid <= lo || mid >= hi) break;
      if (sturm_count(d, e2, n, mid, pivmin) > j) hi = mid; else lo = mid;
    }
    ev[j] = 0.5 * (lo + hi);
  }
  __syncthreads();
  for (int j = tid; j < n; j += bs) g.eig[o + j] = ev[j];
  if (mode == 1) {
    if (tid == 0) g.nvec[s] = n;
    return;
  }
  const int warp = tid >> 5;
  double ent = 0.0;
  if (warp == 0) warp_fermi(ev, n, g.nel_a[s], kt, fa, ent);
  if (warp == 1) warp_fermi(ev, n, g.nel_b[s], kt, fb, ent);
  if ((tid & 31) == 0 && warp < 2) red[warp] = ent;
  __syncthreads();
  __shared__ int last;
  if (tid == 0) last = -1;
  __syncthreads();
  for (int j = tid; j < n; j += bs) {
    const double f = fa[j] + fb[j];
    g.occ[o + j] = f;
    g.occ_eps[o + j] = f * ev[j];
    if (f > 1e-14) atomicMax(&last, j);
  }
  __syncthreads();
  if (tid == 0) {
    g.nvec[s] = last + 1;
    g.entropy[s] = red[0] + red[1];
  }
}

// ---------------------------------------------------------------------------
// Inverse iteration for eigenvectors 0..nvec-1 of the tridiagonal matrix.
// One thread per eigenvalue cluster; output ZT[j][0..n) (eigenvector-major).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double hash_unit(uint32_t a, uint32_t b) {
  uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u + (a << 6) + (a >> 2));
  h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
  return (double)h * (2.0 / 4294967296.0) - 1.0;
}

__global__ void __launch_bounds__(128) k_inverse_iteration(EigArgs g) {
  const int s = g.list[blockIdx.x];
  const int n = g.nao[s];
  const int m = g.nvec[s];
  const int64_t o = g.ao_off[s];
  const double* d = g.d + o;
  const double* e = g.e + o;
  const double* ev = g.eig + o;
  double* Z = g.Z + g.mat_off[s];
  double* scr = g.scratch + g.scratch_off[s] + (int64_t)threadIdx.x * 5 * n;
  double* u1 = scr;
  double* u2 = scr + n;
  double* u3 = scr + 2 * n;
  double* lm = scr + 3 * n;
  double* pv = scr + 4 * n;
  // one-norm of T and the cluster threshold
  __shared__ double s_onenrm;
  if (threadIdx.x == 0) {
    double nm = 0.0;
    for (int k = 0; k < n; ++k) {
      const double c = fabs(d[k]) + (k > 0 ? fabs(e[k - 1]) : 0.0) + (k < n - 1 ? fabs(e[k]) : 0.0);
      nm = fmax(nm, c);
    }
    s_onenrm = fmax(nm, DBL_MIN);
  }
  __syncthreads();
  const double onenrm = s_onenrm;
  const double ortol = 1e-5 * onenrm;
  const double tiny = DBL_EPSILON * onenrm;
  for (int lead = threadIdx.x; lead < m; lead += blockDim.x) {
    if (lead > 0 && ev[lead] - ev[lead - 1] <= ortol) continue;   // not a cluster leader
    double xprev = -DBL_MAX;
    for (int j = lead; j < m; ++j) {
      if (j > lead && ev[j] - ev[j - 1] > ortol) break;
      double x = ev[j];
      if (j > lead && x - xprev < 10.0 * DBL_EPSILON * fabs(x)) x = xprev + 10.0 * DBL_EPSILON * fabs(x);
      xprev = x;
      // LU with partial pivoting of T - xI
      double diag = d[0] - x, sup = n > 1 ? e[0] : 0.0;
      for (int k = 0; k < n - 1; ++k) {
        const double ck = e[k];
        const double nd = d[k + 1] - x;
        const double ns = (k + 1 < n - 1) ? e[k + 1] : 0.0;
        if (fabs(diag) >= fabs(ck)) {
          const double l = diag != 0.0 ? ck / diag : 0.0;
          u1[k] = diag; u2[k] = sup; u3[k] = 0.0; pv[k] = 0.0; lm[k] = l;
          diag = nd - l * sup;
          sup = ns;
        } else {
          const double l = diag / ck;
          u1[k] = ck; u2[k] = nd; u3[k] = ns; pv[k] = 1.0; lm[k] = l;
          diag = sup - l * nd;
          sup = -l * ns;
        }
      }
      u1[n - 1] = diag;
      for (int k = 0; k < n; ++k)
        if (fabs(u1[k]) < tiny) u1[k] = u1[k] < 0.0 ? -tiny : tiny;
      double* y = Z + (int64_t)j * n;
      for (int k = 0; k < n; ++k) y[k] = hash_unit((uint32_t)k, (uint32_t)(j * 7919 + s));
      const int iters = (j > lead) ? 4 : 3;
      for (int it = 0; it < iters; ++it) {
        // forward elimination
        for (int k = 0; k < n - 1; ++k) {
          if (pv[k] != 0.0) {
            const double tmp = y[k];
            y[k] = y[k + 1];
            y[k + 1] = tmp;
          }
          y[k + 1] -= lm[k] * y[k];
        }
        // back substitution
        y[n - 1] /= u1[n - 1];
        if (n >= 2) y[n - 2] = (y[n - 2] - u2[n - 2] * y[n - 1]) / u1[n - 2];
        for (int k = n - 3; k >= 0; --k) y[k] = (y[k] - u2[k] * y[k + 1] - u3[k] * y[k + 2]) / u1[k];
        // orthogonalise against the earlier members of the cluster
        for (int q = lead; q < j; ++q) {
          const double* zq = Z + (int64_t)q * n;
          double dot = 0.0;
          for (int k = 0; k < n; ++k) dot += y[k] * zq[k];
          for (int k = 0; k < n; ++k) y[k] -= dot * zq[k];
        }
        double nrm = 0.0;
        for (int k = 0; k < n; ++k) nrm += y[k] * y[k];
        const double inv = 1.0 / sqrt(nrm);
        for (int k = 0; k < n; ++k) y[k] *= inv;
      }
      // sign convention: largest component positive
      int kmax = 0;
      double amax = 0.0;
      for (int k = 0; k < n; ++k)
        if (fabs(y[k]) > amax) { amax = fabs(y[k]); kmax = k; }
      if (y[kmax] < 0.0)
        for (int k = 0; k < n; ++k) y[k] = -y[k];
    }
  }
}

// ---------------------------------------------------------------------------
// Back-transform Z <- H_0 H_1 ... H_{n-3} Z (eigenvector-major rows of Z).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_backtransform(EigArgs g) {
  extern __shared__ double sm[];
  const int s = g.list[blockIdx.x];
  const int n = g.nao[s];
  const int m = g.nvec[s];
  const double* a = g.A + g.mat_off[s];
  const double* tau = g.tau + g.ao_off[s];
  double* Z = g.Z + g.mat_off[s];
  double* v = sm;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  for (int i = n - 3; i >= 0; --i) {
    const double ti = tau[i];
    if (ti == 0.0) continue;
    const int L = n - i - 1;
    __syncthreads();
    for (int k = tid; k < L; k += blockDim.x) v[k] = (k == 0) ? 1.0 : a[(int64_t)i * n + i + 1 + k];
    __syncthreads();
    for (int j = warp; j < m; j += nw) {
      double* z = Z + (int64_t)j * n + (i + 1);
      double acc = 0.0;
      for (int k = lane; k < L; k += 32) acc = fma(v[k], z[k], acc);
      acc = ti * warp_sum(acc);
      for (int k = lane; k < L; k += 32) z[k] -= acc * v[k];
    }
  }
}

// Loewdin weights s^-1/2 with the overlap condition guard; failed systems are flagged.
__global__ void k_lowdin_weights(EigArgs g, int32_t* status) {
  const int s = g.list[blockIdx.x];
  const int n = g.nao[s];
  const int64_t o = g.ao_off[s];
  __shared__ double red[33];
  double mn = DBL_MAX, mx = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    mn = fmin(mn, g.eig[o + k]);
    mx = fmax(mx, g.eig[o + k]);
  }
  const double smin = -block_max(-mn, red);
  const double smax = block_max(mx, red);
  const bool ok = smin > 1e-12 * smax && smin > 0.0 && isfinite(smin) && isfinite(smax);
  for (int k = threadIdx.x; k < n; k += blockDim.x) g.occ[o + k] = ok ? 1.0 / sqrt(g.eig[o + k]) : 0.0;
  if (threadIdx.x == 0 && !ok) status[s] = kEigenFailed;
}

void launch_tridiag(const EigArgs& g, int count, int max_n, cudaStream_t stream) {
  if (count == 0) return;
  const size_t sm = (2 * (size_t)max_n + 40) * sizeof(double);
  static const bool attr = cudaFuncSetAttribute(k_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) == cudaSuccess;
  (void)attr;
  k_tridiag<<<count, 512, sm, stream>>>(g);
}

void launch_eigvals(const EigArgs& g, int mode, double kt, int count, int max_n, cudaStream_t stream) {
  if (count == 0) return;
  const size_t sm = (5 * (size_t)max_n + 40) * sizeof(double);
  static const bool attr = cudaFuncSetAttribute(k_tridiag_eigvals, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) == cudaSuccess;
  (void)attr;
  k_tridiag_eigvals<<<count, 256, sm, stream>>>(g, mode, kt);
}

void launch_inverse_iteration(const EigArgs& g, int count, cudaStream_t stream) {
  if (count == 0) return;
  k_inverse_iteration<<<count, 128, 0, stream>>>(g);
}

void launch_backtransform(const EigArgs& g, int count, int max_n, cudaStream_t stream) {
  if (count == 0) return;
  k_backtransform<<<count, 256, ((size_t)max_n + 8) * sizeof(double), stream>>>(g);
}

void launch_lowdin_weights(const EigArgs& g, int32_t* status, int count, cudaStream_t stream) {
  if (count == 0) return;
  k_lowdin_weights<<<count, 256, 0, stream>>>(g, status);
}

}  // namespace xtb
