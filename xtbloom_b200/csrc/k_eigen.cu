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
#include "inverse_iteration.cuh"
#include "kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cfloat>
#include <cstdlib>
#include <cstring>

namespace xtb {

constexpr int GB = 64, GK = 16;

// One FP64 tensor-core product D = A B + D of an 8x8x4 tile (warp-wide):
// lane l holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) .. 2(l%4)+1].
__device__ __forceinline__ void mma_f64(double* d, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// FP64 tile (ti, tj) of edge TB (64, or 32 when few systems are active) of
// system s on the FP64 tensor cores (mma.m8n8k4.f64, FP64 accumulation):
// 256 threads as 2 x 4 warps, each warp a (TB/2) x (TB/4) block of 8x8
// products.  Operand chunks of GK = 16 are staged k-major in shared memory
// (row stride TB + 4: the fragment reads of a half-warp hit distinct banks);
// every element is accumulated over k in the same order (chunks, then steps
// of 4) at either tile width, so both widths give identical results.
template <bool TA, bool W, int TB>
__device__ __forceinline__ void gemm_tile_f64(const GemmArgs& g, int s, int M, int N, int K, int ld,
                                              int ti, int tj, bool mirror, unsigned char* smem) {
  constexpr int LPT = TB * GK / 256;     // elements of each operand chunk per thread
  constexpr int MT = TB / 16, NT = TB / 32;   // 8x8 products per warp and dimension
  constexpr int SP = TB + 4;
  const double* A = g.A + g.offA[s];
  const double* B = g.B + g.offB[s];
  double* C = g.C + g.offC[s];
  const double* w = W ? g.w + g.offW[s] : nullptr;
  // two stages: chunk t is multiplied from one while chunk t+1 is stored
  // into the other, so each chunk needs one barrier
  double (*As)[GK][SP] = reinterpret_cast<double (*)[GK][SP]>(smem);   // [2][GK][SP]
  double (*Bs)[GK][SP] = As + 2;                                       // [2][GK][SP]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;
  const int gq = lane >> 2, tq = lane & 3;
  double acc[MT][NT][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int i0 = ti * TB, j0 = tj * TB;
  // The next chunk's operands are loaded into registers while the current
  // chunk is multiplied, so global latency overlaps the products; they go to
  // the other shared-memory stage after the products.
  double ra[LPT], rb[LPT];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int q = 0; q < LPT; ++q) {
      const int e = tid + q * 256;
      if (TA) {
        // A^T tile: element (i, k) = A[k][i]; load row k, cols i (coalesced)
        const int kk = e / TB, ii = e % TB;
        const int gk = k0 + kk, gi = i0 + ii;
        ra[q] = (gk < K && gi < M) ? A[(int64_t)gk * ld + gi] : 0.0;
      } else {
        const int ii = e / GK, kk = e % GK;
        const int gk = k0 + kk, gi = i0 + ii;
        ra[q] = (gk < K && gi < M) ? A[(int64_t)gi * ld + gk] : 0.0;
      }
      const int kk = e / TB, jj = e % TB;
      const int gk = k0 + kk, gj = j0 + jj;
      double bv = (gk < K && gj < N) ? B[(int64_t)gk * ld + gj] : 0.0;
      if (W && gk < K) bv *= w[gk];
      rb[q] = bv;
    }
  };
  auto stage = [&](int st) {
#pragma unroll
    for (int q = 0; q < LPT; ++q) {
      const int e = tid + q * 256;
      if (TA) As[st][e / TB][e % TB] = ra[q];
      else As[st][e % GK][e / GK] = ra[q];
      Bs[st][e / TB][e % TB] = rb[q];
    }
  };
  fetch(0);
  stage(0);
  __syncthreads();
  int st = 0;
  for (int k0 = 0; k0 < K; k0 += GK) {
    const bool more = k0 + GK < K;
    if (more) fetch(k0 + GK);
#pragma unroll
    for (int ks = 0; ks < GK; ks += 4) {
      double a[MT], b[NT];
#pragma unroll
      for (int i = 0; i < MT; ++i) a[i] = As[st][ks + tq][wm * (TB / 2) + i * 8 + gq];
#pragma unroll
      for (int j = 0; j < NT; ++j) b[j] = Bs[st][ks + tq][wn * (TB / 4) + j * 8 + gq];
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) mma_f64(acc[i][j], a[i], b[j]);
    }
    // every warp finished reading stage st ^ 1 before the previous barrier
    if (more) stage(st ^ 1);
    __syncthreads();
    st ^= 1;
  }
#pragma unroll
  for (int i = 0; i < MT; ++i) {
    const int gi = i0 + wm * (TB / 2) + i * 8 + gq;
    if (gi >= M) continue;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gj = j0 + wn * (TB / 4) + j * 8 + 2 * tq + h;
        if (gj < N) {
          C[(int64_t)gi * ld + gj] = acc[i][j][h];
          if (mirror) C[(int64_t)gj * ld + gi] = acc[i][j][h];
        }
      }
    }
  }
}

// x = hi + lo with hi, lo TF32 (10 explicit mantissa bits each): the pair
// carries about 22 bits of x.
__device__ __forceinline__ void split_tf32(double x, uint32_t& hi, uint32_t& lo) {
  const float f = (float)x;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(f));
  const float r = (float)(x - (double)__uint_as_float(hi));
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

__device__ __forceinline__ void mma_tf32(float* c, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Split-precision tile: A and B are split into TF32 pairs in shared memory and
// multiplied on the tensor cores as a_lo b_hi + a_hi b_lo + a_hi b_hi with FP32
// accumulation (relative error about 1e-6 for the contraction lengths here).
// Eight warps as 2 x 4, each 32 x 16 of the 64 x 64 tile (2 x 2 m16n8k8).
template <bool TA, bool W>
__device__ __forceinline__ void gemm_tile_tf32x3(const GemmArgs& g, int s, int M, int N, int K,
                                                 int ld, int ti, int tj, unsigned char* smem) {
  const double* A = g.A + g.offA[s];
  const double* B = g.B + g.offB[s];
  double* C = g.C + g.offC[s];
  const double* w = W ? g.w + g.offW[s] : nullptr;
  constexpr int AP = GK + 4, BP = GB + 8;   // conflict-free fragment reads
  uint32_t (*Ah)[AP] = reinterpret_cast<uint32_t (*)[AP]>(smem);   // [GB][AP]
  uint32_t (*Al)[AP] = Ah + GB;                                      // [GB][AP]
  uint32_t (*Bh)[BP] = reinterpret_cast<uint32_t (*)[BP]>(Al + GB);  // [GK][BP]
  uint32_t (*Bl)[BP] = Bh + GK;                                      // [GK][BP]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;
  float acc[2][2][4];
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[mi][ni][q] = 0.f;
  const int i0 = ti * GB, j0 = tj * GB;
  for (int k0 = 0; k0 < K; k0 += GK) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;   // 0..1023
      int ii, kk;
      double av;
      if (TA) {
        kk = e / GB;
        ii = e % GB;
        const int gk = k0 + kk, gi = i0 + ii;
        av = (gk < K && gi < M) ? A[(int64_t)gk * ld + gi] : 0.0;
      } else {
        ii = e / GK;
        kk = e % GK;
        const int gk = k0 + kk, gi = i0 + ii;
        av = (gk < K && gi < M) ? A[(int64_t)gi * ld + gk] : 0.0;
      }
      split_tf32(av, Ah[ii][kk], Al[ii][kk]);
      const int kb = e / GB, jj = e % GB;
      const int gk = k0 + kb, gj = j0 + jj;
      double bv = (gk < K && gj < N) ? B[(int64_t)gk * ld + gj] : 0.0;
      if (W && gk < K) bv *= w[gk];
      split_tf32(bv, Bh[kb][jj], Bl[kb][jj]);
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < GK; ks += 8) {
      uint32_t ah[2][4], al[2][4], bh[2][2], bl[2][2];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        const int m0 = wm * 32 + mi * 16 + gq;
        ah[mi][0] = Ah[m0][ks + tq];
        ah[mi][1] = Ah[m0 + 8][ks + tq];
        ah[mi][2] = Ah[m0][ks + tq + 4];
        ah[mi][3] = Ah[m0 + 8][ks + tq + 4];
        al[mi][0] = Al[m0][ks + tq];
        al[mi][1] = Al[m0 + 8][ks + tq];
        al[mi][2] = Al[m0][ks + tq + 4];
        al[mi][3] = Al[m0 + 8][ks + tq + 4];
      }
#pragma unroll
      for (int ni = 0; ni < 2; ++ni) {
        const int n0 = wn * 16 + ni * 8 + gq;
        bh[ni][0] = Bh[ks + tq][n0];
        bh[ni][1] = Bh[ks + tq + 4][n0];
        bl[ni][0] = Bl[ks + tq][n0];
        bl[ni][1] = Bl[ks + tq + 4][n0];
      }
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 2; ++ni) {
          mma_tf32(acc[mi][ni], al[mi], bh[ni]);
          mma_tf32(acc[mi][ni], ah[mi], bl[ni]);
          mma_tf32(acc[mi][ni], ah[mi], bh[ni]);
        }
    }
    __syncthreads();
  }
  const bool mirror = g.sym && ti != tj;
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 2; ++ni)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int gi = i0 + wm * 32 + mi * 16 + gq + (q >= 2 ? 8 : 0);
        const int gj = j0 + wn * 16 + ni * 8 + 2 * tq + (q & 1);
        if (gi < M && gj < N) {
          const double v = (double)acc[mi][ni][q];
          C[(int64_t)gi * ld + gj] = v;
          if (mirror) C[(int64_t)gj * ld + gi] = v;
        }
      }
}

// ---------------------------------------------------------------------------
// Ragged batched GEMM.  C = op(A) * diag(w) * B with op(A) = A or A^T.
// Every matrix of system s is row-major with leading dimension nao[s].  With
// g.sym the product is known to be symmetric (M = N): only the tiles on and
// below the diagonal are computed and each off-diagonal tile is also stored
// transposed.  g.prec selects, per system, the split-precision tile.
// ---------------------------------------------------------------------------
template <bool TA, bool W, int TB>
__global__ void __launch_bounds__(256, 3) k_gemm(GemmArgs g) {
  // one buffer for whichever tile runs: the FP64 tile's two operand stages
  // or the split tile's TF32 parts
  constexpr int kF64Bytes = 2 * 2 * GK * (TB + 4) * 8;
  constexpr int kTf32Bytes = (2 * GB * (GK + 4) + 2 * GK * (GB + 8)) * 4;
  __shared__ __align__(16) unsigned char gsm[kF64Bytes > kTf32Bytes ? kF64Bytes : kTf32Bytes];
  const int s = g.list[blockIdx.y];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int M = g.dm[s], N = g.dn[s], K = g.dk[s];
  const int ld = g.nao[s];
  const int tn = (N + TB - 1) / TB;
  const int tm = (M + TB - 1) / TB;
  int ti, tj;
  bool mirror = false;
  if (g.sym) {
    // tiles on and below the diagonal, mirrored; 32-wide tiles also compute
    // the upper tile of each diagonal 64 x 64 block instead of mirroring it,
    // so that every element is formed exactly as by the 64-wide tiles (the
    // two orders of a symmetric product differ in rounding)
    const int t = blockIdx.x;
    const int lower = tm * (tm + 1) / 2;
    if (t < lower) {
      ti = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);   // ti(ti+1)/2 <= t
      while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
      while (ti * (ti + 1) / 2 > t) --ti;
      tj = t - ti * (ti + 1) / 2;
      mirror = TB == GB ? ti != tj : (ti >> 1) != (tj >> 1);
    } else {
      const int p = t - lower;
      if (TB == GB || 2 * p + 1 >= tm) return;
      ti = 2 * p;
      tj = 2 * p + 1;
    }
  } else {
    if ((int)blockIdx.x >= tm * tn) return;
    ti = blockIdx.x / tn;
    tj = blockIdx.x % tn;
  }
  // the split-precision tile exists for 64-wide tiles; the few-system
  // 32-wide launch multiplies every system in FP64
  if (TB == GB && g.prec != nullptr && g.prec[g.prec_of != nullptr ? g.prec_of[s] : s] == 0) {
    if (g.umma) return;   // formed by k_gemm_umma
    gemm_tile_tf32x3<TA, W>(g, s, M, N, K, ld, ti, tj, gsm);
  } else
    gemm_tile_f64<TA, W, TB>(g, s, M, N, K, ld, ti, tj, mirror, gsm);
}

template <int TB>
void launch_gemm_tb(const GemmArgs& g, bool transA, bool weighted, int tm, int count, cudaStream_t stream) {
  const int tiles = g.sym ? tm * (tm + 1) / 2 + (TB == GB ? 0 : tm / 2) : tm * tm;
  dim3 grid(tiles, count);
  if (transA && weighted) k_gemm<true, true, TB><<<grid, 256, 0, stream>>>(g);
  else if (transA) k_gemm<true, false, TB><<<grid, 256, 0, stream>>>(g);
  else if (weighted) k_gemm<false, true, TB><<<grid, 256, 0, stream>>>(g);
  else k_gemm<false, false, TB><<<grid, 256, 0, stream>>>(g);
}

void launch_gemm(const GemmArgs& g, bool transA, bool weighted, int max_tiles, int count,
                 cudaStream_t stream, int width) {
  if (count == 0) return;
  const int tm = (int)std::lround(std::sqrt((double)max_tiles));   // max_tiles = tm * tm (64-wide)
  // Fewer 64-wide tiles than SMs: 32-wide tiles put four times as many SMs
  // on each product (a 64 x 64 x 240 FP64 tile alone takes ~8 us on one SM).
  const int tiles64 = g.sym ? tm * (tm + 1) / 2 : tm * tm;
  if (width == 32 || (width == 0 && (int64_t)tiles64 * count < sm_count())) {
    launch_gemm_tb<32>(g, transA, weighted, 2 * tm, count, stream);
  } else {
    // split-precision systems on the tcgen05 tiles; XTBLOOM_B200_SPLIT_TILE=mma
    // selects the mma.sync tiles instead (read per launch: a comparison switch)
    const char* tile = std::getenv("XTBLOOM_B200_SPLIT_TILE");
    const bool legacy = tile != nullptr && std::strcmp(tile, "mma") == 0;
    GemmArgs gu = g;
    gu.umma = (g.prec != nullptr && !legacy) ? 1 : 0;
    if (gu.umma) launch_gemm_umma(gu, transA, weighted, tm, count, stream);
    launch_gemm_tb<GB>(gu, transA, weighted, tm, count, stream);
  }
}

// ---------------------------------------------------------------------------
// Householder tridiagonalisation, one CTA per system.  Step i applies
// reflector i's rank-2 update and forms the product of the next reflector
// with the updated block in the same pass over the lower triangle:
//   (A) update the block's first column with (v_i, w_i); it gives x_{i+1};
//   (B) v_{i+1}, tau_{i+1} from x_{i+1};
//   (C) 8 x 32 tiles of the rest, dealt round-robin to the warps: update with
//       (v_i, w_i), then accumulate A v_{i+1} (see fused_tile);
//   (D) w_{i+1} = tau p - (tau/2)(p.v) v, kept as tau p and the scalar
//       (tau/2)(p.v); readers of w apply the correction.
// The global-memory prefix (k_tridiag_prefix, columns above the shared-memory
// block) runs these four phases with a barrier after each; the
// shared-memory kernel (k_tridiag_smem) merges (B) and (D) into its other
// passes and needs two barriers per column.  Both keep the trailing block's
// lower triangle only: packed ((r, c), r >= c, at r(r+1)/2 + c) in shared
// memory, or in place in the square matrix.  Reflectors are stored in the
// global matrix in the layout the back-transform reads (row i, columns i+2..).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int pk32(int r, int c) { return r * (r + 1) / 2 + c; }

// Block-wide sum with a single barrier: every warp posts its partial to
// buf[warp] and every thread adds the posted partials.  Two reductions that
// use the same buf must be separated by another barrier (the kernel below
// alternates two buffers between its two reductions per column).
template <int NW>
__device__ __forceinline__ double block_sum1(double v, double* buf) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) buf[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < NW; ++w) t += buf[w];
  return t;
}

// One tile of kTileRows rows (R0..) and 32 columns (C0..) of the lower
// triangle of the block that starts at row/column o of the packed storage
// (size m), for one warp: update every element with (vi, wi), then lane j
// accumulates the transposed part of A vn for column C0+j directly and keeps
// kTileRows row partials, which a butterfly reduce-scatter (over the low lane
// bits, then exchanges across the remaining lane groups) leaves with lane i
// (and every lane congruent to it) holding row R0+i.  Eight-row tiles keep
// the row values and partials in few enough registers that the rows of a
// tile overlap instead of running one after another.  Elements on the
// diagonal count once.  Results go to the warp's pw.  wi holds w + kw v (the
// previous reflector's correction kw is applied here).  The tile's elements
// are all loaded before any is stored and the row values come from registers
// by shuffles, so the shared-memory loads issue back to back.
// SQ: L is a square row-major matrix with leading dimension ld (the lower
// triangle is used) instead of the packed triangle.
constexpr int kTileRows = 8;
template <bool SQ = false>
__device__ __forceinline__ void fused_tile(double* L, int o, int m, int R0, int C0,
                                           const double* vi, const double* wi, double kw,
                                           const double* vn, double* pw, int lane, bool want_mv,
                                           int ld = 0) {
  const int cj = C0 + lane;
  const bool cok = cj < m;
  const double vn_c = cok ? vn[cj] : 0.0;
  const double vi_c = cok ? vi[cj] : 0.0;
  const double wi_c = cok ? fma(-kw, vi_c, wi[cj]) : 0.0;
  const int rl = R0 + (lane & (kTileRows - 1));
  const double vi_r = rl < m ? vi[rl] : 0.0;
  const double wi_r = rl < m ? fma(-kw, vi_r, wi[rl]) : 0.0;
  const double vn_r = rl < m ? vn[rl] : 0.0;
  const int rows = min(kTileRows, m - R0);
  const int dcol = cj - R0;            // element (R0+i, cj) is on/below the diagonal iff dcol <= i
  double a[kTileRows];
  const int base0 = SQ ? (o + R0) * ld + o + cj : pk32(o + R0, o) + cj;
  {
    int base = base0;
#pragma unroll
    for (int i = 0; i < kTileRows; ++i) {
      const bool ok = i < rows && cok && dcol <= i;
      a[i] = ok ? L[base] : 0.0;
      base += SQ ? ld : o + R0 + i + 1;
    }
  }
  double col = 0.0;
#pragma unroll
  for (int i = 0; i < kTileRows; ++i) {
    const double vr = __shfl_sync(0xffffffffu, vi_r, i);
    const double wr = __shfl_sync(0xffffffffu, wi_r, i);
    const double nr = __shfl_sync(0xffffffffu, vn_r, i);
    const double u = a[i] - (vr * wi_c + wr * vi_c);
    a[i] = dcol > i ? 0.0 : u;   // rows past m and columns past m give 0
    if (dcol < i) col = fma(a[i], nr, col);
  }
  {
    int base = base0;
#pragma unroll
    for (int i = 0; i < kTileRows; ++i) {
      const bool ok = i < rows && cok && dcol <= i;
      if (ok) L[base] = a[i];
      base += SQ ? ld : o + R0 + i + 1;
    }
  }
  if (!want_mv) return;
#pragma unroll
  for (int i = 0; i < kTileRows; ++i) a[i] *= vn_c;
#pragma unroll
  for (int sh = kTileRows / 2; sh >= 1; sh >>= 1) {
    const bool up = (lane & sh) != 0;
#pragma unroll
    for (int k = 0; k < sh; ++k) {
      const double send = up ? a[k] : a[k + sh];
      const double keep = up ? a[k + sh] : a[k];
      a[k] = keep + __shfl_xor_sync(0xffffffffu, send, sh);
    }
  }
#pragma unroll
  for (int x = kTileRows; x < 32; x <<= 1) a[0] += __shfl_xor_sync(0xffffffffu, a[0], x);
  if (lane < kTileRows && rl < m) pw[rl] += a[0];
  if (cok) pw[cj] += col;
}

// Tiles of the lower triangle of an m x m block: row blocks of kTileRows,
// column blocks of 32; with G = 32 / kTileRows, row blocks G p .. G p + G - 1
// hold p + 1 tiles each, so the tiles of the row blocks below G p number
// G p (p + 1) / 2.
constexpr int kTileGroup = 32 / kTileRows;
__device__ __forceinline__ int tri_tiles(int m) {
  const int nr = (m + kTileRows - 1) / kTileRows;
  const int p = nr / kTileGroup;
  return kTileGroup * p * (p + 1) / 2 + (nr % kTileGroup) * (p + 1);
}
__device__ __forceinline__ void tri_tile(int tl, int& R, int& C) {
  int p = (int)((sqrtf(8.0f * tl / kTileGroup + 1.0f) - 1.0f) * 0.5f);
  while (kTileGroup * (p + 1) * (p + 2) / 2 <= tl) ++p;
  while (kTileGroup * p * (p + 1) / 2 > tl) --p;
  const int rem = tl - kTileGroup * p * (p + 1) / 2;
  R = kTileGroup * p + rem / (p + 1);
  C = rem % (p + 1);
}


// tri_tile as a table for blocks of up to 256 rows (tri_tiles(256) = 144
// tiles): the shared-memory kernel looks a tile up with one warp-uniform
// constant load instead of a square root and an integer division per tile.
constexpr int kTileTableRows = 256;
constexpr int kTileTableSize = 144;
struct TileTable {
  unsigned short rc[kTileTableSize];   // row block | column block << 8
};
constexpr TileTable make_tile_table() {
  TileTable t{};
  int tl = 0;
  for (int R = 0; tl < kTileTableSize; ++R)
    for (int C = 0; C <= R / kTileGroup && tl < kTileTableSize; ++C)
      t.rc[tl++] = (unsigned short)(R | (C << 8));
  return t;
}
__constant__ TileTable c_tile_table = make_tile_table();

// Shared-memory kernel: the trailing nl x nl block (rows/columns i0..n-1,
// i0 = max(0, n - nloc)) in packed lower storage in one CTA's shared memory,
// two barriers per column.  The reflector of a column is kept unscaled (the
// column's own values) and scaled by 1/(alpha - beta) where its own column's
// tiles read it, so no pass has to wait for a scaled copy; the next column's
// first pass, which forms v_r for its row anyway, stores that scaled value in
// place for the next column's tiles.  The warps' partial products
// A v and their dot products with v are posted by the tile pass and summed by
// the next column's first pass, where w = tau p - (tau/2)(tau p.v) v is formed.
// Per column:
//   (A) row r (one thread): p_r = sum of the warps' partials (row 0's partials
//       sit in a separate double-buffered array, because every thread reads
//       them), w_r, the update of the block's first column with (v_i, w_i),
//       the column's norm -> one barrier;
//   (C) every working thread (one with a row in (A), or in a warp with
//       tiles) forms alpha, beta, tau and the scale redundantly; the 8 x 32
//       tiles of the rest (indices from c_tile_table, dealt round-robin to
//       the warps) are updated with (v_i, w_i) and multiplied by v_{i+1};
//       the warps' partials of p and p.v are posted -> one barrier.
// KIND (what the caller guarantees; the masks that then select nothing are
// compiled out, the operations on the elements are the same):
//   kTileFull  every row inside the block and the tile strictly below the
//              diagonal (R0 + kTileRows <= m, C0 + 32 <= R0): no masks;
//   kTileRowsIn every row inside the block: only the diagonal mask (an
//              element on or below the diagonal has its column inside too);
//   kTileEdge  the last row block: every mask.
constexpr int kTileEdge = 0, kTileRowsIn = 1, kTileFull = 2;
template <int KIND>
__device__ __forceinline__ void fused_tile2(double* L, int o, int m, int R0, int C0,
                                            const double* vi, const double* wi,
                                            const double* vn, double scn, double* pw, double* pw0,
                                            int lane, bool want_mv, double& dot) {
  const int cj = C0 + lane;
  constexpr bool FULL = KIND == kTileFull, RIN = KIND != kTileEdge;
  const bool cok = FULL || cj < m;
  const double vn_c = cok ? (cj == 0 ? 1.0 : vn[cj] * scn) : 0.0;
  const double vi_c = cok ? vi[cj] : 0.0;
  const double wi_c = cok ? wi[cj] : 0.0;
  const int rl = R0 + (lane & (kTileRows - 1));
  const bool rok = RIN || rl < m;
  const double vn_r = rok ? ((!FULL && rl == 0) ? 1.0 : vn[rl] * scn) : 0.0;
  const int rows = RIN ? kTileRows : min(kTileRows, m - R0);
  const int dcol = cj - R0;
  double a[kTileRows];
  const int base0 = pk32(o + R0, o) + cj;
  {
    int base = base0;
#pragma unroll
    for (int i = 0; i < kTileRows; ++i) {
      const bool ok = FULL || (RIN ? dcol <= i : (i < rows && cok && dcol <= i));
      a[i] = ok ? L[base] : 0.0;
      base += o + R0 + i + 1;
    }
  }
  double col = 0.0;
  // The row values are warp-uniform: one broadcast shared-memory load each
  // (a shuffle of a double is two shuffles, and the shuffles, not the
  // arithmetic, bound this loop on large blocks).  Rows past m read in-bounds
  // scratch that the select discards.
#pragma unroll
  for (int i = 0; i < kTileRows; ++i) {
    const bool ri = RIN || i < rows;
    const double vr = ri ? vi[R0 + i] : 0.0;
    const double wr = ri ? wi[R0 + i] : 0.0;
    const double nr = ri ? ((!FULL && R0 + i == 0) ? 1.0 : vn[R0 + i] * scn) : 0.0;
    // contraction written out, so that the rounding does not depend on the
    // compiler's choice of which product to fuse
    const double u = a[i] - fma(vr, wi_c, wr * vi_c);
    a[i] = (!FULL && dcol > i) ? 0.0 : u;
    if (FULL || dcol < i) col = fma(a[i], nr, col);
  }
  {
    int base = base0;
#pragma unroll
    for (int i = 0; i < kTileRows; ++i) {
      const bool ok = FULL || (RIN ? dcol <= i : (i < rows && cok && dcol <= i));
      if (ok) L[base] = a[i];
      base += o + R0 + i + 1;
    }
  }
  if (!want_mv) return;
#pragma unroll
  for (int i = 0; i < kTileRows; ++i) a[i] *= vn_c;
#pragma unroll
  for (int sh = kTileRows / 2; sh >= 1; sh >>= 1) {
    const bool up = (lane & sh) != 0;
#pragma unroll
    for (int k = 0; k < sh; ++k) {
      const double send = up ? a[k] : a[k + sh];
      const double keep = up ? a[k + sh] : a[k];
      a[k] = keep + __shfl_xor_sync(0xffffffffu, send, sh);
    }
  }
#pragma unroll
  for (int x = kTileRows; x < 32; x <<= 1) a[0] += __shfl_xor_sync(0xffffffffu, a[0], x);
  if (lane < kTileRows && rok) {
    double* dst = (!FULL && rl == 0) ? pw0 : pw + rl;
    *dst += a[0];
    dot = fma(a[0], vn_r, dot);
  }
  if (cok) {
    double* dst = cj == 0 ? pw0 : pw + cj;
    *dst += col;
    dot = fma(col, vn_c, dot);
  }
}

template <int NT>
__global__ void __launch_bounds__(NT, 512 / NT) k_tridiag_smem(EigArgs g, const int32_t* list, int nloc) {
  extern __shared__ double sm[];
  constexpr int nw = NT / 32;
  static_assert(NT >= 256, "(A) gives each thread at most one row: blocks have at most 228 rows");
  const int s = list[blockIdx.x];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int n = g.nao[s];
  const int i0 = n > nloc ? n - nloc : 0;
  const int nl = n - i0;
  double* ga = g.A + g.mat_off[s];
  double* d = g.d + g.ao_off[s] + i0;
  double* e = g.e + g.ao_off[s] + i0;
  double* tau = g.tau + g.ao_off[s] + i0;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  double* L = sm;
  double* vb0 = L + pk32(nl, 0);
  double* vb1 = vb0 + nl;
  double* wb = vb1 + nl;
  double* priv = wb + nl;             // nw x nl: the warps' partials of p (rows >= 1)
  double* red = priv + nw * nl;       // 32: norm partials
  double* dots = red + 32;            // 32: the warps' partials of p.v
  double* row0 = dots + 32;           // 2 x 32: the warps' partials of p_0
  for (int r = warp; r < nl; r += nw)
    for (int c = lane; c <= r; c += 32) L[pk32(r, c)] = ga[(int64_t)(i0 + r) * n + i0 + c];
  for (int k = tid; k < nw * nl; k += NT) priv[k] = 0.0;
  for (int k = tid; k < nl; k += NT) vb0[k] = vb1[k] = wb[k] = 0.0;
  if (tid < 32) { dots[tid] = 0.0; row0[tid] = 0.0; row0[32 + tid] = 0.0; }
  __syncthreads();
  if (nl == 1) {
    if (tid == 0) { d[0] = L[0]; e[0] = 0.0; tau[0] = 0.0; }
    return;
  }
  int cur = 0;
  double sc_prev = 0.0, tau_prev = 0.0;
  for (int i = -1; i + 2 < nl; ++i) {
    const int o = i + 1, m = nl - o;
    double* vi = cur ? vb1 : vb0;
    double* vn = cur ? vb0 : vb1;
    double* r0c = row0 + 32 * cur;
    double* r0n = row0 + 32 * (cur ^ 1);
    const bool next = o + 3 <= nl;
    const int m1 = m - 1;
    const int ntiles = tri_tiles(m1);
    // A thread without a row in (A) skips the sums that only (A) uses, and a
    // warp without a tile that stores no reflector element skips the
    // reflector: blocks only shrink, so such a thread stays idle to the end
    // and its values are never read.
    const bool has_row = tid < m;
    const bool forms = has_row || warp < ntiles;
    // (A) w_i from the posted partials, then the block's first column
    double pv = 0.0, p0 = 0.0;
    if (has_row) {
#pragma unroll
      for (int w = 0; w < nw; ++w) {
        pv += dots[w];
        p0 += r0c[w];
      }
    }
    const double kw = 0.5 * tau_prev * tau_prev * pv;
    // contractions in this kernel are written out (fma), so that the rounding
    // does not depend on the compiler's choice
    const double w0 = fma(tau_prev, p0, -kw);      // v_i[0] = 1
    double part = 0.0;
    for (int r = tid; r < m; r += NT) {
      double wr = w0;
      double vr = 1.0;
      if (r > 0) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < nw; ++w) {
          t += priv[w * nl + r];
          priv[w * nl + r] = 0.0;
        }
        vr = vi[r] * sc_prev;
        vi[r] = vr;        // the tiles below read the scaled reflector
        wr = fma(-kw, vr, tau_prev * t);
      }
      wb[r] = wr;
      const int idx = pk32(o + r, o);
      const double c = L[idx] - fma(vr, w0, wr);
      L[idx] = c;
      if (r == 0) d[o] = c;
      if (r >= 1) vn[r - 1] = c;
      if (r >= 2) part = fma(c, c, part);
    }
    // the column's norm (block_sum1, with the final sum only where it is used)
    double xn2 = 0.0;
    {
      const double ws = warp * 32 < m ? warp_sum(part) : 0.0;
      if (lane == 0) red[warp] = ws;
      __syncthreads();
      if (forms) {
#pragma unroll
        for (int w = 0; w < nw; ++w) xn2 += red[w];
      }
    }
    // reflector o+1 from the updated column (every working thread, same operands)
    double ti = 0.0, sc = 0.0;
    if (next && forms) {
      const double alpha = vn[0];
      double beta = alpha;
      if (xn2 > 0.0) {
        beta = -copysign(sqrt(fma(alpha, alpha, xn2)), alpha);
        ti = (beta - alpha) / beta;
        sc = 1.0 / (alpha - beta);
        for (int k = tid + 1; k < m - 1; k += NT)
          ga[(int64_t)(i0 + o) * n + i0 + o + 1 + k] = vn[k] * sc;
      }
      if (tid == 0) {
        e[o] = beta;
        tau[o] = ti;
      }
    }
    if (tid < nw) r0c[tid] = 0.0;     // read above, before the barrier; next used two columns on
    // (C) rank-2 update of the rest of the block, fused with A v_{o+1}
    if (warp < ntiles) {
      double* pw = priv + warp * nl;
      const bool mv = next && ti != 0.0;
      double dot = 0.0;
      for (int tl = warp; tl < ntiles; tl += nw) {
        const unsigned rc = c_tile_table.rc[tl];
        const int R = rc & 0xff, C = rc >> 8;
        // most tiles of a large block lie strictly below the diagonal with
        // every row inside it, and only the last row block needs row masks
        if ((R + 1) * kTileRows > m1)
          fused_tile2<kTileEdge>(L, o + 1, m1, R * kTileRows, C << 5, vi + 1, wb + 1, vn, sc, pw,
                                 r0n + warp, lane, mv, dot);
        else if ((C << 5) + 32 <= R * kTileRows)
          fused_tile2<kTileFull>(L, o + 1, m1, R * kTileRows, C << 5, vi + 1, wb + 1, vn, sc, pw,
                                 r0n + warp, lane, mv, dot);
        else
          fused_tile2<kTileRowsIn>(L, o + 1, m1, R * kTileRows, C << 5, vi + 1, wb + 1, vn, sc, pw,
                                   r0n + warp, lane, mv, dot);
      }
      dot = warp_sum(dot);
      if (lane == 0) dots[warp] = mv ? dot : 0.0;
    } else if (lane == 0) {
      dots[warp] = 0.0;
    }
    __syncthreads();
    if (!next) break;
    tau_prev = ti;
    sc_prev = sc;
    cur ^= 1;
  }
  if (tid == 0) {
    e[nl - 2] = L[pk32(nl - 1, nl - 2)];
    tau[nl - 2] = 0.0;
    d[nl - 1] = L[pk32(nl - 1, nl - 1)];
    e[nl - 1] = 0.0;
    tau[nl - 1] = 0.0;
  }
}

size_t tridiag_smem_bytes(int nl, int nt) {
  return ((size_t)nl * (nl + 1) / 2 + (3 + nt / 32) * (size_t)nl + 32 + 32 + 64 + 8) * sizeof(double);
}

// Global-memory prefix of the same reduction for systems larger than the
// shared-memory block: the first K = n - nloc reflectors are formed in place
// on the lower triangle of the square matrix (L2 / HBM resident), with the
// four phases per column described above, so each column
// reads and writes the trailing triangle once, in coalesced 8 x 32 tiles.
// The last step (column K) applies reflector K-1 to the trailing block and
// forms no reflector: the block from row/column K is then A^(K), which the
// shared-memory kernel loads and finishes.  Only the vectors and the warps'
// partial products live in shared memory ((4 + NT/32) n doubles).
template <int NT>
__global__ void __launch_bounds__(NT) k_tridiag_prefix(EigArgs g, int nloc) {
  extern __shared__ double sm[];
  constexpr int nw = NT / 32;
  const int s = g.list[blockIdx.x];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int n = g.nao[s];
  const int K = n - nloc;
  if (K <= 0) return;
  double* A = g.A + g.mat_off[s];
  double* d = g.d + g.ao_off[s];
  double* e = g.e + g.ao_off[s];
  double* tau = g.tau + g.ao_off[s];
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  double* vb0 = sm;
  double* vb1 = vb0 + n;
  double* wb0 = vb1 + n;
  double* wb1 = wb0 + n;
  double* priv = wb1 + n;             // nw x n
  double* red = priv + nw * n;        // 2 x 32
  __shared__ double s_alpha;
  for (int k = tid; k < nw * n; k += NT) priv[k] = 0.0;
  for (int k = tid; k < n; k += NT) vb0[k] = wb0[k] = vb1[k] = wb1[k] = 0.0;
  __syncthreads();
  int cur = 0;
  double kw = 0.0;
  for (int i = -1; i < K; ++i) {
    const int o = i + 1, m = n - o;
    const double* vi = cur ? vb1 : vb0;
    const double* wi = cur ? wb1 : wb0;
    double* vn = cur ? vb0 : vb1;
    double* wn = cur ? wb0 : wb1;
    const bool next = o < K && o + 3 <= n;
    // (A) first column of the block, updated with (v_i, w_i)
    double part = 0.0;
    const double vi0 = vi[0], wi0 = fma(-kw, vi0, wi[0]);
    for (int r = tid; r < m; r += NT) {
      const int idx = (o + r) * n + o;
      const double vr = vi[r];
      const double c = A[idx] - (vr * wi0 + fma(-kw, vr, wi[r]) * vi0);
      A[idx] = c;
      if (r == 0) d[o] = c;
      if (r >= 1) vn[r - 1] = c;
      if (r == 1) s_alpha = c;
      if (r >= 2) part += c * c;
    }
    const double xn2 = block_sum1<nw>(part, red);
    // (B) reflector o (row o of the matrix keeps it, columns o+2..)
    double ti = 0.0;
    if (next) {
      const double alpha = s_alpha;
      double beta = alpha;
      if (xn2 > 0.0) {
        beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
        ti = (beta - alpha) / beta;
        const double sc = 1.0 / (alpha - beta);
        for (int k = tid + 1; k < m - 1; k += NT) {
          const double vk = vn[k] * sc;
          vn[k] = vk;
          A[o * n + o + 1 + k] = vk;
        }
      } else {
        for (int k = tid + 1; k < m - 1; k += NT) vn[k] = 0.0;
      }
      if (tid == 0) {
        vn[0] = 1.0;
        e[o] = beta;
        tau[o] = ti;
      }
    } else {
      for (int k = tid; k < m; k += NT) vn[k] = 0.0;
    }
    __syncthreads();
    // (C) rank-2 update of the rest of the block, fused with A v_next
    const int m1 = m - 1;
    {
      const int ntiles = tri_tiles(m1);
      double* pw = priv + warp * n;
      const bool mv = next && ti != 0.0;
      for (int tl = warp; tl < ntiles; tl += nw) {
        int R, C;
        tri_tile(tl, R, C);
        fused_tile<true>(A, o + 1, m1, R * kTileRows, C << 5, vi + 1, wi + 1, kw, vn, pw, lane, mv, n);
      }
    }
    __syncthreads();
    if (!next) break;
    // (D) w_next = tau p and its correction kw = (tau/2)(tau p . v)
    double pv = 0.0;
    for (int k = tid; k < m1; k += NT) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < nw; ++w) {
        t += priv[w * n + k];
        priv[w * n + k] = 0.0;
      }
      t *= ti;
      wn[k] = t;
      pv += t * vn[k];
    }
    kw = 0.5 * ti * block_sum1<nw>(pv, red + 32);
    cur ^= 1;
  }
}

size_t tridiag_prefix_bytes(int n, int nt) { return ((4 + (size_t)nt / 32) * n + 64) * sizeof(double); }


// Largest trailing block the shared-memory kernel holds (227 KB per CTA).
constexpr int kTridiagSmemMax = 228;
static_assert(kTridiagSmemMax <= kTileTableRows, "the shared-memory kernel's tiles come from c_tile_table");

void launch_tridiag_smem(const EigArgs& g, const int32_t* list, int count, int max_n, cudaStream_t stream) {
  if (count == 0) return;
  const size_t cap256 = allow_max_dynamic_smem(k_tridiag_smem<256>);
  const size_t cap512 = allow_max_dynamic_smem(k_tridiag_smem<512>);
  static const int per_sm = [] {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess) v = 0;
    return v;
  }();
  int nloc = std::min(max_n, kTridiagSmemMax);
  while (nloc > 2 && tridiag_smem_bytes(nloc, 256) > cap256) --nloc;
  // 512 threads shorten one system's critical path.  They are used when the
  // SM would hold a single 256-thread CTA anyway (its packed triangle) or
  // when there are fewer systems than SMs; otherwise two 256-thread CTAs per
  // SM overlap each other's barrier waits.  The 512-thread block is a few
  // columns smaller (its per-warp partials); the prefix takes those columns.
  const bool one_per_sm = per_sm > 0 && 2 * (tridiag_smem_bytes(nloc, 256) + 1024) > (size_t)per_sm;
  const bool wide = count < sm_count() || one_per_sm;
  if (wide)
    while (nloc > 2 && tridiag_smem_bytes(nloc, 512) > cap512) --nloc;
  if (max_n > nloc) {
    // columns that do not fit: reduced in global memory first
    const size_t capp = allow_max_dynamic_smem(k_tridiag_prefix<512>);
    const size_t bp = tridiag_prefix_bytes(max_n, 512);
    if (bp <= capp) {
      k_tridiag_prefix<512><<<count, 512, bp, stream>>>(g, nloc);
    } else {
      const size_t cap2 = allow_max_dynamic_smem(k_tridiag_prefix<256>);
      (void)cap2;
      k_tridiag_prefix<256><<<count, 256, tridiag_prefix_bytes(max_n, 256), stream>>>(g, nloc);
    }
  }
  if (wide) {
    k_tridiag_smem<512><<<count, 512, tridiag_smem_bytes(nloc, 512), stream>>>(g, list, nloc);
  } else {
    k_tridiag_smem<256><<<count, 256, tridiag_smem_bytes(nloc, 256), stream>>>(g, list, nloc);
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

// Number of eigenvalues below x for four shifts at once, from the sign changes
// of the three-term (Givens) Sturm sequence p_{k+1} = (d_k - x) p_k - e_{k-1}^2 p_{k-1},
// p_0 = 1.  No divisions.  The caller scales T by a power of two so that its
// spectrum lies in [-1, 1] and floors e^2 at 1e-40: then |p| grows at most
// 3x and shrinks at most 3e40x per step, and rescaling the pair (p_{k-1}, p_k)
// by a power of two every fourth step (exact, sign-preserving) keeps it far
// from overflow and underflow.  Sign changes are read from the sign bits.  An
// exact zero inside the sequence lies between two terms of opposite sign
// (p_{k+1} = -e_k^2 p_{k-1}, and e^2 > 0), so the sign it is given does not
// change the count; a zero last term means x is an eigenvalue, which either
// count brackets correctly.
__device__ __forceinline__ void rescale_pair(double& a, double& b) {
  const int ea = __double2hiint(a) & 0x7ff00000;
  const int eb = __double2hiint(b) & 0x7ff00000;
  // 2^-(exponent of max(|a|, |b|)); 2^1023 when both are zero or subnormal
  const double f = __hiloint2double(0x7fe00000 - max(ea, eb), 0);
  a *= f;
  b *= f;
}

__device__ __forceinline__ void sturm4(const double* d, const double* e2, int n, const double x[4],
                                       int c[4]) {
  double p0[4], p1[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    p0[q] = 1.0;
    p1[q] = d[0] - x[q];
    c[q] = (int)((unsigned)__double2hiint(p1[q]) >> 31);
  }
  auto step = [&](int k) {
    const double dk = d[k], ek = e2[k - 1];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double p2 = fma(dk - x[q], p1[q], -ek * p0[q]);
      c[q] += (int)((unsigned)(__double2hiint(p2) ^ __double2hiint(p1[q])) >> 31);
      p0[q] = p1[q];
      p1[q] = p2;
    }
  };
  int k = 1;
  for (; k + 4 <= n; k += 4) {
    step(k);
    step(k + 1);
    step(k + 2);
    step(k + 3);
#pragma unroll
    for (int q = 0; q < 4; ++q) rescale_pair(p0[q], p1[q]);
  }
  for (; k < n; ++k) step(k);
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
  // The root of q(mu) = target to the reference's tolerance |q - target| <=
  // 64 eps target (it bisects; any mu inside that band gives the same
  // occupations to rounding).  Newton steps on q' = sum f (1 - f) / kT inside
  // the bisection bracket: a few iterations where bisection needs ~55, which
  // matters when few systems are left and this loop is on the critical path.
  const double ikt = 1.0 / kt;
  double mu = lo + 0.5 * (hi - lo);
  for (int it = 0; it < 400; ++it) {
    double q = 0.0, dq = 0.0;
    for (int j = lane; j < n; j += 32) {
      double x = ((eps[j] - ref) - mu) * ikt;
      if (holes) x = -x;
      const double ex = exp(-fabs(x));
      const double r = 1.0 / (1.0 + ex);
      const double fj = x > 0.0 ? ex * r : r;
      q += fj;
      dq = fma(fj, 1.0 - fj, dq);
    }
    q = warp_sum(q);
    dq = warp_sum(dq) * (holes ? -ikt : ikt);
    if (fabs(q - target) <= tol) break;
    if ((!holes && q < target) || (holes && q > target)) lo = mu; else hi = mu;
    const double mid = lo + 0.5 * (hi - lo);
    if (mid == lo || mid == hi) break;   // bracket at the resolution limit
    double nm = dq != 0.0 ? mu - (q - target) / dq : mid;
    if (!(nm > lo && nm < hi)) nm = mid;
    mu = nm;
  }
  double sacc = 0.0;
  for (int j = lane; j < n; j += 32) {
    const double fj = fermi_f((eps[j] - ref) - mu, kt);
    f[j] = fj;
    if (fj > 0.0 && fj < 1.0) sacc -= fj * log(fj) + (1.0 - fj) * log(1.0 - fj);
  }
  entropy = warp_sum(sacc);
  __syncwarp();
}

__device__ void bisect_range(const double* d, const double* e2, int n, double glo, double ghi,
                             double pivmin, int j0, int j1, double unscale, int tpe_max,
                             int tpe_block, double* ev);

// Number of eigenvalues the SCC needs: the occupied levels and eight above
// them (mode 0); all of them for the overlap (mode 1) and for an SCC
// iteration that also seeds the warm-started refinement (mode 2).
__device__ __forceinline__ int levels_needed(const EigArgs& g, int s, int n, int mode) {
  if (mode != 0) return n;
  return min(n, (int)ceil(fmax(g.nel_a[s], g.nel_b[s])) + 8);
}

struct ScaledTridiag {
  double glo, ghi;     // bracket of the whole spectrum (scaled)
  double pivmin;       // (scaled)
  double unscale;      // 2^ex: eigenvalue of T = scaled eigenvalue * unscale
};

// Loads the tridiagonal of system s into shared memory as T / 2^ex with the
// spectrum inside [-1, 1] (exact; see sturm4): d, e2 = squared off-diagonal
// floored at 1e-40.  Gershgorin bounds give the bracket.  Block-wide.
__device__ ScaledTridiag load_scaled_tridiag(const EigArgs& g, int64_t o, int n, double* d, double* e2,
                                             double* red) {
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
  int ex = 0;
  frexp(tnorm, &ex);
  const double sc = ldexp(1.0, -ex);
  for (int k = tid; k < n; k += bs) {
    d[k] *= sc;
    e2[k] = fmax(e2[k] * sc * sc, 1e-40);
  }
  __syncthreads();
  ScaledTridiag t;
  t.glo = (gl - 2.0 * tnorm * DBL_EPSILON * n - 4.0 * pivmin) * sc;
  t.ghi = (gu + 2.0 * tnorm * DBL_EPSILON * n + 4.0 * pivmin) * sc;
  t.pivmin = pivmin * sc * sc;
  t.unscale = ldexp(1.0, ex);
  return t;
}

// Latency form for few systems: part blockIdx.x of `parts` CTAs of system
// blockIdx.y bisects a contiguous slice of the needed eigenvalues, with up to
// a warp per eigenvalue, and writes them to g.eig.
__global__ void __launch_bounds__(256) k_eigvals_part(EigArgs g, int mode, int parts) {
  extern __shared__ double sm[];
  const int s = g.list[blockIdx.y];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int n = g.nao[s];
  const int64_t o = g.ao_off[s];
  const int nk = levels_needed(g, s, n, mode);
  const int per = (nk + parts - 1) / parts;
  const int j0 = blockIdx.x * per, j1 = min(nk, j0 + per);
  if (j0 >= j1) return;   // uniform over the block
  double* d = sm;
  double* e2 = sm + n;
  double* red = sm + 2 * n;
  const ScaledTridiag t = load_scaled_tridiag(g, o, n, d, e2, red);
  bisect_range(d, e2, n, t.glo, t.ghi, t.pivmin, j0, j1, t.unscale, 32, (int)blockDim.x, g.eig + o);
}

// The block size k_tridiag_eigvals chooses its threads per eigenvalue for
// (bisect_range's tpe_block), whatever block it is launched with.
constexpr int kEigvalsTpeBlock = 256;

// mode 0: SCC (occupations, needed vectors); mode 1: all vectors, no
// occupations; mode 2: SCC occupations from the whole spectrum.
// have != 0: the needed eigenvalues are already in g.eig (k_eigvals_part).
// Bisection here uses at most tpe_max threads per eigenvalue.
__global__ void __launch_bounds__(256) k_tridiag_eigvals(EigArgs g, int mode, double kt, int have,
                                                         int tpe_max) {
  extern __shared__ double sm[];
  const int s = g.list[blockIdx.x];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int n = g.nao[s];
  const int64_t o = g.ao_off[s];
  double* d = sm;
  double* e2 = sm + n;
  double* ev = sm + 2 * n;
  double* fa = sm + 3 * n;
  double* fb = sm + 4 * n;
  double* red = sm + 5 * n;
  const int tid = threadIdx.x, bs = blockDim.x;
  const ScaledTridiag t = load_scaled_tridiag(g, o, n, d, e2, red);
  // In the SCC only the occupied eigenpairs and a few above them are needed:
  // the Fermi level is found on that partial spectrum (the higher levels count
  // as empty) and the rest is computed only if the last one is not empty.
  int nk = levels_needed(g, s, n, mode);
  if (have) {
    for (int j = tid; j < nk; j += bs) ev[j] = g.eig[o + j];
  } else {
    bisect_range(d, e2, n, t.glo, t.ghi, t.pivmin, 0, nk, t.unscale, tpe_max, kEigvalsTpeBlock, ev);
  }
  __syncthreads();
  if (mode == 1) {
    if (!have)
      for (int j = tid; j < n; j += bs) g.eig[o + j] = ev[j];
    if (tid == 0) g.nvec[s] = n;
    return;
  }
  const int warp = tid >> 5;
  __shared__ int last;
  __shared__ int need_more;
  for (int pass = 0; pass < 2; ++pass) {
    double ent = 0.0;
    if (warp == 0) warp_fermi(ev, nk, g.nel_a[s], kt, fa, ent);
    if (warp == 1) warp_fermi(ev, nk, g.nel_b[s], kt, fb, ent);
    if ((tid & 31) == 0 && warp < 2) red[warp] = ent;
    __syncthreads();
    if (tid == 0) {
      last = -1;
      need_more = (nk < n && fa[nk - 1] + fb[nk - 1] > 1e-14) ? 1 : 0;
    }
    __syncthreads();
    if (!need_more) break;
    bisect_range(d, e2, n, t.glo, t.ghi, t.pivmin, nk, n, t.unscale, 8, kEigvalsTpeBlock, ev);
    nk = n;
    __syncthreads();
  }
  for (int j = tid; j < n; j += bs) {
    const double f = j < nk ? fa[j] + fb[j] : 0.0;
    g.eig[o + j] = j < nk ? ev[j] : DBL_MAX;
    g.occ[o + j] = f;
    g.occ_eps[o + j] = j < nk ? f * ev[j] : 0.0;
    if (f > 1e-14) atomicMax(&last, j);
  }
  __syncthreads();
  if (tid == 0) {
    g.nvec[s] = last + 1;
    g.entropy[s] = red[0] + red[1];
  }
}

// Eigenvalues j0..j1-1 (ascending) of the scaled symmetric tridiagonal (d, e2)
// by multisection.  A group of tpe threads (a power of two, as many as a
// block of tpe_block threads has to spare, at most tpe_max <= 32) shares one
// eigenvalue: each thread evaluates four interleaved Sturm sequences
// (sturm4), so a round cuts the interval into 4 tpe + 1 parts.  tpe fixes
// every eigenvalue's sequence of brackets; the block's threads take the
// eigenvalues in turn, so the results do not depend on the actual block
// size.  Results are written unscaled (times `unscale`).
__device__ void bisect_range(const double* d, const double* e2, int n, double glo, double ghi,
                             double pivmin, int j0, int j1, double unscale, int tpe_max,
                             int tpe_block, double* ev) {
  const int cnt = j1 - j0;
  if (cnt <= 0) return;
  int tpe = 1;
  while (tpe < tpe_max && cnt * tpe * 2 <= tpe_block) tpe *= 2;
  const int r = threadIdx.x & (tpe - 1);
  const int lane = threadIdx.x & 31;
  const unsigned gmask = (tpe == 32 ? 0xffffffffu : ((1u << tpe) - 1u)) << (lane & ~(tpe - 1));
  const double inv_parts = 1.0 / (4 * tpe + 1);
  for (int jj = threadIdx.x / tpe; jj < cnt; jj += blockDim.x / tpe) {
    const int j = j0 + jj;
    double lo = glo, hi = ghi;
    for (int it = 0; it < 80; ++it) {
      const double w = hi - lo;
      if (w <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + 4.0 * pivmin) break;
      double x[4];
      int c[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) x[q] = lo + (4 * r + q + 1) * inv_parts * w;
      sturm4(d, e2, n, x, c);
      double nlo = lo, nhi = hi;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (c[q] <= j) nlo = x[q];
#pragma unroll
      for (int q = 3; q >= 0; --q)
        if (c[q] > j) nhi = x[q];
      for (int off = 1; off < tpe; off <<= 1) {
        nlo = fmax(nlo, __shfl_xor_sync(gmask, nlo, off));
        nhi = fmin(nhi, __shfl_xor_sync(gmask, nhi, off));
      }
      if (!(nlo > lo) && !(nhi < hi)) break;   // resolution limit reached
      lo = nlo;
      hi = nhi;
    }
    if (r == 0) ev[j] = 0.5 * (lo + hi) * unscale;
  }
}

__global__ void __launch_bounds__(128) k_inverse_iteration(EigArgs g, double ortol_rel) {
  const int s = g.list[blockIdx.x];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int64_t o = g.ao_off[s];
  inverse_iteration_block<128>(g.d + o, g.e + o, g.eig + o, g.nao[s], g.all_vectors ? g.nao[s] : g.nvec[s],
                               g.Z + g.mat_off[s], g.scratch + g.scratch_off[s], ortol_rel,
                               (uint32_t)s, 0, 128);
}

// Latency form for few systems: grid (parts, systems) of 16-thread CTAs whose
// work vectors live in shared memory (5 n 16 doubles) instead of global
// scratch; part p leads the clusters starting at p*16 + t, stepping 16 parts.
constexpr int kInvSmemThreads = 16;
__global__ void __launch_bounds__(kInvSmemThreads) k_inverse_iteration_smem(EigArgs g, double ortol_rel) {
  extern __shared__ double sm[];
  const int s = g.list[blockIdx.y];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int64_t o = g.ao_off[s];
  inverse_iteration_block<kInvSmemThreads>(g.d + o, g.e + o, g.eig + o, g.nao[s],
                                           g.all_vectors ? g.nao[s] : g.nvec[s],
                                           g.Z + g.mat_off[s], sm, ortol_rel, (uint32_t)s,
                                           blockIdx.x * kInvSmemThreads,
                                           gridDim.x * kInvSmemThreads);
}


// ---------------------------------------------------------------------------
// Blocked back-transform (compact WY form, LAPACK larft/larfb order): the
// reflectors H_i0 ... H_i0+31 of one block are I - V T V^T with T upper
// triangular, so each block costs one pass over Z: Z <- Z - V (T (V^T Z)).
// Blocks are applied from the last to the first.
// ---------------------------------------------------------------------------
constexpr int WB = 32;

// Reflectors i0 .. i0+k-1 of one block into V (L x WB, row stride WB + 1):
// V[r][c] = v_{i0+c}[i0+1+r], unit diagonal, zeros above it and past k.
// Reflector i is row i of the reduced matrix (columns i+2..n-1), so a warp
// reads one reflector with consecutive lanes (coalesced) and writes one
// column of V (stride WB + 1: no bank conflicts).
// With 256 threads a warp takes columns warp + 8 q (q < 4) and issues the
// loads of all four columns for 128 rows before storing any (one memory
// round trip per 128 rows instead of one per 32).
__device__ __forceinline__ void load_wy_block(const double* a, int n, int i0, int k, int L, double* V) {
  constexpr int P = WB + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (nw == 8) {
    for (int r0 = 0; r0 < L; r0 += 128) {
      double v[4][4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int c = warp + 8 * q;
        const double* row = a + (int64_t)(i0 + c) * n + i0 + 1;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int r = r0 + lane + 32 * u;
          v[q][u] = (c < k && r > c && r < L) ? row[r] : 0.0;
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int c = warp + 8 * q;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int r = r0 + lane + 32 * u;
          if (r < L) V[r * P + c] = (c < k && r == c) ? 1.0 : v[q][u];
        }
      }
    }
    return;
  }
  for (int c = warp; c < WB; c += nw) {
    const double* row = a + (int64_t)(i0 + c) * n + i0 + 1;
    for (int r = lane; r < L; r += 32) {
      double val = 0.0;
      if (c < k) {
        if (r == c) val = 1.0;
        else if (r > c) val = row[r];
      }
      V[r * P + c] = val;
    }
  }
}

size_t wy_factor_bytes(int n) { return ((size_t)n * (WB + 1) + 2 * WB * (WB + 1)) * sizeof(double); }

size_t backtransform_wy_bytes(int n, int m) {
  return ((size_t)n * (WB + 1) + WB * (WB + 1) + (size_t)WB * m + 8) * sizeof(double);
}

// T factor of every 32-reflector block (LAPACK larft, forward columnwise):
// H_i0 ... H_i0+k-1 = I - V T V^T with T upper triangular,
//   T[j][j] = tau_j,  T[0:j, j] = -tau_j T[0:j, 0:j] (V^T v_j)[0:j].
// Grid (blocks, systems): the blocks are independent, so the serial
// triangular recurrence runs once per block and in parallel over blocks, off
// the back-transform's critical path.  T goes to the system's scratch, block
// b at b WB^2 (row-major WB x WB, zeros below the diagonal).
__global__ void __launch_bounds__(256) k_wy_factor(EigArgs g) {
  extern __shared__ double sm[];
  const int s = g.list[blockIdx.y];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int n = g.nao[s];
  const int nr = n - 2;
  const int b = blockIdx.x;
  const int i0 = b * WB;
  if (nr <= 0 || i0 >= nr) return;   // uniform over the block
  const int k = min(WB, nr - i0);
  const int L = n - i0 - 1;
  constexpr int P = WB + 1;
  double* V = sm;
  double* G = V + (size_t)n * P;
  double* T = G + WB * P;
  const double* tau = g.tau + g.ao_off[s];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  load_wy_block(g.A + g.mat_off[s], n, i0, k, L, V);
  __syncthreads();
  // G[p][q] = v_p . v_q for p < q < k (v_q is zero above row q)
  for (int idx = tid; idx < WB * WB; idx += blockDim.x) {
    const int p = idx / WB, q = idx - (idx / WB) * WB;
    if (p < q && q < k) {
      double acc = 0.0;
      for (int r = q; r < L; ++r) acc = fma(V[r * P + p], V[r * P + q], acc);
      G[p * P + q] = acc;
    }
  }
  __syncthreads();
  if (warp == 0) {
    const double tl = lane < k ? tau[i0 + lane] : 0.0;   // one load, not one per column
    for (int j = 0; j < WB; ++j) {
      const double tj = __shfl_sync(0xffffffffu, tl, j);
      double t = 0.0;
      if (lane < j && j < k) {
        for (int q = lane; q < j; ++q) t = fma(T[lane * P + q], G[q * P + j], t);
        t *= -tj;
      }
      if (lane == j) t = tj;
      T[lane * P + j] = (lane <= j) ? t : 0.0;
      __syncwarp();
    }
    double* out = g.scratch + g.scratch_off[s] + wy_t_offset(n) + (int64_t)b * WB * WB;
    for (int j = 0; j < WB; ++j) out[lane * WB + j] = T[lane * P + j];
  }
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// load_wy_block and the T factor of block b, issued as asynchronous copies
// (one commit group) so that they overlap the work on the previous block;
// the unit diagonal and the zeros above it are plain stores.
__device__ __forceinline__ void prefetch_wy_block(const double* a, const double* tf, int n, int nr,
                                                  int b, double* V, double* T) {
  constexpr int P = WB + 1;
  const int i0 = b * WB, k = min(WB, nr - i0), L = n - i0 - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c = warp; c < WB; c += nw) {
    const double* row = a + (int64_t)(i0 + c) * n + i0 + 1;
    for (int r = lane; r < L; r += 32) {
      double* dst = V + r * P + c;
      if (c < k && r > c) cp_async8(dst, row + r);
      else *dst = (c < k && r == c) ? 1.0 : 0.0;
    }
  }
  for (int idx = threadIdx.x; idx < WB * WB; idx += blockDim.x)
    cp_async8(T + (idx / WB) * P + (idx % WB), tf + (int64_t)b * WB * WB + idx);
  cp_async_commit();
}

// Blocked back-transform (compact WY form, LAPACK larfb order): each block of
// 32 reflectors costs one pass over Z: Z <- Z - V (T (V^T Z)), blocks from the
// last to the first, T from k_wy_factor.  Grid (parts, systems): part
// blockIdx.x transforms its contiguous slice of the system's eigenvectors
// (parts > 1 only when few systems are active, so that one system's vectors
// are spread over several SMs).  STAGED: the slice lives in shared memory for
// the whole pass (few vectors per CTA), so no block waits on global loads of Z.
template <bool STAGED>
__global__ void __launch_bounds__(256) k_backtransform_wy(EigArgs g, int wcap, int per_cap) {
  extern __shared__ double sm[];
  const int s = g.list[blockIdx.y];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int n = g.nao[s];
  const int mt = g.all_vectors ? n : g.nvec[s];
  const int per = (mt + gridDim.x - 1) / gridDim.x;
  const int jbeg = blockIdx.x * per;
  const int m = min(mt - jbeg, per);
  const double* a = g.A + g.mat_off[s];
  const double* tf = g.scratch + g.scratch_off[s] + wy_t_offset(n);
  double* gZ = g.Z + g.mat_off[s] + (int64_t)jbeg * n;
  const int nr = n - 2;
  if (nr <= 0 || m <= 0) return;
  const int tid = threadIdx.x, bs = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = bs >> 5;
  constexpr int P = WB + 1;
  // V (n x P) and T (WB x P) of one block; STAGED keeps two of each so that
  // the next block arrives by cp.async while this one is applied
  double* V0 = sm;
  double* T0 = V0 + (size_t)n * P;
  double* V1 = STAGED ? T0 + WB * P : V0;
  double* T1 = STAGED ? V1 + (size_t)n * P : T0;
  double* W = T1 + WB * P;               // WB x wcap
  // per_cap x n staging buffer; a slice larger than planned stays in global memory
  const bool stage = STAGED && per <= per_cap;
  double* Z = stage ? W + (size_t)WB * wcap : gZ;
  if (stage)
    for (int64_t k = tid; k < (int64_t)m * n; k += bs) Z[k] = gZ[k];
  const int nblk = (nr + WB - 1) / WB;
  if (STAGED) prefetch_wy_block(a, tf, n, nr, nblk - 1, V0, T0);
  for (int it = 0; it < nblk; ++it) {
    const int b = nblk - 1 - it;
    const int i0 = b * WB;
    const int k = min(WB, nr - i0);
    const int L = n - i0 - 1;
    const bool odd = STAGED && (it & 1);
    double* V = odd ? V1 : V0;
    double* T = odd ? T1 : T0;
    if (STAGED) {
      if (b > 0) {
        prefetch_wy_block(a, tf, n, nr, b - 1, odd ? V0 : V1, odd ? T0 : T1);
        cp_async_wait<1>();   // this block's copies are done, the next one's may fly
      } else {
        cp_async_wait<0>();
      }
    } else {
      load_wy_block(a, n, i0, k, L, V);
      for (int idx = tid; idx < WB * WB; idx += bs) {
        const int p = idx / WB, q = idx - (idx / WB) * WB;
        T[p * P + q] = tf[(int64_t)b * WB * WB + idx];
      }
    }
    __syncthreads();
    // eigenvectors in chunks of at most wcap (the W buffer's capacity)
    for (int j0 = 0; j0 < m; j0 += wcap) {
    const int jc = min(wcap, m - j0);
    // W = T (V^T Z_block): one warp per eigenvector, lane = reflector
    for (int jj = warp; jj < jc; jj += nw) {
      const int j = j0 + jj;
      const double* z = Z + (int64_t)j * n + i0 + 1;
      double acc = 0.0;
      for (int r0 = 0; r0 < L; r0 += 32) {
        const double zv = (r0 + lane < L) ? z[r0 + lane] : 0.0;
        const int rmax = min(32, L - r0);
        for (int rr = 0; rr < rmax; ++rr) {
          const double zr = __shfl_sync(0xffffffffu, zv, rr);
          const int r = r0 + rr;
          if (lane < k && r >= lane) acc = fma(V[r * P + lane], zr, acc);
        }
      }
      double w2 = 0.0;
      for (int q = 0; q < WB; ++q) {
        const double w1 = __shfl_sync(0xffffffffu, acc, q);
        if (q >= lane) w2 = fma(T[lane * P + q], w1, w2);
      }
      W[lane * wcap + jj] = w2;
    }
    __syncthreads();
    for (int64_t idx = tid; idx < (int64_t)jc * L; idx += bs) {
      const int jj = (int)(idx / L), r = (int)(idx - (idx / L) * L);
      const int amax = min(k, r + 1);
      double acc = 0.0;
      for (int q = 0; q < amax; ++q) acc = fma(V[r * P + q], W[q * wcap + jj], acc);
      Z[(int64_t)(j0 + jj) * n + i0 + 1 + r] -= acc;
    }
    __syncthreads();
    }
  }
  if (stage)
    for (int64_t k = tid; k < (int64_t)m * n; k += bs) gZ[k] = Z[k];
}

// Blocked back-transform on the FP64 tensor cores (many systems, one CTA per
// system): per 32-reflector block, Y = V^T Z (32 x m) as 8 x 8 x 4 DMMA tiles,
// each warp a strip of four 8-row blocks for one block of eight eigenvectors
// (one global load of Z feeds four products), W = T Y in shared memory, and
// Z <- Z - V W as transposed tiles (eigenvector x row: each lane updates two
// adjacent rows of one eigenvector).  Z stays in global memory (vector-major
// rows of n), V and T of the block in shared memory.
__global__ void __launch_bounds__(256) k_backtransform_dmma(EigArgs g, int mcap) {
  extern __shared__ double sm[];
  const int s = g.list[blockIdx.x];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int n = g.nao[s];
  const int m = g.all_vectors ? n : g.nvec[s];
  const int nr = n - 2;
  if (nr <= 0 || m <= 0) return;
  constexpr int P = WB + 1;
  const double* a = g.A + g.mat_off[s];
  const double* tf = g.scratch + g.scratch_off[s] + wy_t_offset(n);
  double* Z = g.Z + g.mat_off[s];
  double* V = sm;                        // n x P
  double* T = V + (size_t)n * P;         // WB x P
  double* Y = T + WB * P;                // WB x mcap
  double* Wm = Y + (size_t)WB * mcap;    // WB x mcap
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const int nblk = (nr + WB - 1) / WB;
  for (int it = 0; it < nblk; ++it) {
    const int b = nblk - 1 - it;
    const int i0 = b * WB;
    const int k = min(WB, nr - i0);
    const int L = n - i0 - 1;
    __syncthreads();
    load_wy_block(a, n, i0, k, L, V);
    for (int idx = tid; idx < WB * WB; idx += blockDim.x)
      T[(idx / WB) * P + (idx % WB)] = tf[(int64_t)b * WB * WB + idx];
    __syncthreads();
    // eigenvectors in chunks of mcap (the Y and W buffers' width): the count
    // of a system's needed vectors is set on the device and can exceed the
    // bucket's estimate
    for (int j0 = 0; j0 < m; j0 += mcap) {
      const int mc = min(mcap, m - j0);
      const int jb_count = (mc + 7) / 8;
      // Y = V^T Z over the block's rows
      for (int jb = warp; jb < jb_count; jb += nw) {
        double d[4][2];
#pragma unroll
        for (int q = 0; q < 4; ++q) d[q][0] = d[q][1] = 0.0;
        const int jl = jb * 8 + gq;
        const double* z = Z + (int64_t)(j0 + jl) * n + i0 + 1;
        // four K steps' loads of Z issued before their products (the
        // products run in the same order as one step at a time)
        for (int r0 = 0; r0 < L; r0 += 16) {
          double bz[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int r = r0 + 4 * u + tq;
            bz[u] = (jl < mc && r < L) ? z[r] : 0.0;
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int r = r0 + 4 * u + tq;
            if (r0 + 4 * u < L) {
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                const double av = r < L ? V[r * P + q * 8 + gq] : 0.0;
                mma_f64(d[q], av, bz[u]);
              }
            }
          }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int h = 0; h < 2; ++h) Y[(q * 8 + gq) * mcap + jb * 8 + 2 * tq + h] = d[q][h];
      }
      __syncthreads();
      // W = T Y (T upper triangular)
      for (int idx = tid; idx < WB * mc; idx += blockDim.x) {
        const int p = idx / mc, jj = idx - (idx / mc) * mc;
        double acc = 0.0;
        for (int q = p; q < WB; ++q) acc = fma(T[p * P + q], Y[q * mcap + jj], acc);
        Wm[p * mcap + jj] = acc;
      }
      __syncthreads();
      // Z^T tile (eigenvectors jb x rows rb) -= W^T V^T
      const int rb_count = (L + 7) / 8;
      for (int t = warp; t < jb_count * rb_count; t += nw) {
        const int jb = t / rb_count, rb = t - (t / rb_count) * rb_count;
        double d[2] = {0.0, 0.0};
        const int jl = jb * 8 + gq, rr = rb * 8 + gq;
        // the two elements of Z this lane updates, loaded before the products
        double* z = Z + (int64_t)(j0 + jl) * n + i0 + 1;
        double zold[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = rb * 8 + 2 * tq + h;
          zold[h] = (jl < mc && r < L) ? z[r] : 0.0;
        }
#pragma unroll
        for (int q0 = 0; q0 < WB; q0 += 4) {
          const double aw = jl < mc ? Wm[(q0 + tq) * mcap + jl] : 0.0;
          const double bv = rr < L ? V[rr * P + q0 + tq] : 0.0;
          mma_f64(d, aw, bv);
        }
        if (jl < mc) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = rb * 8 + 2 * tq + h;
            if (r < L) z[r] = zold[h] - d[h];
          }
        }
      }
      __syncthreads();
    }
  }
}

size_t backtransform_dmma_bytes(int n, int mcap) {
  return ((size_t)n * (WB + 1) + WB * (WB + 1) + 2 * (size_t)WB * mcap) * sizeof(double);
}

void launch_wy_factor(const EigArgs& g, int count, int max_n, cudaStream_t stream) {
  if (count == 0) return;
  allow_max_dynamic_smem(k_wy_factor);
  const int nblk = std::max(1, (max_n - 2 + WB - 1) / WB);
  k_wy_factor<<<dim3(nblk, count), 256, wy_factor_bytes(max_n), stream>>>(g);
}

void launch_backtransform_wy(const EigArgs& g, int count, int max_n, int max_m, int want_m,
                             cudaStream_t stream, bool factored) {
  if (count == 0) return;
  const size_t cap = allow_max_dynamic_smem(k_backtransform_wy<false>);
  const size_t cap_s = allow_max_dynamic_smem(k_backtransform_wy<true>);
  if (!factored) launch_wy_factor(g, count, max_n, stream);
  // Few systems: split each system's vectors over CTAs, at least 8 vectors
  // each, and keep each CTA's slice in shared memory when it fits.
  const int sms = sm_count();
  const int parts = count >= sms ? 1 : std::max(1, std::min((want_m + 7) / 8, 2 * sms / count));
  const int per = (want_m + parts - 1) / parts;
  const int wc = std::min(max_m, per);
  const size_t staged = backtransform_wy_bytes(max_n, wc) + (size_t)per * max_n * sizeof(double) +
                        ((size_t)max_n * (WB + 1) + WB * (WB + 1)) * sizeof(double);
  if (parts > 1 && staged <= cap_s) {
    k_backtransform_wy<true><<<dim3(parts, count), 256, staged, stream>>>(g, wc, per);
    return;
  }
  // one CTA per system: the block products on the FP64 tensor cores
  const int mcap = (want_m + 7) / 8 * 8;
  const size_t capd = allow_max_dynamic_smem(k_backtransform_dmma);
  if (parts == 1 && backtransform_dmma_bytes(max_n, mcap) <= capd) {
    k_backtransform_dmma<<<count, 256, backtransform_dmma_bytes(max_n, mcap), stream>>>(g, mcap);
    return;
  }
  (void)cap;
  k_backtransform_wy<false><<<dim3(parts, count), 256, backtransform_wy_bytes(max_n, max_m), stream>>>(
      g, max_m, 0);
}

// ---------------------------------------------------------------------------
// Large systems (a 32-reflector block of n rows no longer fits in shared
// memory): the same compact-WY algebra with the reflectors streamed through
// shared memory in chunks of rows.
// ---------------------------------------------------------------------------
constexpr int kWyRows = 128;

// Rows r0 .. r0+rc-1 of the block's V (row stride WB + 1): one warp per
// reflector, lanes along the reflector's row of the matrix (coalesced).
__device__ __forceinline__ void load_wy_rows(const double* a, int n, int i0, int k, int r0, int rc,
                                             double* Vc) {
  constexpr int P = WB + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c = warp; c < WB; c += nw) {
    const double* row = a + (int64_t)(i0 + c) * n + i0 + 1;
    for (int r = lane; r < rc; r += 32) {
      const int rr = r0 + r;
      double val = 0.0;
      if (c < k) {
        if (rr == c) val = 1.0;
        else if (rr > c) val = row[rr];
      }
      Vc[r * P + c] = val;
    }
  }
}

// T factors as k_wy_factor, with G = V^T V accumulated over row chunks (each
// thread sums its pairs in ascending row order, as the one-tile kernel does).
__global__ void __launch_bounds__(256) k_wy_factor_rows(EigArgs g) {
  extern __shared__ double sm[];
  const int s = g.list[blockIdx.y];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int n = g.nao[s];
  const int nr = n - 2;
  const int b = blockIdx.x;
  const int i0 = b * WB;
  if (nr <= 0 || i0 >= nr) return;   // uniform over the block
  const int k = min(WB, nr - i0);
  const int L = n - i0 - 1;
  constexpr int P = WB + 1;
  constexpr int RC = 2 * kWyRows;
  double* Vc = sm;
  double* G = Vc + RC * P;
  double* T = G + WB * P;
  const double* tau = g.tau + g.ao_off[s];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int kPer = WB * WB / 256;
  double acc[kPer];
#pragma unroll
  for (int u = 0; u < kPer; ++u) acc[u] = 0.0;
  for (int r0 = 0; r0 < L; r0 += RC) {
    const int rc = min(RC, L - r0);
    load_wy_rows(g.A + g.mat_off[s], n, i0, k, r0, rc, Vc);
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int idx = tid + 256 * u;
      const int p = idx / WB, q = idx - (idx / WB) * WB;
      if (p < q && q < k)
        for (int r = max(q - r0, 0); r < rc; ++r) acc[u] = fma(Vc[r * P + p], Vc[r * P + q], acc[u]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int idx = tid + 256 * u;
    const int p = idx / WB, q = idx - (idx / WB) * WB;
    if (p < q && q < k) G[p * P + q] = acc[u];
  }
  __syncthreads();
  if (warp == 0) {
    const double tl = lane < k ? tau[i0 + lane] : 0.0;
    for (int j = 0; j < WB; ++j) {
      const double tj = __shfl_sync(0xffffffffu, tl, j);
      double t = 0.0;
      if (lane < j && j < k) {
        for (int q = lane; q < j; ++q) t = fma(T[lane * P + q], G[q * P + j], t);
        t *= -tj;
      }
      if (lane == j) t = tj;
      T[lane * P + j] = (lane <= j) ? t : 0.0;
      __syncwarp();
    }
    double* out = g.scratch + g.scratch_off[s] + wy_t_offset(n) + (int64_t)b * WB * WB;
    for (int j = 0; j < WB; ++j) out[lane * WB + j] = T[lane * P + j];
  }
}

size_t wy_factor_rows_bytes() { return ((size_t)2 * kWyRows * (WB + 1) + 2 * WB * (WB + 1)) * sizeof(double); }

// Back-transform of large systems: grid (vector slices of MC, systems); each
// CTA keeps its MC eigenvectors in shared memory for the whole pass and, per
// block (last to first), forms Y = V^T Z over row chunks, W = T Y, and
// Z -= V W over the same chunks, the reflectors read from the matrix (L2).
template <int MC>
__global__ void __launch_bounds__(256) k_backtransform_rows(EigArgs g) {
  extern __shared__ double sm[];
  const int s = g.list[blockIdx.y];
  if (g.only != nullptr && g.only[s] == 0) return;
  const int n = g.nao[s];
  const int mt = g.all_vectors ? n : g.nvec[s];
  const int nr = n - 2;
  if (nr <= 0) return;
  const double* a = g.A + g.mat_off[s];
  const double* tf = g.scratch + g.scratch_off[s] + wy_t_offset(n);
  constexpr int P = WB + 1;
  double* Z = sm;                          // MC x n
  double* Vc = Z + (size_t)MC * n;         // kWyRows x P
  double* T = Vc + kWyRows * P;            // WB x P
  double* Y = T + WB * P;                  // WB x MC
  double* W = Y + WB * MC;                 // WB x MC
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const int nblk = (nr + WB - 1) / WB;
  // slices of MC eigenvectors; the count of needed vectors is set on the
  // device, so a CTA takes every gridDim.x-th slice until all are done
  for (int jbeg = blockIdx.x * MC; jbeg < mt; jbeg += gridDim.x * MC) {
    const int m = min(mt - jbeg, MC);
    double* gZ = g.Z + g.mat_off[s] + (int64_t)jbeg * n;
    __syncthreads();
    for (int64_t k = tid; k < (int64_t)m * n; k += blockDim.x) Z[k] = gZ[k];
    for (int it = 0; it < nblk; ++it) {
      const int b = nblk - 1 - it;
      const int i0 = b * WB;
      const int k = min(WB, nr - i0);
      const int L = n - i0 - 1;
      for (int idx = tid; idx < WB * WB; idx += blockDim.x)
        T[(idx / WB) * P + (idx % WB)] = tf[(int64_t)b * WB * WB + idx];
      for (int idx = tid; idx < WB * MC; idx += blockDim.x) Y[idx] = 0.0;
      // Y = V^T Z: lane = reflector, warps over this CTA's vectors
      for (int r0 = 0; r0 < L; r0 += kWyRows) {
        const int rc = min(kWyRows, L - r0);
        __syncthreads();
        load_wy_rows(a, n, i0, k, r0, rc, Vc);
        __syncthreads();
        for (int j = warp; j < m; j += nw) {
          const double* z = Z + (int64_t)j * n + i0 + 1 + r0;
          double acc = 0.0;
          for (int r = 0; r < rc; ++r) acc = fma(Vc[r * P + lane], z[r], acc);
          Y[lane * MC + j] += acc;
        }
      }
      __syncthreads();
      // W = T Y (T upper triangular)
      for (int idx = tid; idx < WB * MC; idx += blockDim.x) {
        const int p = idx / MC, j = idx - (idx / MC) * MC;
        double acc = 0.0;
        for (int q = p; q < WB; ++q) acc = fma(T[p * P + q], Y[q * MC + j], acc);
        W[idx] = acc;
      }
      // Z -= V W
      for (int r0 = 0; r0 < L; r0 += kWyRows) {
        const int rc = min(kWyRows, L - r0);
        __syncthreads();
        load_wy_rows(a, n, i0, k, r0, rc, Vc);
        __syncthreads();
        for (int idx = tid; idx < rc * m; idx += blockDim.x) {
          const int j = idx / rc, r = idx - (idx / rc) * rc;
          const int qmax = min(k, r0 + r + 1);
          double acc = 0.0;
          for (int q = 0; q < qmax; ++q) acc = fma(Vc[r * P + q], W[q * MC + j], acc);
          Z[(int64_t)j * n + i0 + 1 + r0 + r] -= acc;
        }
      }
      __syncthreads();
    }
    for (int64_t k = tid; k < (int64_t)m * n; k += blockDim.x) gZ[k] = Z[k];
  }
}

template <int MC>
size_t backtransform_rows_bytes(int n) {
  return ((size_t)MC * n + kWyRows * (WB + 1) + WB * (WB + 1) + 2 * WB * MC) * sizeof(double);
}

void launch_backtransform_rows(const EigArgs& g, int count, int max_n, int want_m, cudaStream_t stream) {
  if (count == 0) return;
  const int nblk = std::max(1, (max_n - 2 + WB - 1) / WB);
  const size_t capf = allow_max_dynamic_smem(k_wy_factor_rows);
  (void)capf;
  k_wy_factor_rows<<<dim3(nblk, count), 256, wy_factor_rows_bytes(), stream>>>(g);
  const size_t cap16 = allow_max_dynamic_smem(k_backtransform_rows<16>);
  if (backtransform_rows_bytes<16>(max_n) <= cap16) {
    k_backtransform_rows<16><<<dim3((want_m + 15) / 16, count), 256, backtransform_rows_bytes<16>(max_n),
                               stream>>>(g);
    return;
  }
  const size_t cap4 = allow_max_dynamic_smem(k_backtransform_rows<4>);
  (void)cap4;
  k_backtransform_rows<4><<<dim3((want_m + 3) / 4, count), 256, backtransform_rows_bytes<4>(max_n), stream>>>(g);
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

int sm_count() {
  static const int n = [] {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    return v;
  }();
  return n;
}

void launch_eigvals(const EigArgs& g, int mode, double kt, int count, int max_n, int max_levels,
                    cudaStream_t stream) {
  if (count == 0) return;
  const int kNumSMs = sm_count();
  const size_t sm = (5 * (size_t)max_n + 40) * sizeof(double);
  const size_t cap = allow_max_dynamic_smem(k_tridiag_eigvals);
  (void)cap;
  // Enough systems to fill the GPU: one CTA each, one thread per eigenvalue
  // (fewest Sturm sequences in total), and in the SCC (mode 0) no more
  // threads than the bucket's needed levels (at least the two Fermi warps),
  // so that more systems share an SM.  Few systems: spread each system's
  // eigenvalues over several CTAs, up to a warp per eigenvalue (fewest rounds).
  if (count >= kNumSMs) {
    int threads = kEigvalsTpeBlock;
    if (mode == 0) threads = std::max(64, std::min(kEigvalsTpeBlock, (std::min(max_levels, max_n) + 31) / 32 * 32));
    k_tridiag_eigvals<<<count, threads, sm, stream>>>(g, mode, kt, 0, 1);
    return;
  }
  // Sturm steps are issue-bound: 128-thread parts (a warp per scheduler,
  // two eigenvalues per warp, 16 threads each) take the fewest cycles per
  // round for the rounds they need.
  const int need = mode == 0 ? max_n / 2 + 16 : max_n;
  const int parts = std::max(1, std::min((need + 7) / 8, 2 * kNumSMs / count));
  const size_t smp = (2 * (size_t)max_n + 40) * sizeof(double);
  k_eigvals_part<<<dim3(parts, count), 128, smp, stream>>>(g, mode, parts);
  k_tridiag_eigvals<<<count, 256, sm, stream>>>(g, mode, kt, 1, 8);
}

void launch_inverse_iteration(const EigArgs& g, int count, int max_n, int want_m, double ortol_rel,
                              cudaStream_t stream) {
  if (count == 0) return;
  const size_t smem = (size_t)5 * max_n * kInvSmemThreads * sizeof(double);
  const size_t cap = allow_max_dynamic_smem(k_inverse_iteration_smem);
  if (count < sm_count() && smem <= cap) {
    const int parts = std::max(1, (want_m + kInvSmemThreads - 1) / kInvSmemThreads);
    k_inverse_iteration_smem<<<dim3(parts, count), kInvSmemThreads, smem, stream>>>(g, ortol_rel);
    return;
  }
  k_inverse_iteration<<<count, 128, 0, stream>>>(g, ortol_rel);
}


void launch_lowdin_weights(const EigArgs& g, int32_t* status, int count, cudaStream_t stream) {
  if (count == 0) return;
  k_lowdin_weights<<<count, 256, 0, stream>>>(g, status);
}

}  // namespace xtb
