// Householder tridiagonalisation with the matrix held in registers across a
// thread-block cluster (sm_100a), one cluster barrier per column.
//
// One cluster of G CTAs reduces one system's full symmetric n x n matrix
// (n <= NMAX).  Warp wg = rank * NW + warp of the cluster owns rows
// r = wg + R i (R = G * NW warps, i < IR); lane l owns columns c = l + 32 j
// (j < JC).  Every element lives in exactly one register of one thread.
//
// A^(m) is the matrix after reflectors 0..m-1 (LAPACK sytd2 order, lower).
// Entering step k, every CTA holds in shared memory, posted by the row
// owners during step k-1:  C = column k of A^(k-1) and P = p_{k-1} =
// tau_{k-1} A^(k-1) v_{k-1} (rows >= k), and every warp holds x_{k-1} in
// registers.  Step k then runs without any exchange until its end:
//   (1) every warp, redundantly: w_{k-1} = p - (tau/2)(p.v) v, column k of
//       A^(k) = C - v w[k] - w (v[k] = 1), its norm, and reflector k
//       (beta, tau, v_k = x_k / (alpha - beta));
//   (2) own rows: the trailing block (rows, columns > k) is updated with
//       reflector k-1 and multiplied by v_k in the same pass; row sums give
//       p_k;
//   (3) the owners post p_k and column k+1 of A^(k) into every CTA.
//       -- cluster barrier --
// Buffers alternate by step parity: a CTA writes parity (k+1) & 1 only after
// the barrier of step k-1, when every CTA has finished reading it.
// Outputs match the shared-memory kernel: d, e, tau, and reflector k in row k
// of the global matrix (columns k+2..n-1; v[k+1] = 1 implicit).
//
// Reference behaviour: the reduction LAPACK's dsytrd performs inside dsyevd
// (model/gfn2/eigensolver.cpp:1221-1254 of the reference calls it on the
// Cholesky-reduced matrix); the eigenpairs are basis independent.
#include <cooperative_groups.h>

#include "kernels.cuh"

#include <algorithm>
#include <type_traits>

namespace xtb {
namespace cg = cooperative_groups;

namespace {

// v[idx] for an index known to lie in [LO, HI] and uniform over the warp:
// HI - LO selects instead of an indexed (local-memory) access.
template <int LO, int HI, int N>
__device__ __forceinline__ double pick(const double (&v)[N], int idx) {
  double t = v[LO];
#pragma unroll
  for (int j = LO + 1; j <= HI; ++j)
    if (j == idx) t = v[j];
  return t;
}

// Column-register slot of row slot i of a warp: rows r = wg + R i with
// wg < R, so r >> 5 lies in [(R i) >> 5, (R i + R - 1) >> 5].
template <int R, int JC, int I = 0, int IRMAX = 8>
__device__ __forceinline__ double pick_row(const double (&v)[JC], int i, int slot) {
  if constexpr (I >= IRMAX) {
    return 0.0;
  } else {
    if (i == I) {
      constexpr int LO = (R * I) >> 5;
      constexpr int HI0 = (R * I + R - 1) >> 5;
      constexpr int HI = HI0 < JC ? HI0 : JC - 1;
      return pick<LO < JC ? LO : JC - 1, HI>(v, slot);
    }
    return pick_row<R, JC, I + 1, IRMAX>(v, i, slot);
  }
}

// Calls f(std::integral_constant<int, jb>) for a runtime jb in [J, JC).
template <int J, int JC, class F>
__device__ __forceinline__ bool dispatch(int jb, F& f) {
  if constexpr (J + 1 >= JC) {
    return f(std::integral_constant<int, J>{});
  } else {
    if (jb == J) return f(std::integral_constant<int, J>{});
    return dispatch<J + 1, JC>(jb, f);
  }
}

template <int G, int NT, int NMAX>
__global__ void __launch_bounds__(NT) k_tridiag_reg(EigArgs g, const int32_t* list) {
  constexpr int NW = NT / 32;
  constexpr int R = G * NW;
  constexpr int IR = (NMAX + R - 1) / R;
  constexpr int JC = NMAX / 32;
  static_assert(IR * G <= 32, "one lane per (row slot, CTA) pair");
  static_assert(R * IR == NMAX && JC * 32 == NMAX, "rows and columns tile NMAX exactly");
  static_assert((IR & (IR - 1)) == 0, "row slots per warp must be a power of two");
  static_assert(R % 32 == 0 || 32 % R == 0, "row slots map to column registers by a fixed rule");
  cg::cluster_group cluster = cg::this_cluster();
  const int crank = (int)cluster.block_rank();
  const int s = list[blockIdx.x / G];
  // uniform over the cluster (every CTA of it has the same system): all of
  // them return before any cluster barrier
  if (g.only != nullptr && g.only[s] == 0) return;
  const int n = g.nao[s];
  double* ga = g.A + g.mat_off[s];
  double* d = g.d + g.ao_off[s];
  double* e = g.e + g.ao_off[s];
  double* tau = g.tau + g.ao_off[s];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wg = crank * NW + warp;

  __shared__ double C[2][NMAX];     // column k of A^(k-1), rows >= k, by step parity
  __shared__ double P[2][NMAX];     // p_{k-1}, rows >= k

  if (n <= 2) {   // uniform over the cluster; no cluster barrier is reached
    if (crank == 0 && tid == 0) {
      if (n == 2) {
        d[0] = ga[0];
        e[0] = ga[1];
        tau[0] = 0.0;
        d[1] = ga[3];
        e[1] = 0.0;
        tau[1] = 0.0;
      } else {
        d[0] = ga[0];
        e[0] = 0.0;
        tau[0] = 0.0;
      }
    }
    return;
  }

  double a[IR][JC];
#pragma unroll
  for (int i = 0; i < IR; ++i) {
    const int r = wg + R * i;
#pragma unroll
    for (int j = 0; j < JC; ++j) {
      const int c = lane + 32 * j;
      a[i][j] = (r < n && c < n) ? ga[(int64_t)r * n + c] : 0.0;
    }
  }
  for (int k = tid; k < 2 * NMAX; k += NT) {
    (&C[0][0])[k] = 0.0;
    (&P[0][0])[k] = 0.0;
  }
  // stores into the exchange arrays of CTA q of the cluster
  auto remote = [&](double* local, int q) { return cluster.map_shared_rank(local, q); };
  // lane l sends row slot l % IR to CTA l / IR
  const int pslot = lane & (IR - 1);
  const int prow = wg + R * pslot;
  const int pcta = lane / IR;
  // row r = wg + R i of this warp lives in column register slot r >> 5 of lane r & 31
  auto rslot = [&](int i) { return (wg + R * i) >> 5; };
  auto rlane = [&](int i) { return (wg + R * i) & 31; };

  cluster.sync();   // every CTA's buffers are zero before anyone posts
  {
    double t[IR];
#pragma unroll
    for (int i = 0; i < IR; ++i) t[i] = __shfl_sync(0xffffffffu, a[i][0], 0);
    if (lane < IR * G && prow < n) {
      double v = t[0];
#pragma unroll
      for (int i = 1; i < IR; ++i)
        if (i == pslot) v = t[i];
      *remote(&C[0][prow], pcta) = v;
    }
  }
  cluster.sync();

  // reflector k-1 in the column layout: x (column k-1 of A^(k-1) at c >= k),
  // v = sc x with v[k] = 1, tau
  double xp[JC];
#pragma unroll
  for (int j = 0; j < JC; ++j) xp[j] = 0.0;
  double scp = 0.0, taup = 0.0;
  int k = 0;
  // One column step with JB = k >> 5 known at compile time: columns below
  // 32 JB are finished, so every loop starts at slot JB.
  auto step = [&](auto jbc) -> bool {
    constexpr int JB = decltype(jbc)::value;
    constexpr int JN = JB + 1 < JC ? JB + 1 : JB;   // slot of column k+1
    const int b = k & 1, nb = b ^ 1;
    const bool prev = k >= 1;
    const bool next = k + 2 < n;    // reflector k exists
    // ---- (1) w_{k-1}, column k of A^(k), reflector k (every warp) ----
    double wp[JC], xk[JC];
#pragma unroll
    for (int j = 0; j < JB; ++j) wp[j] = xk[j] = 0.0;   // finished columns
    // v_{k-1} at column slot j (recomputed where needed: fewer live registers)
    auto vpj = [&](int j) {
      const int c = lane + 32 * j;
      return (prev && c >= k && c < n) ? (c == k ? 1.0 : scp * xp[j]) : 0.0;
    };
    double pv = 0.0;
#pragma unroll
    for (int j = JB; j < JC; ++j) {
      const int c = lane + 32 * j;
      const bool act = prev && c >= k && c < n;
      wp[j] = act ? P[b][c] : 0.0;
      pv = fma(wp[j], vpj(j), pv);
    }
    pv = warp_sum(pv);
    const double kw = 0.5 * taup * pv;
#pragma unroll
    for (int j = JB; j < JC; ++j) wp[j] = fma(-kw, vpj(j), wp[j]);
    const double wk = __shfl_sync(0xffffffffu, wp[JB], k & 31);
    double nrm = 0.0;
#pragma unroll
    for (int j = JB; j < JC; ++j) {
      const int c = lane + 32 * j;
      double v = (c >= k && c < n) ? C[b][c] : 0.0;
      v -= vpj(j) * wk + wp[j];   // v_{k-1}[k] = 1; zero where !prev
      xk[j] = v;
      if (c >= k + 2 && c < n) nrm = fma(v, v, nrm);
    }
    nrm = warp_sum(nrm);
    const double dk = __shfl_sync(0xffffffffu, xk[JB], k & 31);
    const double alpha = __shfl_sync(0xffffffffu, pick<JB, JN>(xk, (k + 1) >> 5), (k + 1) & 31);
    double ti = 0.0, sc = 0.0, beta = alpha;
    if (next && nrm > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + nrm), alpha);
      ti = (beta - alpha) / beta;
      sc = 1.0 / (alpha - beta);
    }
    if (crank == 0 && tid == 0) {
      d[k] = dk;
      e[k] = beta;   // for k = n-2 this is the updated (n-1, n-2) element
      tau[k] = ti;
    }
    if (next && crank == 0 && warp == 0) {
#pragma unroll
      for (int j = JB; j < JC; ++j) {
        const int c = lane + 32 * j;
        if (c >= k + 2 && c < n) ga[(int64_t)k * n + c] = sc * xk[j];
      }
    }
    // ---- (2) own rows > k: update with reflector k-1, multiply by v_k ----
    double vr[IR], wr[IR], acc[IR];
#pragma unroll
    for (int i = 0; i < IR; ++i) {
      const int r = wg + R * i;
      const bool act = r >= k + 1 && r < n;   // uniform over the warp
      // rows below 32 JB are finished; the slot of row r lies in
      // [(R i) >> 5, (R i + R - 1) >> 5] whatever the warp
      double v = 0.0, w = 0.0;
      if (act) {
        // v_{k-1}[r] for r > k is sc x[r]
        v = scp * __shfl_sync(0xffffffffu, pick_row<R, JC>(xp, i, rslot(i)), rlane(i));
        w = __shfl_sync(0xffffffffu, pick_row<R, JC>(wp, i, rslot(i)), rlane(i));
      }
      vr[i] = v;
      wr[i] = w;
      acc[i] = 0.0;
    }
#pragma unroll
    for (int j = JB; j < JC; ++j) {
      const int c = lane + 32 * j;
      const bool cact = c >= k + 1 && c < n;
      const double vc = cact ? vpj(j) : 0.0;
      const double wc = cact ? wp[j] : 0.0;
      const double nc = (next && cact) ? (c == k + 1 ? 1.0 : sc * xk[j]) : 0.0;
#pragma unroll
      for (int i = 0; i < IR; ++i) {
        if (wg + R * i < k + 1) continue;   // uniform over the warp
        double x = fma(-vr[i], wc, a[i][j]);
        x = fma(-wr[i], vc, x);
        a[i][j] = x;
        acc[i] = fma(x, nc, acc[i]);
      }
    }
    if (!next) {
      // last step: the (n-1, n-1) element of A^(n-2) is final
#pragma unroll
      for (int i = 0; i < IR; ++i) {
        const int r = wg + R * i;
#pragma unroll
        for (int j = JB; j < JC; ++j)
          if (r == n - 1 && lane + 32 * j == n - 1) {
            d[n - 1] = a[i][j];
            e[n - 1] = 0.0;
            tau[n - 1] = 0.0;
          }
      }
      return true;
    }
    // row sums: butterfly reduce-scatter over the IR slots, then across lanes
#pragma unroll
    for (int sh = IR / 2; sh >= 1; sh >>= 1) {
      const bool up = (lane & sh) != 0;
#pragma unroll
      for (int q = 0; q < sh; ++q) {
        const double send = up ? acc[q] : acc[q + sh];
        const double keep = up ? acc[q + sh] : acc[q];
        acc[q] = keep + __shfl_xor_sync(0xffffffffu, send, sh);
      }
    }
#pragma unroll
    for (int sh = IR; sh < 32; sh <<= 1) acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], sh);
    // ---- (3) post p_k (lane l holds row slot l % IR) and column k+1 of A^(k) ----
    const bool post = lane < IR * G && prow >= k + 1 && prow < n;
    if (post) *remote(&P[nb][prow], pcta) = ti * acc[0];
    double t[IR];
#pragma unroll
    for (int i = 0; i < IR; ++i)
      t[i] = __shfl_sync(0xffffffffu, pick<JB, JN>(a[i], (k + 1) >> 5), (k + 1) & 31);
    if (post) {
      double v = t[0];
#pragma unroll
      for (int i = 1; i < IR; ++i)
        if (i == pslot) v = t[i];
      *remote(&C[nb][prow], pcta) = v;
    }
#pragma unroll
    for (int j = JB; j < JC; ++j) xp[j] = xk[j];
    scp = sc;
    taup = ti;
    cluster.sync();
    return false;
  };
  for (; k + 1 < n; ++k)
    if (dispatch<0, JC>(k >> 5, step)) break;
  // no CTA may leave while others could still store into its shared memory
  cluster.sync();
}

template <int G, int NT, int NMAX>
cudaError_t launch_cfg(const EigArgs& g, const int32_t* list, int count, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(G * count, 1, 1);
  cfg.blockDim = dim3(NT, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = G;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_tridiag_reg<G, NT, NMAX>, g, list);
}

}  // namespace

int tridiag_reg_max_n() { return 256; }

// Tridiagonalises the systems of `list` (all with n <= 256), one cluster per
// system; meant for few systems (it trades SM time for a shorter critical
// path per column).
void launch_tridiag_reg(const EigArgs& g, const int32_t* list, int count, int max_n,
                        cudaStream_t stream) {
  if (count == 0) return;
  if (max_n <= 64) launch_cfg<4, 128, 64>(g, list, count, stream);
  else if (max_n <= 128) launch_cfg<8, 128, 128>(g, list, count, stream);
  else launch_cfg<8, 256, 256>(g, list, count, stream);
}

}  // namespace xtb
