// Householder tridiagonalisation with the matrix held in registers across a
// thread-block cluster (sm_100a).
//
// One cluster of G CTAs reduces one system's full symmetric n x n matrix
// (n <= NMAX).  Warp wg = rank * NW + warp of the cluster owns rows
// r = wg + R i (R = G * NW warps, i < IR); lane l owns columns c = l + 32 j
// (j < JC).  Every element lives in exactly one register of one thread, so a
// column step costs no shared-memory traffic for the matrix itself: only the
// Householder vectors travel, through distributed shared memory (every CTA
// keeps a full copy of x and p, written by their owners with remote stores).
//
// Column step k (LAPACK sytd2 order, lower), fused as in the shared-memory
// kernel:
//   (A) column k is updated with reflector k-1 (v, w); its tail x gives
//       reflector k.  Owners store x and their partial |x|^2 into every CTA.
//       -- cluster barrier --
//   (B) every thread forms beta, tau, and the scale of v = x / (alpha - beta)
//       from the posted partials (redundantly, no further exchange).
//   (C) the trailing block (rows, columns > k) is updated with reflector k-1
//       and multiplied by v_k in the same pass over the registers; row sums
//       (butterfly across lanes) give p = tau A v, stored into every CTA with
//       the partial dots p.v.
//       -- cluster barrier --
//   (D) kw = (tau/2)(p.v); w_k = p - kw v_k is applied where w is read.
// Outputs match the shared-memory kernel: d, e, tau, and reflector k in row k
// of the global matrix (columns k+2..n-1; v[k+1] = 1 implicit).
//
// Reference behaviour: the reduction LAPACK's dsytrd performs inside dsyevd
// (model/gfn2/eigensolver.cpp:1221-1254 of the reference calls it on the
// Cholesky-reduced matrix); the eigenpairs are basis independent.
#include <cooperative_groups.h>

#include "kernels.cuh"

#include <algorithm>

namespace xtb {
namespace cg = cooperative_groups;

namespace {

template <int G, int NT, int NMAX>
__global__ void __launch_bounds__(NT) k_tridiag_reg(EigArgs g, const int32_t* list) {
  constexpr int NW = NT / 32;
  constexpr int R = G * NW;
  constexpr int IR = (NMAX + R - 1) / R;
  constexpr int JC = NMAX / 32;
  static_assert(IR * G <= 32, "one lane per (row slot, CTA) pair");
  static_assert((IR & (IR - 1)) == 0, "row slots per warp must be a power of two");
  static_assert(R % 32 == 0 || R < 32, "reduction layout");
  cg::cluster_group cluster = cg::this_cluster();
  const int crank = (int)cluster.block_rank();
  const int s = list[blockIdx.x / G];
  const int n = g.nao[s];
  double* ga = g.A + g.mat_off[s];
  double* d = g.d + g.ao_off[s];
  double* e = g.e + g.ao_off[s];
  double* tau = g.tau + g.ao_off[s];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wg = crank * NW + warp;

  __shared__ double X[2][NMAX];     // x of reflector k (rows > k), by step parity
  __shared__ double P[2][NMAX];     // tau A v of reflector k (rows > k)
  __shared__ double NRM[2][R];      // per-warp partial |x|^2
  __shared__ double PV[2][R];       // per-warp partial p.v

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
    (&X[0][0])[k] = 0.0;
    (&P[0][0])[k] = 0.0;
  }
  for (int k = tid; k < 2 * R; k += NT) {
    (&NRM[0][0])[k] = 0.0;
    (&PV[0][0])[k] = 0.0;
  }
  // stores into the exchange arrays of CTA q of the cluster
  auto remote = [&](double* local, int q) { return cluster.map_shared_rank(local, q); };
  cluster.sync();

  // scalars of the previous reflector: v = sc x (v[k] = 1), w = p - kw v
  double sc_p = 0.0, kw_p = 0.0;
  for (int k = 0; k + 1 < n; ++k) {
    const int kb = k & 1, pb = kb ^ 1;
    const bool prev = k >= 1;
    const bool next = k + 2 < n;    // reflector k exists
    const double* Xp = X[pb];
    const double* Pp = P[pb];
    // v and w of reflector k-1 at row r >= k
    auto vprev = [&](int r) { return r == k ? 1.0 : sc_p * Xp[r]; };
    auto wprev = [&](int r) { return Pp[r] - kw_p * vprev(r); };
    // ---- (A) column k ----
    const int l0 = k & 31, j0 = k >> 5;
    const double wk = prev ? wprev(k) : 0.0;
    double vals[IR];
    double nrm = 0.0;
#pragma unroll
    for (int i = 0; i < IR; ++i) {
      const int r = wg + R * i;
      double mine = 0.0;
#pragma unroll
      for (int j = 0; j < JC; ++j)
        if (j == j0) mine = a[i][j];
      double v = __shfl_sync(0xffffffffu, mine, l0);
      if (prev && r >= k && r < n) v -= vprev(r) * wk + wprev(r);
      if (lane == l0) {
#pragma unroll
        for (int j = 0; j < JC; ++j)
          if (j == j0) a[i][j] = v;
      }
      vals[i] = v;
      if (r >= k + 2 && r < n) nrm = fma(v, v, nrm);
      if (r == k && lane == 0) d[k] = v;
    }
    // x (rows > k) and the partial norm into every CTA
#pragma unroll
    for (int i = 0; i < IR; ++i) {
      const int r = wg + R * i;
      if (r >= k + 1 && r < n && lane >= i * G && lane < (i + 1) * G)
        *remote(&X[kb][r], lane - i * G) = vals[i];
    }
    if (lane < G) *remote(&NRM[kb][wg], lane) = nrm;
    cluster.sync();
    // ---- (B) reflector k ----
    double xn2 = 0.0;
#pragma unroll
    for (int q = lane; q < R; q += 32) xn2 += NRM[kb][q];
    xn2 = warp_sum(xn2);
    const double alpha = X[kb][k + 1];
    double ti = 0.0, sc = 0.0, beta = alpha;
    if (next && xn2 > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
      ti = (beta - alpha) / beta;
      sc = 1.0 / (alpha - beta);
    }
    if (crank == 0 && tid == 0) {
      e[k] = beta;   // for k = n-2 this is the updated (n-1, n-2) element
      tau[k] = ti;
    }
    if (next) {
#pragma unroll
      for (int i = 0; i < IR; ++i) {
        const int r = wg + R * i;
        if (lane == 0 && r >= k + 2 && r < n) ga[(int64_t)k * n + r] = sc * vals[i];
      }
    }
    auto vcur = [&](int r) { return r == k + 1 ? 1.0 : sc * X[kb][r]; };
    // ---- (C) trailing block: update with reflector k-1, multiply by v_k ----
    double vr[IR], wr[IR], acc[IR];
#pragma unroll
    for (int i = 0; i < IR; ++i) {
      const int r = wg + R * i;
      const bool act = prev && r >= k + 1 && r < n;
      vr[i] = act ? vprev(r) : 0.0;
      wr[i] = act ? wprev(r) : 0.0;
      acc[i] = 0.0;
    }
    const int jlo = (k + 1) >> 5;
#pragma unroll
    for (int j = 0; j < JC; ++j) {
      if (j < jlo) continue;   // uniform: every column of this slot is done
      const int c = lane + 32 * j;
      const bool cact = c >= k + 1 && c < n;
      const double vc = (prev && cact) ? vprev(c) : 0.0;
      const double wc = (prev && cact) ? wprev(c) : 0.0;
      const double nc = (next && cact) ? vcur(c) : 0.0;
#pragma unroll
      for (int i = 0; i < IR; ++i) {
        const int r = wg + R * i;
        if (r < k + 1) continue;   // uniform over the warp
        a[i][j] -= vr[i] * wc + wr[i] * vc;
        acc[i] = fma(a[i][j], nc, acc[i]);
      }
    }
    if (!next) {
      // last step: the (n-1, n-1) element is final
#pragma unroll
      for (int i = 0; i < IR; ++i) {
        const int r = wg + R * i;
#pragma unroll
        for (int j = 0; j < JC; ++j)
          if (r == n - 1 && lane + 32 * j == n - 1) {
            d[n - 1] = a[i][j];
            e[n - 1] = 0.0;
            tau[n - 1] = 0.0;
          }
      }
      break;
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
    // lane l now holds row slot l % IR
    const int slot = lane & (IR - 1);
    const int rs = wg + R * slot;
    const double pr = ti * acc[0];
    const bool ract = rs >= k + 1 && rs < n;
    if (ract && lane < IR * G) *remote(&P[kb][rs], lane / IR) = pr;
    double pv = (lane < IR && ract) ? pr * vcur(rs) : 0.0;
    pv = warp_sum(pv);
    if (lane < G) *remote(&PV[kb][wg], lane) = pv;
    cluster.sync();
    // ---- (D) ----
    double tpv = 0.0;
#pragma unroll
    for (int q = lane; q < R; q += 32) tpv += PV[kb][q];
    tpv = warp_sum(tpv);
    kw_p = 0.5 * ti * tpv;
    sc_p = sc;
  }
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
