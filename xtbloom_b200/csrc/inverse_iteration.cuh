// Inverse iteration for eigenvectors of a symmetric tridiagonal matrix: the
// block-wide routine shared by the batched SCC kernel and the single-matrix
// static-scratch entry point.
#pragma once

#include <cfloat>
#include <cstdint>

namespace xtb {

// ---------------------------------------------------------------------------
// Inverse iteration for eigenvectors 0..nvec-1 of the tridiagonal matrix.
// One thread per eigenvalue cluster; output ZT[j][0..n) (eigenvector-major).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double hash_unit(uint32_t a, uint32_t b) {
  uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u + (a << 6) + (a >> 2));
  h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
  return (double)h * (2.0 / 4294967296.0) - 1.0;
}

// ortol_rel: eigenvalues closer than ortol_rel * ||T||_1 form a cluster whose
// vectors are re-orthogonalised.  Outside clusters inverse-iteration vectors
// are orthogonal to ~eps ||T|| / gap, i.e. better than 1e-9 for the
// thresholds used (2e-7 for Hamiltonians, 2e-6 for overlap matrices).
//
// Block-wide: eigenvectors of the n x n tridiagonal (d, e) for the ascending
// eigenvalues ev[0..m), written as rows Z[j*n .. j*n+n).  Thread t of the
// block leads the clusters starting at lead0 + t, lead0 + t + lead_step, ...
// scratch holds 5 n LD doubles: per-thread work vectors interleaved across
// the CTA's LD thread slots (element k of array a for thread t at
// ((a*n + k) * LD + t)) so that every sequential sweep over k is a coalesced
// access.  Every scratch element is written before it is read.  seed varies
// the start vectors.
// The sweeps load the inputs of kAhead steps before running them, so that
// several scratch loads of a thread are in flight at once (the sweeps are
// bound by their latency).
constexpr int kAhead = 8;
template <int LD>
__device__ __forceinline__ void inverse_iteration_block(const double* d, const double* e,
                                                        const double* ev, int n, int m, double* Z,
                                                        double* scratch, double ortol_rel,
                                                        uint32_t seed, int lead0, int lead_step) {
  double* scr = scratch + threadIdx.x;
  constexpr int64_t ld = LD;
  auto U1 = [&](int k) -> double& { return scr[((int64_t)0 * n + k) * ld]; };
  auto U2 = [&](int k) -> double& { return scr[((int64_t)1 * n + k) * ld]; };
  auto U3 = [&](int k) -> double& { return scr[((int64_t)2 * n + k) * ld]; };
  auto LM = [&](int k) -> double& { return scr[((int64_t)3 * n + k) * ld]; };
  auto Y = [&](int k) -> double& { return scr[((int64_t)4 * n + k) * ld]; };
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
  const double ortol = ortol_rel * onenrm;
  const double tiny = DBL_EPSILON * onenrm;
  for (int lead = lead0 + threadIdx.x; lead < m; lead += lead_step) {
    if (lead > 0 && ev[lead] - ev[lead - 1] <= ortol) continue;   // not a cluster leader
    double xprev = -DBL_MAX;
    for (int j = lead; j < m; ++j) {
      if (j > lead && ev[j] - ev[j - 1] > ortol) break;
      double x = ev[j];
      if (j > lead && x - xprev < 10.0 * DBL_EPSILON * fabs(x)) x = xprev + 10.0 * DBL_EPSILON * fabs(x);
      xprev = x;
      // LU with partial pivoting of T - xI; U1 holds reciprocal pivots and the
      // sign of LM encodes the row interchange (pivoted rows store -l - 4; both |l| <= 1).
      // One reciprocal per step on the dependency chain: the multiplier is
      // the off-pivot element times the reciprocal pivot (within an ulp of
      // the quotient), and the reciprocal is reused as U1 unless the pivot
      // is replaced by +-tiny.
      // The first forward elimination runs inside the factorisation: the
      // start vector's elements are formed where the elimination reads them
      // and y_k is final once step k has chosen its pivot (the same
      // operations, in the same order, as a separate sweep).
      const uint32_t hseed = (uint32_t)j * 7919u + seed;
      double diag = d[0] - x, sup = n > 1 ? e[0] : 0.0;
      double yk = hash_unit(0u, hseed);
      auto lustep = [&](double ck, double nd, double ns, int k) {
        const bool keep = fabs(diag) >= fabs(ck);
        const double u1 = keep ? diag : ck;
        const double r = __drcp_rn(u1);
        double l;
        double yn = hash_unit((uint32_t)(k + 1), hseed);
        if (keep) {
          l = diag != 0.0 ? ck * r : 0.0;
          U2(k) = sup; U3(k) = 0.0; LM(k) = l;
          diag = nd - l * sup;
          sup = ns;
          yn -= l * yk;
        } else {
          l = diag * r;
          const double lenc = -l - 4.0;   // the stored encoding; the sweeps decode -lenc - 4
          U2(k) = nd; U3(k) = ns; LM(k) = lenc;
          diag = sup - l * nd;
          sup = -l * ns;
          const double tmp = yk;
          yk = yn;
          yn = tmp - (-lenc - 4.0) * yk;
        }
        U1(k) = fabs(u1) < tiny ? __drcp_rn(u1 < 0.0 ? -tiny : tiny) : r;
        Y(k) = yk;
        yk = yn;
      };
      {
        // the matrix entries of kAhead steps are loaded before the steps run
        int k = 0;
        for (; k + kAhead <= n - 1; k += kAhead) {
          double cv[kAhead], dv[kAhead], sv[kAhead];
#pragma unroll
          for (int u = 0; u < kAhead; ++u) {
            cv[u] = e[k + u];
            dv[u] = d[k + u + 1] - x;
            sv[u] = (k + u + 1 < n - 1) ? e[k + u + 1] : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kAhead; ++u) lustep(cv[u], dv[u], sv[u], k + u);
        }
        for (; k < n - 1; ++k) lustep(e[k], d[k + 1] - x, (k + 1 < n - 1) ? e[k + 1] : 0.0, k);
      }
      Y(n - 1) = yk;
      {
        double u1 = diag;
        if (fabs(u1) < tiny) u1 = u1 < 0.0 ? -tiny : tiny;
        U1(n - 1) = 1.0 / u1;
      }
      const int iters = (j > lead) ? 3 : 2;
      // scale: the normalisation of the previous sweep, applied where the
      // next one reads y (the product is the value the scaled vector held)
      double scale = 1.0;
      for (int it = 0; it < iters; ++it) {
        if (it > 0) {
          // forward elimination with the recorded interchanges; the inputs of
          // kAhead steps are loaded before the steps run (the sweep writes only
          // elements it has passed, so the loads see the values they would)
          double yk2 = Y(0) * scale;
          auto fstep = [&](double ynext, double lk, int k) {
            double yn = ynext * scale;
            if (lk < -2.0) {
              const double tmp = yk2;
              yk2 = yn;
              yn = tmp - (-lk - 4.0) * yk2;
            } else {
              yn -= lk * yk2;
            }
            Y(k) = yk2;
            yk2 = yn;
          };
          int k = 0;
          for (; k + kAhead <= n - 1; k += kAhead) {
            double yv[kAhead], lv[kAhead];
#pragma unroll
            for (int u = 0; u < kAhead; ++u) {
              yv[u] = Y(k + 1 + u);
              lv[u] = LM(k + u);
            }
#pragma unroll
            for (int u = 0; u < kAhead; ++u) fstep(yv[u], lv[u], k + u);
          }
          for (; k < n - 1; ++k) fstep(Y(k + 1), LM(k), k);
          Y(n - 1) = yk2;
        }
        // back substitution
        double y2 = 0.0, y1 = Y(n - 1) * U1(n - 1);
        Y(n - 1) = y1;
        if (n >= 2) {
          const double y0 = (Y(n - 2) - U2(n - 2) * y1) * U1(n - 2);
          Y(n - 2) = y0;
          y2 = y1;
          y1 = y0;
        }
        double nrm = y1 * y1 + (n >= 2 ? y2 * y2 : 0.0);
        auto bstep = [&](double yv, double u1, double u2, double u3, int k) {
          const double y0 = (yv - u2 * y1 - u3 * y2) * u1;
          Y(k) = y0;
          nrm += y0 * y0;
          y2 = y1;
          y1 = y0;
        };
        {
          // back substitution, kAhead steps' inputs loaded ahead as above
          int k = n - 3;
          for (; k >= kAhead - 1; k -= kAhead) {
            double yv[kAhead], a1[kAhead], a2[kAhead], a3[kAhead];
#pragma unroll
            for (int u = 0; u < kAhead; ++u) {
              yv[u] = Y(k - u);
              a1[u] = U1(k - u);
              a2[u] = U2(k - u);
              a3[u] = U3(k - u);
            }
#pragma unroll
            for (int u = 0; u < kAhead; ++u) bstep(yv[u], a1[u], a2[u], a3[u], k - u);
          }
          for (; k >= 0; --k) bstep(Y(k), U1(k), U2(k), U3(k), k);
        }
        // orthogonalise against the earlier members of the cluster
        if (j > lead) {
          for (int q = lead; q < j; ++q) {
            const double* zq = Z + (int64_t)q * n;
            double dot = 0.0;
            for (int k = 0; k < n; ++k) dot += Y(k) * zq[k];
            // kAhead elements loaded before they are stored (the compiler
            // cannot tell the scratch from Z, so it would not reorder them)
            int k = 0;
            for (; k + kAhead <= n; k += kAhead) {
              double yv[kAhead], zv[kAhead];
#pragma unroll
              for (int u = 0; u < kAhead; ++u) {
                yv[u] = Y(k + u);
                zv[u] = zq[k + u];
              }
#pragma unroll
              for (int u = 0; u < kAhead; ++u) Y(k + u) = yv[u] - dot * zv[u];
            }
            for (; k < n; ++k) Y(k) -= dot * zq[k];
          }
          nrm = 0.0;
          for (int k = 0; k < n; ++k) nrm += Y(k) * Y(k);
        }
        scale = 1.0 / sqrt(nrm);
      }
      // sign convention: largest component positive; publish row j of Z
      // (normalised as it is read)
      int kmax = 0;
      double amax = 0.0, vmax = 0.0;
      for (int k = 0; k < n; ++k) {
        const double v = Y(k) * scale;
        if (fabs(v) > amax) { amax = fabs(v); kmax = k; vmax = v; }
      }
      (void)kmax;
      const double sgn = vmax < 0.0 ? -1.0 : 1.0;
      double* y = Z + (int64_t)j * n;
      int k = 0;
      for (; k + kAhead <= n; k += kAhead) {   // loads ahead of the stores, as above
        double yv[kAhead];
#pragma unroll
        for (int u = 0; u < kAhead; ++u) yv[u] = Y(k + u);
#pragma unroll
        for (int u = 0; u < kAhead; ++u) y[k + u] = sgn * (yv[u] * scale);
      }
      for (; k < n; ++k) y[k] = sgn * (Y(k) * scale);
    }
  }
}


}  // namespace xtb
