// Device helpers for the classical terms: D4 reference weights and pair
// damping (model/gfn2/d4.cpp:283-366, 640-700), AES2 damped pair kernels
// (model/gfn2/aes2.cpp:385-424).
#pragma once

#include "common.cuh"

namespace xtb {

// Charge-dependent D4 reference weights of one atom.  w[r] = cn-Gaussian
// weight * charge scaling; optional derivatives w.r.t. CN and charge.
__device__ __forceinline__ int d4_weights(const DevTopo& t, int z, double cn, double q, double* w,
                                          double* dwcn, double* dwq) {
  const int off = t.d4_roff[z - 1], cnt = t.d4_rcnt[z - 1];
  double num[kMaxD4Refs], dnum[kMaxD4Refs];
  double norm = 0.0, dnorm = 0.0, maxcn = -1e300;
  for (int r = 0; r < cnt; ++r) {
    const double rcn = t.ref_cn[off + r];
    maxcn = fmax(maxcn, rcn);
    double a = 0.0, da = 0.0;
    for (int g = 1; g <= t.ref_ng[off + r]; ++g) {
      const double f = g * 6.0;
      const double dl = cn - rcn;
      const double val = exp(-f * dl * dl);
      a += val;
      da += 2.0 * f * (rcn - cn) * val;
    }
    num[r] = a;
    dnum[r] = da;
    norm += a;
    dnorm += da;
  }
  const double inv = fabs(norm) > 1.4916681462400413e-154 ? 1.0 / norm : 0.0;
  const double zeff = t.d4_zeff[z - 1];
  const double qmod = q + zeff;
  const double cst = t.d4_eta[z - 1] * 2.0;
  for (int r = 0; r < cnt; ++r) {
    const double rcn = t.ref_cn[off + r];
    double cw = num[r] * inv;
    double dcw = inv * (dnum[r] - num[r] * dnorm * inv);
    if (inv == 0.0 || !isfinite(cw)) cw = fabs(maxcn - rcn) < 1e-12 ? 1.0 : 0.0;
    if (inv == 0.0 || !isfinite(dcw)) dcw = 0.0;
    const double qref = t.ref_q[off + r] + zeff;
    double scl, dscl;
    if (qmod < 0.0) {
      scl = exp(3.0);
      dscl = 0.0;
    } else {
      const double inner = exp(cst * (1.0 - qref / qmod));
      scl = exp(3.0 * (1.0 - inner));
      dscl = -3.0 * cst * inner * scl * qref / (qmod * qmod);
    }
    w[r] = cw * scl;
    if (dwcn) dwcn[r] = dcw * scl;
    if (dwq) dwq[r] = cw * dscl;
  }
  return cnt;
}

// Rational BJ damping of a pair at squared distance r2 (zero beyond 50 bohr);
// ddamp = (1/r) d damp / dr.
__device__ __forceinline__ void d4_pair_damping(const DevTopo& t, int zf, int zs, double r2,
                                                double& damp, double& ddamp) {
  damp = 0.0;
  ddamp = 0.0;
  if (r2 > 2500.0) return;
  const double rrij = 3.0 * t.d4_r4r2[zf - 1] * t.d4_r4r2[zs - 1];
  const double r0 = t.m.d4_a1 * sqrt(rrij) + t.m.d4_a2;
  const double r4 = r2 * r2, r6 = r4 * r2;
  const double r0_2 = r0 * r0, r0_4 = r0_2 * r0_2, r0_6 = r0_4 * r0_2;
  const double t6 = 1.0 / (r6 + r0_6);
  const double t8 = 1.0 / (r4 * r4 + r0_4 * r0_4);
  damp = t.m.d4_s6 * t6 + t.m.d4_s8 * rrij * t8;
  ddamp = t.m.d4_s6 * (-6.0 * r4 * t6 * t6) + t.m.d4_s8 * rrij * (-8.0 * r6 * t8 * t8);
}

__device__ __forceinline__ double d4_r0(const DevTopo& t, int zf, int zs) {
  const double rrij = 3.0 * t.d4_r4r2[zf - 1] * t.d4_r4r2[zs - 1];
  return t.m.d4_a1 * sqrt(rrij) + t.m.d4_a2;
}

// C6 = w_f^T C6ref w_s with optional first-order partners.
__device__ __forceinline__ double d4_c6(const DevTopo& t, int zf, int zs, const double* wf,
                                        const double* ws, const double* xf, const double* xs,
                                        double* cf, double* cs) {
  const int of = t.d4_roff[zf - 1], nf = t.d4_rcnt[zf - 1];
  const int os = t.d4_roff[zs - 1], ns = t.d4_rcnt[zs - 1];
  double c6 = 0.0, a = 0.0, b = 0.0;
  for (int i = 0; i < nf; ++i) {
    const double* row = t.ref_c6 + (int64_t)(of + i) * t.ref_count + os;
    double rw = 0.0, rx = 0.0;
    for (int j = 0; j < ns; ++j) {
      rw += row[j] * ws[j];
      if (xs) rx += row[j] * xs[j];
    }
    c6 += wf[i] * rw;
    if (xf) a += xf[i] * rw;
    if (xs) b += wf[i] * rx;
  }
  if (cf) *cf = a;
  if (cs) *cs = b;
  return c6;
}

// AES2 damped kernels f3/r^3 and f5/r^5 with the average multipole radius R.
__device__ __forceinline__ void aes2_kernels(double r, double R, double& k3, double& k5) {
  const double inv = 1.0 / r;
  const double inv2 = inv * inv, inv3 = inv2 * inv, inv5 = inv3 * inv2;
  const double sc = R * inv;
  const double sc2 = sc * sc, sc3 = sc2 * sc, sc4 = sc2 * sc2;
  k3 = inv3 / (1.0 + 6.0 * sc3);
  k5 = inv5 / (1.0 + 6.0 * sc4);
}

__device__ __forceinline__ void pair_from_index(int64_t p, int64_t& i, int64_t& j) {
  // p -> (i, j) with i > j >= 0, p = i (i - 1) / 2 + j
  i = (int64_t)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
  while (i * (i - 1) / 2 > p) --i;
  while ((i + 1) * i / 2 <= p) ++i;
  j = p - i * (i - 1) / 2;
}

}  // namespace xtb
