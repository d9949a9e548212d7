// Device helpers for the classical terms: D4 reference weights and pair
// damping (model/gfn2/d4.cpp:283-366, 640-700), AES2 damped pair kernels
// (model/gfn2/aes2.cpp:385-424).
#pragma once

#include <cfloat>

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

// ---------------------------------------------------------------------------
// GFN1: DFT-D3(BJ) two-body dispersion at the GFN1 coordination numbers
// (model/gfn1/d3.cpp:255-410).  Reference weights are Gaussians
// exp(-4 (CN_ref - CN)^2), normalised (with the reference's fallback to the
// largest reference CN when the sum underflows); C6 interpolates the
// reference C6 table; Becke-Johnson damping radius a1 sqrt(3 Q_A Q_B) + a2 and
// a smooth cutoff over the last 0.05 bohr before 50 bohr.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void d3_weights(const DevTopo& t, int z, double cn, double* w, double* dw) {
  const int off = t.d3_roff[z - 1], cnt = t.d3_rcnt[z - 1];
  double u[kD3MaxRefs];
  double norm = 0.0, dnorm = 0.0, maxcn = -DBL_MAX;
  for (int r = 0; r < cnt; ++r) {
    const double delta = t.d3_ref_cn[off + r] - cn;
    u[r] = exp(-4.0 * delta * delta);
    norm += u[r];
    dnorm += 8.0 * delta * u[r];
    maxcn = fmax(maxcn, t.d3_ref_cn[off + r]);
  }
  const double inv = 1.0 / norm;
  for (int r = 0; r < kD3MaxRefs; ++r) {
    if (r >= cnt) {
      w[r] = dw[r] = 0.0;
      continue;
    }
    const double rcn = t.d3_ref_cn[off + r];
    const double delta = rcn - cn;
    double weight = u[r] * inv;
    if (!isfinite(weight)) weight = rcn == maxcn ? 1.0 : 0.0;
    double d = 8.0 * delta * u[r] * inv - u[r] * dnorm * inv * inv;
    if (!isfinite(d)) d = 0.0;
    w[r] = weight;
    dw[r] = d;
  }
}

// C6 of an atom pair and its derivatives with respect to the two CNs.
__device__ __forceinline__ double d3_c6(const DevTopo& t, int za, int zb, const double* wa,
                                        const double* dwa, const double* wb, const double* dwb,
                                        double& dca, double& dcb) {
  const int oa = t.d3_roff[za - 1], ca = t.d3_rcnt[za - 1];
  const int ob = t.d3_roff[zb - 1], cb = t.d3_rcnt[zb - 1];
  double c6 = 0.0;
  dca = dcb = 0.0;
  for (int i = 0; i < ca; ++i) {
    const double* row = t.d3_c6 + (int64_t)(oa + i) * kD3Refs + ob;
    for (int j = 0; j < cb; ++j) {
      const double c = row[j];
      c6 += wa[i] * wb[j] * c;
      dca += dwa[i] * wb[j] * c;
      dcb += wa[i] * dwb[j] * c;
    }
  }
  return c6;
}

// Damped pair kernel: e = -(s6 t6 + s8 rrij t8) times the cutoff, and
// de/dr / r; the pair energy is c6 * e.
__device__ __forceinline__ void d3_pair(const DevTopo& t, int za, int zb, double r2, double& e,
                                        double& de_over_r) {
  const double rrij = 3.0 * t.d3_r4r2[za - 1] * t.d3_r4r2[zb - 1];
  const double r0 = t.m.d3_a1 * sqrt(rrij) + t.m.d3_a2;
  const double r02 = r0 * r0, r04 = r02 * r02;
  const double r06 = r04 * r02, r08 = r04 * r04;
  const double r4 = r2 * r2;
  const double t6 = 1.0 / (r4 * r2 + r06);
  const double t8 = 1.0 / (r4 * r4 + r08);
  const double phi = t.m.d3_s6 * t6 + t.m.d3_s8 * rrij * t8;
  const double dphi = t.m.d3_s6 * (-6.0 * r4 * t6 * t6) + t.m.d3_s8 * rrij * (-8.0 * r4 * r2 * t8 * t8);
  const double r = sqrt(r2);
  constexpr double kCut = 50.0, kWidth = 0.05;
  double cut = 1.0, dcut = 0.0;
  if (r >= kCut) {
    cut = 0.0;
  } else if (r > kCut - kWidth) {
    const double x = (kCut - r) / kWidth;
    cut = x * x * x * (10.0 + x * (-15.0 + 6.0 * x));
    dcut = -30.0 * x * x * (1.0 - x) * (1.0 - x) / kWidth;
  }
  e = -cut * phi;
  de_over_r = -(cut * dphi + dcut * phi / r);
}

}  // namespace xtb
