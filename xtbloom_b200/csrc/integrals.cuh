// Contracted-Gaussian overlap and multipole integrals for one spherical element
// pair, with optional first derivatives.
//
// Algorithm (restated from common/integrals.cpp:356-652 of the reference):
// each primitive pair contributes exp(-mu r^2) (pi/p)^(3/2) c_a c_b times a
// product of three 1-D Obara-Saika overlap factors T[a][b] (ket power a about
// the ket centre, bra power b about the bra centre).  Multipole moments of the
// operator (r - R_ket) raise the ket power; derivatives with respect to the ket
// centre are 2 alpha_ket T[a+1][b] - a T[a-1][b].  Cartesian blocks are mapped
// to tblite's real spherical harmonics and the second moments are projected to
// the traceless form Q = 3/2 rr - r^2/2.
//
// The kernels evaluate one spherical element pair at a time so that the ten
// values (S, three dipole, six quadrupole components) and their thirty
// derivatives stay in registers.
#pragma once

#include "common.cuh"

namespace xtb {

__device__ __forceinline__ void cart_exponents(int l, int i, int e[3]) {
  // tblite Cartesian order: s; x y z; xx xy xz yy yz zz
  int x = 0, y = 0, z = 0;
  if (l == 1) {
    x = (i == 0); y = (i == 1); z = (i == 2);
  } else if (l == 2) {
    switch (i) {
      case 0: x = 2; break;
      case 1: x = 1; y = 1; break;
      case 2: x = 1; z = 1; break;
      case 3: y = 2; break;
      case 4: y = 1; z = 1; break;
      default: z = 2; break;
    }
  }
  e[0] = x; e[1] = y; e[2] = z;
}

// Spherical function m of shell l as a sparse sum of Cartesian functions.
struct SphTerms {
  int n;
  int c[3];
  double w[3];
};

__device__ __forceinline__ SphTerms sph_terms(int l, int m) {
  constexpr double s3 = 1.7320508075688772935274463415058723;
  SphTerms t{};
  if (l == 0) {
    t.n = 1; t.c[0] = 0; t.w[0] = 1.0;
  } else if (l == 1) {
    // real spherical order [y, z, x]
    t.n = 1; t.c[0] = (m == 0) ? 1 : (m == 1 ? 2 : 0); t.w[0] = 1.0;
  } else {
    switch (m) {
      case 0: t.n = 1; t.c[0] = 1; t.w[0] = s3; break;                       // xy
      case 1: t.n = 1; t.c[0] = 4; t.w[0] = s3; break;                       // yz
      case 2: t.n = 3; t.c[0] = 0; t.w[0] = -0.5; t.c[1] = 3; t.w[1] = -0.5;
              t.c[2] = 5; t.w[2] = 1.0; break;                               // 2zz-xx-yy
      case 3: t.n = 1; t.c[0] = 2; t.w[0] = s3; break;                       // xz
      default: t.n = 2; t.c[0] = 0; t.w[0] = 0.5 * s3; t.c[1] = 3; t.w[1] = -0.5 * s3; break;
    }
  }
  return t;
}

// 1-D factors for one axis: O[e] = T[ek+e][eb] (e = 0..2) and, with GRAD,
// G[e] = 2 a_k T[ek+e+1][eb] - (ek+e) T[ek+e-1][eb].
template <bool GRAD>
__device__ __forceinline__ void axis_factors(double pa, double pb, double inv2p, double ak, int ek,
                                             int eb, double O[3], double G[3]) {
  double T[6][3];
#pragma unroll
  for (int a = 0; a < 6; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) T[a][b] = 0.0;
  T[0][0] = 1.0;
#pragma unroll
  for (int a = 1; a < 6; ++a) {
    T[a][0] = pa * T[a - 1][0];
    if (a > 1) T[a][0] += (a - 1) * inv2p * T[a - 2][0];
  }
#pragma unroll
  for (int b = 1; b < 3; ++b) {
    T[0][b] = pb * T[0][b - 1];
    if (b > 1) T[0][b] += (b - 1) * inv2p * T[0][b - 2];
#pragma unroll
    for (int a = 1; a < 6; ++a) {
      T[a][b] = pa * T[a - 1][b] + b * inv2p * T[a - 1][b - 1];
      if (a > 1) T[a][b] += (a - 1) * inv2p * T[a - 2][b];
    }
  }
  // select the needed column entries without dynamic register indexing
  double col[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) col[a] = (eb == 0) ? T[a][0] : ((eb == 1) ? T[a][1] : T[a][2]);
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    double o = 0.0, up = 0.0, dn = 0.0;
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      o = (a == ek + e) ? col[a] : o;
      up = (a == ek + e + 1) ? col[a] : up;
      dn = (a == ek + e - 1) ? col[a] : dn;
    }
    O[e] = o;
    if (GRAD) G[e] = 2.0 * ak * up - (ek + e) * dn;
  }
}

// Multipole powers along x,y,z for the nine moment components
// [x, y, z, xx, xy, yy, xz, yz, zz].
__device__ __forceinline__ void moment_powers(int m, int p[3]) {
  const int px[9] = {1, 0, 0, 2, 1, 0, 1, 0, 0};
  const int py[9] = {0, 1, 0, 0, 1, 2, 0, 1, 0};
  const int pz[9] = {0, 0, 1, 0, 0, 0, 1, 1, 2};
  p[0] = px[m]; p[1] = py[m]; p[2] = pz[m];
}

// Accumulate w * (S, 9 raw moments) [and derivatives w.r.t. the ket centre]
// of one Cartesian pair.  v = R_ket - R_bra.
template <bool GRAD>
__device__ __forceinline__ void cart_pair_acc(const int eb[3], const int ek[3], const double* ab,
                                              const double* cb, int npb, const double* ak,
                                              const double* ck, int npk, const double v[3],
                                              double w, double out[10], double dout[3][10]) {
  const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
  for (int ik = 0; ik < npk; ++ik) {
    const double aK = ak[ik];
    for (int ib = 0; ib < npb; ++ib) {
      const double aB = ab[ib];
      const double inv = 1.0 / (aK + aB);
      const double est = aK * aB * r2 * inv;
      if (est > kIntegralCutoff) continue;
      const double pref = w * exp(-est) * kSqrtPi3 * inv * sqrt(inv) * ck[ik] * cb[ib];
      const double inv2p = 0.5 * inv;
      double O[3][3], G[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        axis_factors<GRAD>(-v[c] * aB * inv, v[c] * aK * inv, inv2p, aK, ek[c], eb[c], O[c], G[c]);
      out[0] += pref * O[0][0] * O[1][0] * O[2][0];
      if (GRAD) {
        dout[0][0] += pref * G[0][0] * O[1][0] * O[2][0];
        dout[1][0] += pref * O[0][0] * G[1][0] * O[2][0];
        dout[2][0] += pref * O[0][0] * O[1][0] * G[2][0];
      }
#pragma unroll
      for (int m = 0; m < 9; ++m) {
        int p[3];
        moment_powers(m, p);
        const double ox = O[0][p[0]], oy = O[1][p[1]], oz = O[2][p[2]];
        out[1 + m] += pref * ox * oy * oz;
        if (GRAD) {
          dout[0][1 + m] += pref * G[0][p[0]] * oy * oz;
          dout[1][1 + m] += pref * ox * G[1][p[1]] * oz;
          dout[2][1 + m] += pref * ox * oy * G[2][p[2]];
        }
      }
    }
  }
}

// Primitive-pair factors of one shell pair at separation v (independent of
// the Cartesian components): 1/(a_k + a_b), the screening exponent and, for
// the pairs that pass the screen, exp(-est) and sqrt(1/(a_k + a_b)).  Index
// ik * npb + ib.  cart_pair_acc_pp reads them instead of recomputing them
// for every component pair; the values and the order of every product are
// those of cart_pair_acc.
constexpr int kPrimPairs = 36;   // shells with at most 6 primitives
struct PrimPairs {
  double inv[kPrimPairs], est[kPrimPairs], e[kPrimPairs], sinv[kPrimPairs];
};
__device__ __forceinline__ void prim_pairs(const double* ab, int npb, const double* ak, int npk,
                                           const double v[3], PrimPairs& pp) {
  // the contraction cart_pair_acc's r^2 compiles to, written out
  const double r2 = fma(v[2], v[2], fma(v[0], v[0], v[1] * v[1]));
  for (int ik = 0; ik < npk; ++ik) {
    const double aK = ak[ik];
    for (int ib = 0; ib < npb; ++ib) {
      const double aB = ab[ib];
      const int q = ik * npb + ib;
      const double inv = 1.0 / (aK + aB);
      const double est = aK * aB * r2 * inv;
      pp.inv[q] = inv;
      pp.est[q] = est;
      if (est > kIntegralCutoff) continue;
      pp.e[q] = exp(-est);
      pp.sinv[q] = sqrt(inv);
    }
  }
}

template <bool GRAD>
__device__ __forceinline__ void cart_pair_acc_pp(const int eb[3], const int ek[3], const double* ab,
                                                 const double* cb, int npb, const double* ak,
                                                 const double* ck, int npk, const double v[3],
                                                 double w, const PrimPairs& pp, double out[10],
                                                 double dout[3][10]) {
  for (int ik = 0; ik < npk; ++ik) {
    const double aK = ak[ik];
    for (int ib = 0; ib < npb; ++ib) {
      const double aB = ab[ib];
      const int q = ik * npb + ib;
      const double inv = pp.inv[q];
      if (pp.est[q] > kIntegralCutoff) continue;
      const double pref = w * pp.e[q] * kSqrtPi3 * inv * pp.sinv[q] * ck[ik] * cb[ib];
      const double inv2p = 0.5 * inv;
      double O[3][3], G[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        axis_factors<GRAD>(-v[c] * aB * inv, v[c] * aK * inv, inv2p, aK, ek[c], eb[c], O[c], G[c]);
      out[0] += pref * O[0][0] * O[1][0] * O[2][0];
      if (GRAD) {
        dout[0][0] += pref * G[0][0] * O[1][0] * O[2][0];
        dout[1][0] += pref * O[0][0] * G[1][0] * O[2][0];
        dout[2][0] += pref * O[0][0] * O[1][0] * G[2][0];
      }
#pragma unroll
      for (int m = 0; m < 9; ++m) {
        int p[3];
        moment_powers(m, p);
        const double ox = O[0][p[0]], oy = O[1][p[1]], oz = O[2][p[2]];
        out[1 + m] += pref * ox * oy * oz;
        if (GRAD) {
          dout[0][1 + m] += pref * G[0][p[0]] * oy * oz;
          dout[1][1 + m] += pref * ox * G[1][p[1]] * oz;
          dout[2][1 + m] += pref * ox * oy * G[2][p[2]];
        }
      }
    }
  }
}

__device__ __forceinline__ void make_traceless(double* m /* 6 raw: xx xy yy xz yz zz */) {
  const double tr = 0.5 * (m[0] + m[2] + m[5]);
  m[0] = 1.5 * m[0] - tr;
  m[1] *= 1.5;
  m[2] = 1.5 * m[2] - tr;
  m[3] *= 1.5;
  m[4] *= 1.5;
  m[5] = 1.5 * m[5] - tr;
}

// One spherical element pair (bra function mb of shell lb, ket function mk of
// shell lk).  out = [S, Dx, Dy, Dz, Qxx, Qxy, Qyy, Qxz, Qyz, Qzz] with the
// operator origin at the ket atom; dout[c][.] = derivatives w.r.t. R_ket[c].
template <bool GRAD>
__device__ __forceinline__ void sph_pair(int lb, int mb, int lk, int mk, const double* ab,
                                         const double* cb, int npb, const double* ak,
                                         const double* ck, int npk, const double v[3],
                                         double out[10], double dout[3][10]) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    out[i] = 0.0;
    if (GRAD) { dout[0][i] = 0.0; dout[1][i] = 0.0; dout[2][i] = 0.0; }
  }
  const SphTerms tb = sph_terms(lb, mb);
  const SphTerms tk = sph_terms(lk, mk);
  for (int i = 0; i < tb.n; ++i) {
    int eb[3];
    cart_exponents(lb, tb.c[i], eb);
    for (int j = 0; j < tk.n; ++j) {
      int ek[3];
      cart_exponents(lk, tk.c[j], ek);
      cart_pair_acc<GRAD>(eb, ek, ab, cb, npb, ak, ck, npk, v, tb.w[i] * tk.w[j], out, dout);
    }
  }
  make_traceless(out + 4);
  if (GRAD) {
    make_traceless(dout[0] + 4);
    make_traceless(dout[1] + 4);
    make_traceless(dout[2] + 4);
  }
}

// sph_pair with the primitive-pair factors of prim_pairs.
template <bool GRAD>
__device__ __forceinline__ void sph_pair_pp(int lb, int mb, int lk, int mk, const double* ab,
                                            const double* cb, int npb, const double* ak,
                                            const double* ck, int npk, const double v[3],
                                            const PrimPairs& pp, double out[10],
                                            double dout[3][10]) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    out[i] = 0.0;
    if (GRAD) { dout[0][i] = 0.0; dout[1][i] = 0.0; dout[2][i] = 0.0; }
  }
  const SphTerms tb = sph_terms(lb, mb);
  const SphTerms tk = sph_terms(lk, mk);
  for (int i = 0; i < tb.n; ++i) {
    int eb[3];
    cart_exponents(lb, tb.c[i], eb);
    for (int j = 0; j < tk.n; ++j) {
      int ek[3];
      cart_exponents(lk, tk.c[j], ek);
      cart_pair_acc_pp<GRAD>(eb, ek, ab, cb, npb, ak, ck, npk, v, tb.w[i] * tk.w[j], pp, out, dout);
    }
  }
  make_traceless(out + 4);
  if (GRAD) {
    make_traceless(dout[0] + 4);
    make_traceless(dout[1] + 4);
    make_traceless(dout[2] + 4);
  }
}

// Reverse element (ket row, bra column): the operator origin moves to the bra
// atom.  D' = D + v S;  Q' = Q + 3/2 shift - tr(shift)/2 (common/integrals.cpp:824-850).
__device__ __forceinline__ void shift_to_bra(const double v[3], const double in[10], double o[10]) {
  const double S = in[0];
  const double dx = in[1], dy = in[2], dz = in[3];
  o[0] = S;
  o[1] = dx + v[0] * S;
  o[2] = dy + v[1] * S;
  o[3] = dz + v[2] * S;
  double sh[6];
  sh[0] = 2.0 * v[0] * dx + v[0] * v[0] * S;
  sh[1] = v[0] * dy + v[1] * dx + v[0] * v[1] * S;
  sh[2] = 2.0 * v[1] * dy + v[1] * v[1] * S;
  sh[3] = v[0] * dz + v[2] * dx + v[0] * v[2] * S;
  sh[4] = v[1] * dz + v[2] * dy + v[1] * v[2] * S;
  sh[5] = 2.0 * v[2] * dz + v[2] * v[2] * S;
  const double tr = 0.5 * (sh[0] + sh[2] + sh[5]);
  o[4] = in[4] + 1.5 * sh[0] - tr;
  o[5] = in[5] + 1.5 * sh[1];
  o[6] = in[6] + 1.5 * sh[2] - tr;
  o[7] = in[7] + 1.5 * sh[3];
  o[8] = in[8] + 1.5 * sh[4];
  o[9] = in[9] + 1.5 * sh[5] - tr;
}

}  // namespace xtb
