// Extended-Hueckel H0 factors shared by the integral kernel and the force
// kernel: shell levels shifted by the coordination number, the shell-pair
// scaling of each model and the distance polynomial.
//
// GFN2 (model/gfn2/h0.cpp:248-466): zeta, electronegativity and
// angular-momentum scaling.  GFN1 (model/gfn1/h0.cpp:380-420,690-740):
// valence pairs take the angular-momentum scale k_ll' times the element-pair
// scale kpair and the electronegativity factor; a valence with a
// polarisation shell the mean of k_ll and kpol; two polarisation shells kpol.
#pragma once

#include "common.cuh"

namespace xtb {

__device__ __forceinline__ double h0_shell_level(const DevTopo& t, int sh, const double* cn) {
  return t.sh_level[sh] - t.sh_kcn[sh] * cn[t.sh_atom[sh]];
}

__device__ __forceinline__ double h0_pair_scale(const DevTopo& t, int i, int j) {
  const int A = t.sh_atom[i], B = t.sh_atom[j];
  const int li = t.sh_l[i], lj = t.sh_l[j];
  if (t.m.gfn1) {
    const bool vi = t.sh_val[i] != 0, vj = t.sh_val[j] != 0;
    if (vi && vj) {
      const double den = t.at_en[A] - t.at_en[B];
      return t.m.shell_pair_scale[li * 3 + lj] * t.kpair[(t.Z[A] - 1) * 86 + (t.Z[B] - 1)] *
             (1.0 + t.m.enscale * den * den);
    }
    if (vi) return 0.5 * (t.m.shell_pair_scale[li * 3 + li] + t.m.kpol);
    if (vj) return 0.5 * (t.m.shell_pair_scale[lj * 3 + lj] + t.m.kpol);
    return t.m.kpol;
  }
  const double zi = t.sh_zeta[i], zj = t.sh_zeta[j];
  const double zs = pow(2.0 * sqrt(zi * zj) / (zi + zj), t.m.wexp);
  const double den = t.at_en[A] - t.at_en[B];
  const double es = 1.0 + t.m.enscale * den * den;
  return zs * es * t.m.shell_pair_scale[li * 3 + lj] * t.m.pair_scale_default;
}

// Distance polynomial of a shell pair on different atoms and its radial derivative.
__device__ __forceinline__ void h0_polynomial(const DevTopo& t, int i, int j, double r, double& poly,
                                              double& dpoly) {
  const double rr = sqrt(r / (t.at_rad[t.sh_atom[i]] + t.at_rad[t.sh_atom[j]]));
  const double p1 = 1.0 + t.sh_shpoly[i] * rr;
  const double p2 = 1.0 + t.sh_shpoly[j] * rr;
  poly = p1 * p2;
  dpoly = (t.sh_shpoly[i] * p2 + t.sh_shpoly[j] * p1) * rr / (2.0 * r);
}

__device__ __forceinline__ double h0_factor(const DevTopo& t, int i, int j, const double* cn,
                                            double r, bool same_atom) {
  const double avg = 0.5 * (h0_shell_level(t, i, cn) + h0_shell_level(t, j, cn));
  if (same_atom) return avg;
  double poly, dpoly;
  h0_polynomial(t, i, j, r, poly, dpoly);
  return avg * h0_pair_scale(t, i, j) * poly;
}

}  // namespace xtb
