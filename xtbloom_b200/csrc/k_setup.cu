// Geometry-dependent setup kernels: coordination numbers (GFN2 double
// exponential and D4 covalent), AES2 multipole radii, overlap/multipole
// integrals fused with the H0 build, and the ES2 shell Coulomb matrix.
//
// Restated from the reference CPU model: model/gfn2/coordination.cpp:120-240,
// model/gfn2/d4.cpp:640-700 (D4 CN), model/gfn2/aes2.cpp:366-383 (radii),
// common/integrals.cpp:700-865 and model/gfn2/h0.cpp:248-466 (integrals, H0),
// model/gfn2/es2.cpp:211-300 (Coulomb kernel).
#include "kernels.cuh"
#include "h0.cuh"
#include "integrals.cuh"

namespace xtb {

// One CTA per system: both coordination numbers and AES2 radii.
__global__ void k_coordination(DevTopo t, const int32_t* list, double* cn, double* cn_d4,
                               double* mrad, double* dmrad) {
  extern __shared__ double sm[];
  const int s = list[blockIdx.x];
  const int64_t a0 = t.atom_off[s], na = t.atom_off[s + 1] - a0;
  double* scn = sm;
  double* scn4 = sm + na;
  // warp per atom, lanes over the partners, fixed-order reduction: the same
  // coordination numbers in every run
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int64_t i = warp; i < na; i += nw) {
    const int64_t gi = a0 + i;
    double c1 = 0.0, c4 = 0.0;
    for (int64_t j = lane; j < na; j += 32) {
      if (j == i) continue;
      const int64_t gj = a0 + j;
      const double dx = t.pos[3 * gi] - t.pos[3 * gj];
      const double dy = t.pos[3 * gi + 1] - t.pos[3 * gj + 1];
      const double dz = t.pos[3 * gi + 2] - t.pos[3 * gj + 2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double r = sqrt(r2);
      if (t.m.gfn1) {
        // GFN1: exponential counting function, steepness 16, cutoff 25 bohr
        // (model/gfn1/coordination.cpp:215-265); no D4 CN
        if (r2 <= 625.0 && r2 > 1e-12)
          c1 += logistic(t.m.cn_steepness * ((t.at_rcov[gi] + t.at_rcov[gj]) / r - 1.0));
        continue;
      }
      if (r2 <= 625.0) {
        const double rad = t.at_rcov[gi] + t.at_rcov[gj];
        const double f1 = logistic(10.0 * (rad / r - 1.0));
        const double f2 = logistic(20.0 * ((rad + 2.0) / r - 1.0));
        c1 += f1 * f2;
      }
      if (r2 <= 900.0) {
        const int zi = t.Z[gi] - 1, zj = t.Z[gj] - 1;
        const double rc = t.d4_rcov[zi] + t.d4_rcov[zj];
        const double den = fabs(t.d4_en[zi] - t.d4_en[zj]);
        const double enf = 4.10451 * exp(-(den + 19.08857) * (den + 19.08857) / (2.0 * 11.28174 * 11.28174));
        const double x = 7.5 * (r - rc) / rc;
        c4 += 0.5 * enf * (1.0 + erf(-x));
      }
    }
    c1 = warp_sum(c1);
    c4 = warp_sum(c4);
    if (lane == 0) {
      scn[i] = c1;
      scn4[i] = c4;
    }
  }
  __syncthreads();
  for (int64_t i = threadIdx.x; i < na; i += blockDim.x) {
    const int64_t g = a0 + i;
    cn[g] = scn[i];
    cn_d4[g] = scn4[i];
    const double arg = t.m.mp_kexp * (scn[i] - t.at_mpvcn[g] - t.m.mp_shift);
    const double fr = logistic(arg);
    mrad[g] = t.at_mprad[g] + (t.m.mp_rmax - t.at_mprad[g]) * fr;
    dmrad[g] = (t.m.mp_rmax - t.at_mprad[g]) * t.m.mp_kexp * fr * (1.0 - fr);
  }
}

// One thread per atom pair (A >= B) of one system; writes every element of
// the S, D, Q and H0 blocks (forward: rows on B, columns on A; reverse: rows
// on A, columns on B, operator origin moved to B).
__global__ void k_integrals(DevTopo t, const int32_t* list, const double* cn, double* S,
                            double* D, double* Q, double* H0, int64_t total_mat) {
  const int s = list[blockIdx.y];
  const int64_t a0 = t.atom_off[s], na = t.atom_off[s + 1] - a0;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= na * (na + 1) / 2) return;
  int64_t A = (int64_t)((sqrt(1.0 + 8.0 * (double)p) - 1.0) * 0.5);
  while (A * (A + 1) / 2 > p) --A;
  while ((A + 1) * (A + 2) / 2 <= p) ++A;
  const int64_t B = p - A * (A + 1) / 2;
  const int64_t gA = a0 + A, gB = a0 + B;
  const int n = t.nao[s];
  const int64_t mo = t.mat_off[s];
  const double v[3] = {t.pos[3 * gA] - t.pos[3 * gB], t.pos[3 * gA + 1] - t.pos[3 * gB + 1],
                       t.pos[3 * gA + 2] - t.pos[3 * gB + 2]};
  const double r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  const bool same = (A == B);
  for (int ks = t.atom_sh[gA]; ks < t.atom_sh[gA + 1]; ++ks) {
    const int lk = t.sh_l[ks];
    const int npk = t.sh_np[ks];
    const double* ak = t.p_alpha + t.sh_p0[ks];
    const double* ck = t.p_coeff + t.sh_p0[ks];
    for (int bs = t.atom_sh[gB]; bs < t.atom_sh[gB + 1]; ++bs) {
      if (same && bs > ks) continue;
      const int lb = t.sh_l[bs];
      const int npb = t.sh_np[bs];
      const double* ab = t.p_alpha + t.sh_p0[bs];
      const double* cb = t.p_coeff + t.sh_p0[bs];
      const double fac = h0_factor(t, bs, ks, cn, r, same);
      for (int ib = 0; ib < 2 * lb + 1; ++ib) {
        const int64_t row = t.sh_ao[bs] + ib;
        for (int ik = 0; ik < 2 * lk + 1; ++ik) {
          if (bs == ks && ib > ik) continue;
          const int64_t col = t.sh_ao[ks] + ik;
          double val[10];
          sph_pair<false>(lb, ib, lk, ik, ab, cb, npb, ak, ck, npk, v, val, nullptr);
          const int64_t f = mo + row * n + col;
          const int64_t rv = mo + col * n + row;
          S[f] = val[0];
          H0[f] = val[0] * fac;
#pragma unroll
          for (int c = 0; c < 3; ++c) D[c * total_mat + f] = val[1 + c];
#pragma unroll
          for (int c = 0; c < 6; ++c) Q[c * total_mat + f] = val[4 + c];
          if (f == rv) continue;
          if (bs == ks) {
            // same shell on the same atom: exactly symmetric element pair
            S[rv] = val[0];
            H0[rv] = val[0] * fac;
#pragma unroll
            for (int c = 0; c < 3; ++c) D[c * total_mat + rv] = val[1 + c];
#pragma unroll
            for (int c = 0; c < 6; ++c) Q[c * total_mat + rv] = val[4 + c];
            continue;
          }
          double rev[10];
          shift_to_bra(v, val, rev);
          S[rv] = val[0];
          H0[rv] = val[0] * fac;
#pragma unroll
          for (int c = 0; c < 3; ++c) D[c * total_mat + rv] = rev[1 + c];
#pragma unroll
          for (int c = 0; c < 6; ++c) Q[c * total_mat + rv] = rev[4 + c];
        }
      }
    }
  }
}

// ES2 shell Coulomb matrix gamma_ij = 1/sqrt(r^2 + eta_ij^-2), onsite eta_ij,
// eta_ij the arithmetic mean of the shell hardnesses for GFN2
// (model/gfn2/es2.cpp:211-300), the harmonic mean for GFN1 (model/gfn1/es2.cpp).
__global__ void k_es2_gamma(DevTopo t, const int32_t* list, double* gam) {
  const int s = list[blockIdx.y];
  const int64_t s0 = t.shell_off[s], k = t.shell_off[s + 1] - s0;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= k * k) return;
  const int64_t i = e / k, j = e % k;
  const int gi = (int)(s0 + i), gj = (int)(s0 + j);
  const double ea = t.sh_eta[gi], eb = t.sh_eta[gj];
  const double avg = t.m.gfn1 ? 2.0 / (1.0 / ea + 1.0 / eb) : 0.5 * (ea + eb);
  const int A = t.sh_atom[gi], B = t.sh_atom[gj];
  double g;
  if (A == B) {
    g = avg;
  } else {
    const double dx = t.pos[3 * A] - t.pos[3 * B];
    const double dy = t.pos[3 * A + 1] - t.pos[3 * B + 1];
    const double dz = t.pos[3 * A + 2] - t.pos[3 * B + 2];
    const double ia = 1.0 / avg;
    g = 1.0 / sqrt(dx * dx + dy * dy + dz * dz + ia * ia);
  }
  gam[t.gam_off[s] + e] = g;
}

void launch_setup(const DevTopo& t, const int32_t* list, int count, int max_atoms,
                  int64_t max_pairs, int64_t max_shells, double* cn, double* cn_d4, double* mrad,
                  double* dmrad, double* S, double* D, double* Q, double* H0, double* gam,
                  int64_t total_mat, cudaStream_t stream) {
  if (count == 0) return;
  const size_t sm = 2 * sizeof(double) * (size_t)max_atoms;
  const size_t attr = allow_max_dynamic_smem(k_coordination);
  (void)attr;
  k_coordination<<<count, 256, sm, stream>>>(t, list, cn, cn_d4, mrad, dmrad);
  const int tpb = 64;
  dim3 g1((unsigned)((max_pairs + tpb - 1) / tpb), count);
  k_integrals<<<g1, tpb, 0, stream>>>(t, list, cn, S, D, Q, H0, total_mat);
  dim3 g2((unsigned)((max_shells * max_shells + 255) / 256), count);
  k_es2_gamma<<<g2, 256, 0, stream>>>(t, list, gam);
}

}  // namespace xtb
