// Analytic gradient of the converged GFN2 energy.
//
//  * k_force_pairs: one thread per atom pair recomputes the shell-pair
//    overlap/multipole integrals with their derivatives and contracts them on
//    the fly with the adjoints P*dH0/dS - W and the stationary S/D/Q
//    potential adjoints (so dS/dR is never stored), adds the H0 distance
//    polynomial term and accumulates dE/dCN (model/gfn2/force.cpp:256-300,
//    520-560; model/gfn2/h0.cpp:469-597; common/integrals.cpp:440-496,867-1145).
//  * k_classical: ES2, AES2 (with the multipole-radius CN chain), D4
//    two-body at fixed charges, D4 ATM and repulsion energies/gradients
//    (model/gfn2/es2.cpp:1040-1110, aes2.cpp:596-713, d4.cpp:1034-1362,
//    repulsion.cpp:93-176).
//  * k_cn_chain: chain rule through both coordination numbers.
#include "classical.cuh"
#include "h0.cuh"
#include "integrals.cuh"
#include "kernels.cuh"

namespace xtb {

__device__ __forceinline__ double lev(const DevTopo& t, int sh, const double* cn) {
  return t.sh_level[sh] - t.sh_kcn[sh] * cn[t.sh_atom[sh]];
}

__global__ void __launch_bounds__(128) k_force_pairs(ForceArgs f) {
  const DevTopo& t = f.t;
  const int s = f.list[blockIdx.y];
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
  const double* P = f.P + mo;
  const double* W = f.W + mo;
  // unrestricted: the magnetisation is an overlap population too, so
  // P_alpha - P_beta with the spin potential enters the overlap adjoint
  const bool uhf = t.nch[s] == 2;
  const double* Pm = uhf ? f.Pm + mo : nullptr;
  if (A == B) return;   // onsite blocks: k_force_onsite
  const double v[3] = {t.pos[3 * gA] - t.pos[3 * gB], t.pos[3 * gA + 1] - t.pos[3 * gB + 1],
                       t.pos[3 * gA + 2] - t.pos[3 * gB + 2]};
  const double r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  const double* vdA = f.vd + 3 * gA;
  const double* vdB = f.vd + 3 * gB;
  const double* vqA = f.vq + 6 * gA;
  const double* vqB = f.vq + 6 * gB;
  double g[3] = {0.0, 0.0, 0.0};
  double cnA = 0.0, cnB = 0.0;
  for (int ks = t.atom_sh[gA]; ks < t.atom_sh[gA + 1]; ++ks) {
    const int lk = t.sh_l[ks];
    const int npk = t.sh_np[ks];
    const double* ak = t.p_alpha + t.sh_p0[ks];
    const double* ck = t.p_coeff + t.sh_p0[ks];
    const double vk = f.vsh[ks];
    const double vmk = uhf ? f.vmag[ks] : 0.0;
    for (int bs = t.atom_sh[gB]; bs < t.atom_sh[gB + 1]; ++bs) {
      const int lb = t.sh_l[bs];
      const int npb = t.sh_np[bs];
      const double* ab = t.p_alpha + t.sh_p0[bs];
      const double* cb = t.p_coeff + t.sh_p0[bs];
      const double vb = f.vsh[bs];
      const double vmb = uhf ? f.vmag[bs] : 0.0;
      // H0 factor pieces
      const double avg = 0.5 * (lev(t, bs, f.cn) + lev(t, ks, f.cn));
      const double ps = h0_pair_scale(t, bs, ks);
      const double rr = sqrt(r / (t.at_rad[gB] + t.at_rad[gA]));
      const double p1 = 1.0 + t.sh_shpoly[bs] * rr, p2 = 1.0 + t.sh_shpoly[ks] * rr;
      const double spat = ps * p1 * p2;
      const double dspat = ps * (t.sh_shpoly[bs] * p2 + t.sh_shpoly[ks] * p1) * rr / (2.0 * r);
      const double fac = avg * spat;
      double bw = 0.0;
      // the primitive-pair factors of this shell pair, shared by its 2l+1 x
      // 2l'+1 function pairs (shells with more primitives recompute them)
      const bool cached = npk * npb <= kPrimPairs;
      PrimPairs pp;
      if (cached) prim_pairs(ab, npb, ak, npk, v, pp);
      for (int ib = 0; ib < 2 * lb + 1; ++ib) {
        const int64_t row = t.sh_ao[bs] + ib;
        for (int ik = 0; ik < 2 * lk + 1; ++ik) {
          const int64_t col = t.sh_ao[ks] + ik;
          const double Pv = P[row * n + col];
          const double Wv = W[row * n + col];
          double val[10], dv[3][10];
          if (cached)
            sph_pair_pp<true>(lb, ib, lk, ik, ab, cb, npb, ak, ck, npk, v, pp, val, dv);
          else
            sph_pair<true>(lb, ib, lk, ik, ab, cb, npb, ak, ck, npk, v, val, dv);
          const double S = val[0];
          bw += Pv * S;
          double sA = 2.0 * (Pv * fac - Wv) - Pv * (vb + vk);
          if (uhf) sA -= Pm[row * n + col] * (vmb + vmk);
          double fD[3], rD[3], qadj[6], rQ[6];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            fD[c] = -Pv * vdA[c];
            rD[c] = -Pv * vdB[c];
          }
#pragma unroll
          for (int c = 0; c < 6; ++c) {
            rQ[c] = -Pv * vqB[c];
            qadj[c] = -Pv * vqA[c] + rQ[c];
          }
          const double dsum = rQ[0] + rQ[2] + rQ[5];
          const double axx = 1.5 * rQ[0] - 0.5 * dsum, axy = 1.5 * rQ[1];
          const double ayy = 1.5 * rQ[2] - 0.5 * dsum, axz = 1.5 * rQ[3];
          const double ayz = 1.5 * rQ[4], azz = 1.5 * rQ[5] - 0.5 * dsum;
          const double x = v[0], y = v[1], z = v[2];
          const double sadj = sA + rD[0] * x + rD[1] * y + rD[2] * z + axx * x * x + axy * x * y +
                              ayy * y * y + axz * x * z + ayz * y * z + azz * z * z;
          const double dadj[3] = {fD[0] + rD[0] + 2.0 * axx * x + axy * y + axz * z,
                                  fD[1] + rD[1] + axy * x + 2.0 * ayy * y + ayz * z,
                                  fD[2] + rD[2] + axz * x + ayz * y + 2.0 * azz * z};
          const double Dx = val[1], Dy = val[2], Dz = val[3];
          const double vadj[3] = {
              rD[0] * S + axx * (2.0 * Dx + 2.0 * x * S) + axy * (Dy + y * S) + axz * (Dz + z * S),
              rD[1] * S + axy * (Dx + x * S) + ayy * (2.0 * Dy + 2.0 * y * S) + ayz * (Dz + z * S),
              rD[2] * S + axz * (Dx + x * S) + ayz * (Dy + y * S) + azz * (2.0 * Dz + 2.0 * z * S)};
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            double acc = vadj[c] + sadj * dv[c][0];
#pragma unroll
            for (int k = 0; k < 3; ++k) acc += dadj[k] * dv[c][1 + k];
#pragma unroll
            for (int k = 0; k < 6; ++k) acc += qadj[k] * dv[c][4 + k];
            g[c] += acc;
          }
        }
      }
      const double rad = 2.0 * bw * avg * dspat / r;
      g[0] += rad * v[0];
      g[1] += rad * v[1];
      g[2] += rad * v[2];
      cnB -= t.sh_kcn[bs] * bw * spat;
      cnA -= t.sh_kcn[ks] * bw * spat;
    }
  }
  if (f.want_grad) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      fix_add(&f.grad[3 * gA + c], g[c]);
      fix_add(&f.grad[3 * gB + c], -g[c]);
    }
  }
  fix_add(&f.acn[gA], cnA);
  fix_add(&f.acn[gB], cnB);
}

// Onsite CN adjoint of the shell levels: one thread per atom.
__global__ void k_force_onsite(ForceArgs f) {
  const DevTopo& t = f.t;
  const int s = f.list[blockIdx.y];
  const int64_t a0 = t.atom_off[s], na = t.atom_off[s + 1] - a0;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= na) return;
  const int64_t gA = a0 + i;
  const int n = t.nao[s];
  const double* P = f.P + t.mat_off[s];
  const double* S = f.S + t.mat_off[s];
  double acc = 0.0;
  for (int x = t.atom_sh[gA]; x < t.atom_sh[gA + 1]; ++x) {
    for (int y = t.atom_sh[gA]; y < t.atom_sh[gA + 1]; ++y) {
      double bw = 0.0;
      for (int k = 0; k < 2 * t.sh_l[x] + 1; ++k)
        for (int l = 0; l < 2 * t.sh_l[y] + 1; ++l) {
          const int64_t idx = (int64_t)(t.sh_ao[x] + k) * n + t.sh_ao[y] + l;
          bw += P[idx] * S[idx];
        }
      acc -= 0.5 * bw * (t.sh_kcn[x] + t.sh_kcn[y]);
    }
  }
  fix_add(&f.acn[gA], acc);
}

void launch_force_pairs(const ForceArgs& f, int64_t max_pairs, cudaStream_t stream) {
  if (f.count == 0) return;
  const int tpb = 128;
  dim3 grid((unsigned)((max_pairs + tpb - 1) / tpb), f.count);
  k_force_pairs<<<grid, tpb, 0, stream>>>(f);
}

// ---------------------------------------------------------------------------
// Classical terms: one CTA per system, gradients accumulated in shared memory.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_classical(ForceArgs f) {
  extern __shared__ double sm[];
  const DevTopo& t = f.t;
  const int s = f.list[blockIdx.x];
  const int64_t a0 = t.atom_off[s];
  const int na = (int)(t.atom_off[s + 1] - a0);
  const int64_t s0 = t.shell_off[s];
  const int ns = (int)(t.shell_off[s + 1] - s0);
  double* gr = sm;                         // 3 na
  double* acn = gr + 3 * na;               // na (dexp)
  double* acn4 = acn + na;                 // na (D4)
  double* qat = acn4 + na;                 // na
  double* w = qat + na;                    // 7 na (charged weights)
  double* wcn = w + kMaxD4Refs * na;       // 7 na (d w / d cn)
  double* red = wcn + kMaxD4Refs * na;     // 40
  const int tid = threadIdx.x, bs = blockDim.x;
  const bool grad = f.want_grad != 0;
  for (int i = tid; i < na; i += bs) {
    const int64_t g = a0 + i;
    gr[3 * i] = gr[3 * i + 1] = gr[3 * i + 2] = 0.0;
    acn[i] = 0.0;
    acn4[i] = 0.0;
    double q = 0.0;
    for (int sh = t.atom_sh[g]; sh < t.atom_sh[g + 1]; ++sh) q += f.qsh[sh];
    qat[i] = q;
    if (t.m.gfn1)   // D3 reference weights at the GFN1 CN, and their CN derivatives
      d3_weights(t, t.Z[g], f.cn[g], w + kMaxD4Refs * i, wcn + kMaxD4Refs * i);
    else
      d4_weights(t, t.Z[g], f.cn_d4[g], q, w + kMaxD4Refs * i, wcn + kMaxD4Refs * i, nullptr);
  }
  __syncthreads();
  double erep = 0.0, edisp = 0.0;
  const double* gam = f.gam + t.gam_off[s];
  const int64_t npair = (int64_t)na * (na - 1) / 2;
  for (int64_t p = tid; p < npair; p += bs) {
    int64_t ii, jj;
    pair_from_index(p, ii, jj);     // ii > jj
    const int i = (int)ii, j = (int)jj;
    const int64_t gi = a0 + i, gj = a0 + j;
    const double d[3] = {t.pos[3 * gi] - t.pos[3 * gj], t.pos[3 * gi + 1] - t.pos[3 * gj + 1],
                         t.pos[3 * gi + 2] - t.pos[3 * gj + 2]};
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double r = sqrt(r2);
    double gs = 0.0;   // scalar multiplying d for pair (i <- j)
    // repulsion
    if (r2 <= 625.0) {
      const bool light = t.Z[gi] <= 2 && t.Z[gj] <= 2;
      const double k = light ? t.m.rep_klight : t.m.rep_kexp;
      // r^k: k = 1.5 for heavy pairs; GFN2 takes k = 1 for pairs of H/He
      const double rp = k == 1.0 ? r : (k == 1.5 ? r * sqrt(r) : pow(r, k));
      const double pa = t.at_rep_sa[gi] * t.at_rep_sa[gj];
      const double pe = t.at_rep_z[gi] * t.at_rep_z[gj] * exp(-pa * rp) / r;
      erep += pe;
      gs -= (pa * k * rp + 1.0) * pe / r2;
    }
    // GFN1: D3(BJ) dispersion (not self-consistent; model/gfn1/d3.cpp:690-735)
    if (t.m.gfn1 && r2 >= DBL_EPSILON && r2 <= 2500.0) {
      double dci, dcj, e, der;
      const double c6 = d3_c6(t, t.Z[gi], t.Z[gj], w + kMaxD4Refs * i, wcn + kMaxD4Refs * i,
                              w + kMaxD4Refs * j, wcn + kMaxD4Refs * j, dci, dcj);
      d3_pair(t, t.Z[gi], t.Z[gj], r2, e, der);
      edisp += c6 * e;
      if (grad) {
        gs += c6 * der;
        fix_add(&acn[i], dci * e);
        fix_add(&acn[j], dcj * e);
      }
    }
    if (grad && !t.m.gfn1) {
      // ES2 at fixed shell charges
      double wsum = 0.0;
      for (int x = t.atom_sh[gi]; x < t.atom_sh[gi + 1]; ++x)
        for (int y = t.atom_sh[gj]; y < t.atom_sh[gj + 1]; ++y) {
          const double gv = gam[(int64_t)(x - s0) * ns + (y - s0)];
          wsum += f.qsh[x] * f.qsh[y] * gv * gv * gv;
        }
      gs -= wsum;
      // D4 two-body at fixed charges; pair orientation (first = j, second = i)
      double damp, ddamp;
      d4_pair_damping(t, t.Z[gj], t.Z[gi], r2, damp, ddamp);
      if (damp != 0.0) {
        double cj, ci;
        const double c6 = d4_c6(t, t.Z[gj], t.Z[gi], w + kMaxD4Refs * j, w + kMaxD4Refs * i,
                                wcn + kMaxD4Refs * j, wcn + kMaxD4Refs * i, &cj, &ci);
        // gradient[first=j] += -c6*ddamp*(R_j - R_i), i.e. gradient[i] += -c6*ddamp*d
        gs -= c6 * ddamp;
        fix_add(&acn4[j], -cj * damp);
        fix_add(&acn4[i], -ci * damp);
      }
      // AES2: first = j, second = i, displacement dd = R_j - R_i = -d
      {
        const double dd[3] = {-d[0], -d[1], -d[2]};
        const double R = 0.5 * (f.mrad[gj] + f.mrad[gi]);
        double k3, k5;
        aes2_kernels(r, R, k3, k5);
        const double sc = R / r;
        const double f3 = 1.0 / (1.0 + 6.0 * sc * sc * sc);
        const double f5 = 1.0 / (1.0 + 6.0 * sc * sc * sc * sc);
        const double* dpf = f.dip + 3 * gj;
        const double* dps = f.dip + 3 * gi;
        const double* qf = f.qp + 6 * gj;
        const double* qs = f.qp + 6 * gi;
        const double qfv = qat[j], qsv = qat[i];
        double cdv[3], pf = 0.0, ps = 0.0, ddt = 0.0;
        for (int c = 0; c < 3; ++c) {
          cdv[c] = qfv * dps[c] - qsv * dpf[c];
          pf += dd[c] * dpf[c];
          ps += dd[c] * dps[c];
          ddt += dpf[c] * dps[c];
        }
        const double cdn = dd[0] * cdv[0] + dd[1] * cdv[1] + dd[2] * cdv[2];
        const double ddn = r2 * ddt - 3.0 * pf * ps;
        double T[6];
        for (int c = 0; c < 6; ++c) T[c] = qfv * qs[c] + qsv * qf[c];
        const double tv[3] = {T[0] * dd[0] + T[1] * dd[1] + T[3] * dd[2],
                              T[1] * dd[0] + T[2] * dd[1] + T[4] * dd[2],
                              T[3] * dd[0] + T[4] * dd[1] + T[5] * dd[2]};
        const double cqn = dd[0] * tv[0] + dd[1] * tv[1] + dd[2] * tv[2];
        const double k3d = -3.0 * f3 * k3 / r;
        const double k5d = -(1.0 + 4.0 * f5) * k5 / r;
        const double k3r = -3.0 * (1.0 - f3) * k3 / R;
        const double k5r = -4.0 * (1.0 - f5) * k5 / R;
        const double k5n = ddn + cqn;
        const double erd = k3r * cdn + k5r * k5n;
        for (int c = 0; c < 3; ++c) {
          const double ddd = 2.0 * ddt * dd[c] - 3.0 * (pf * dps[c] + ps * dpf[c]);
          const double gc = k3 * cdv[c] + k3d * cdn * dd[c] / r + k5 * (ddd + 2.0 * tv[c]) +
                            k5d * k5n * dd[c] / r;
          fix_add(&gr[3 * j + c], gc);
          fix_add(&gr[3 * i + c], -gc);
        }
        fix_add(&acn[j], 0.5 * erd * f.dmrad[gj]);
        fix_add(&acn[i], 0.5 * erd * f.dmrad[gi]);
      }
    }
    if (grad && t.m.gfn1) {
      // ES2 at fixed shell charges
      double wsum = 0.0;
      for (int x = t.atom_sh[gi]; x < t.atom_sh[gi + 1]; ++x)
        for (int y = t.atom_sh[gj]; y < t.atom_sh[gj + 1]; ++y) {
          const double gv = gam[(int64_t)(x - s0) * ns + (y - s0)];
          wsum += f.qsh[x] * f.qsh[y] * gv * gv * gv;
        }
      gs -= wsum;
    }
    if (grad) {
      for (int c = 0; c < 3; ++c) {
        fix_add(&gr[3 * i + c], gs * d[c]);
        fix_add(&gr[3 * j + c], -gs * d[c]);
      }
    }
  }
  erep = block_sum(erep, red);
  edisp = block_sum(edisp, red);
  if (tid == 0) {
    f.terms[kTermCount * (int64_t)s + kTermRep] = erep;
    if (t.m.gfn1) f.terms[kTermCount * (int64_t)s + kTermDisp3] = edisp;
  }
  if (!grad) return;
  for (int i = tid; i < na; i += bs) {
    const int64_t g = a0 + i;
    for (int c = 0; c < 3; ++c) fix_merge(&f.grad[3 * g + c], gr[3 * i + c]);
    fix_merge(&f.acn[g], acn[i]);
    fix_merge(&f.acn_d4[g], acn4[i]);
  }
}

// ---------------------------------------------------------------------------
// D4 three-body (Axilrod-Teller-Muto) term at zero charges
// (model/gfn2/d4.cpp of the reference): triples i > j > k with all three
// distances within 25 bohr.  The pair C6 coefficients and their CN
// derivatives are tabulated once per system (O(N^2)), so the O(N^3) triple
// loop only reads them.
// ---------------------------------------------------------------------------
// Table of system s (one CTA): C6[i][j] (symmetric) and D[i][j] = dC6_ij /
// dCN_i, with row stride = atoms, at the system's matrix offset of two work
// arrays of n^2 >= atoms^2 doubles.  Each pair i > j is evaluated with i as
// the first partner, the orientation of the triple loop.
__global__ void __launch_bounds__(256) k_atm_table(ForceArgs f) {
  extern __shared__ double sm[];
  const DevTopo& t = f.t;
  const int s = f.list[blockIdx.x];
  const int64_t a0 = t.atom_off[s];
  const int na = (int)(t.atom_off[s + 1] - a0);
  double* w0 = sm;                         // 7 na zero-charge weights
  double* w0cn = w0 + kMaxD4Refs * na;     // 7 na, d w / d cn
  for (int i = threadIdx.x; i < na; i += blockDim.x) {
    const int64_t g = a0 + i;
    d4_weights(t, t.Z[g], f.cn_d4[g], 0.0, w0 + kMaxD4Refs * i, w0cn + kMaxD4Refs * i, nullptr);
  }
  __syncthreads();
  double* C6 = f.atm_c6 + t.mat_off[s];
  double* D = f.atm_dc6 + t.mat_off[s];
  const int64_t npair = (int64_t)na * (na - 1) / 2;
  for (int64_t p = threadIdx.x; p < npair; p += blockDim.x) {
    int64_t ii, jj;
    pair_from_index(p, ii, jj);
    const int i = (int)ii, j = (int)jj;
    double ci, cj;
    const double c6 = d4_c6(t, t.Z[a0 + i], t.Z[a0 + j], w0 + kMaxD4Refs * i, w0 + kMaxD4Refs * j,
                            w0cn + kMaxD4Refs * i, w0cn + kMaxD4Refs * j, &ci, &cj);
    C6[(int64_t)i * na + j] = c6;
    C6[(int64_t)j * na + i] = c6;
    D[(int64_t)i * na + j] = ci;
    D[(int64_t)j * na + i] = cj;
  }
}

// Grid (parts, systems): warp w of part p takes pairs i > j (p * 8 + w, step
// 8 parts), its lanes the third atoms k < j.  Gradients of k go into shared
// accumulators per triple; those of i and j are reduced over the warp once
// per pair.  The energy of a part goes to the system's work array (parts >
// 1; k_atm_combine adds them in part order) or straight into the terms.
__global__ void __launch_bounds__(256) k_atm(ForceArgs f, int parts) {
  extern __shared__ double sm[];
  __shared__ double red[33];
  const DevTopo& t = f.t;
  const int s = f.list[blockIdx.y];
  const int64_t a0 = t.atom_off[s];
  const int na = (int)(t.atom_off[s + 1] - a0);
  const bool grad = f.want_grad != 0;
  double* gr = sm;            // 3 na
  double* acn4 = gr + 3 * na; // na
  for (int i = threadIdx.x; i < 4 * na; i += blockDim.x) gr[i] = 0.0;
  __syncthreads();
  const double* C6 = f.atm_c6 + t.mat_off[s];
  const double* D = f.atm_dc6 + t.mat_off[s];
  const int lane = threadIdx.x & 31;
  const int nwt = parts * (int)(blockDim.x >> 5);
  const int64_t npair = (int64_t)na * (na - 1) / 2;
  double eatm = 0.0;
  for (int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); p < npair; p += nwt) {
    int64_t ii, jj;
    pair_from_index(p, ii, jj);     // ii > jj
    const int i = (int)ii, j = (int)jj;
    if (j == 0) continue;            // uniform over the warp: no third atom
    const int64_t gi = a0 + i, gj = a0 + j;
    const double vij[3] = {t.pos[3 * gj] - t.pos[3 * gi], t.pos[3 * gj + 1] - t.pos[3 * gi + 1],
                           t.pos[3 * gj + 2] - t.pos[3 * gi + 2]};
    const double r2ij = vij[0] * vij[0] + vij[1] * vij[1] + vij[2] * vij[2];
    if (r2ij > 625.0) continue;
    const int zi = t.Z[gi], zj = t.Z[gj];
    const double cij = C6[(int64_t)i * na + j];
    const double cij_i = D[(int64_t)i * na + j], cij_j = D[(int64_t)j * na + i];
    const double r0ij = d4_r0(t, zi, zj);
    double g_i[3] = {0.0, 0.0, 0.0}, g_j[3] = {0.0, 0.0, 0.0}, a_i = 0.0, a_j = 0.0;
    for (int k = lane; k < j; k += 32) {
      const int64_t gk = a0 + k;
      const double vik[3] = {t.pos[3 * gk] - t.pos[3 * gi], t.pos[3 * gk + 1] - t.pos[3 * gi + 1],
                             t.pos[3 * gk + 2] - t.pos[3 * gi + 2]};
      const double vjk[3] = {t.pos[3 * gk] - t.pos[3 * gj], t.pos[3 * gk + 1] - t.pos[3 * gj + 1],
                             t.pos[3 * gk + 2] - t.pos[3 * gj + 2]};
      const double r2ik = vik[0] * vik[0] + vik[1] * vik[1] + vik[2] * vik[2];
      const double r2jk = vjk[0] * vjk[0] + vjk[1] * vjk[1] + vjk[2] * vjk[2];
      if (r2ik > 625.0 || r2jk > 625.0) continue;
      const int zk = t.Z[gk];
      const double cik = C6[(int64_t)i * na + k], cjk = C6[(int64_t)j * na + k];
      const double r0ik = d4_r0(t, zi, zk), r0jk = d4_r0(t, zj, zk);
      // one reciprocal for every power of r = sqrt(r2ij r2ik r2jk), and
      // (r0 / r)^(16/3) as (r0 / r)^5 cbrt(r0 / r)
      const double r2p = r2ij * r2ik * r2jk;
      const double ir1 = 1.0 / sqrt(r2p);
      const double ir2 = ir1 * ir1;
      const double ir3 = ir2 * ir1;
      const double ir5 = ir3 * ir2;
      const double ratio = r0ij * r0ik * r0jk * ir1;
      const double rat2 = ratio * ratio;
      const double rpow = rat2 * rat2 * ratio * cbrt(ratio);
      const double damp = 1.0 / (1.0 + 6.0 * rpow);
      const double ang = 0.375 * (r2ij + r2jk - r2ik) * (r2ij - r2jk + r2ik) * (-r2ij + r2jk + r2ik) * ir5 +
                         ir3;
      const double prod = cij * cik * cjk;
      const double c9 = -t.m.d4_s9 * sqrt(fabs(prod));
      eatm -= ang * damp * c9;
      if (!grad || !(cij > 0.0) || !(cik > 0.0) || !(cjk > 0.0)) continue;
      const double ddmp = -2.0 * 16.0 * rpow * damp * damp;
      // itt = 1 / tt from the reciprocal of the product: 1/r2ij = r2ik r2jk / r2p
      auto dg = [&](double tt, double o1, double o2, double itt) {
        const double dang = -0.375 *
                            (tt * tt * tt + tt * tt * (o1 + o2) + tt * (3.0 * o1 * o1 + 2.0 * o1 * o2 + 3.0 * o2 * o2) -
                             5.0 * (o1 - o2) * (o1 - o2) * (o1 + o2)) * ir5;
        return c9 * (-dang * damp + ang * ddmp) * itt;
      };
      // vij = R_j - R_i as in the reference's pair cache (first = j, second = i)
      const double sij = dg(r2ij, r2jk, r2ik, r2ik * r2jk * ir2);
      const double sik = dg(r2ik, r2jk, r2ij, r2ij * r2jk * ir2);
      const double sjk = dg(r2jk, r2ik, r2ij, r2ij * r2ik * ir2);
      for (int c = 0; c < 3; ++c) {
        const double gij = sij * vij[c], gik = sik * vik[c], gjk = sjk * vjk[c];
        g_i[c] -= gij + gik;
        g_j[c] += gij - gjk;
        fix_add(&gr[3 * k + c], gik + gjk);
      }
      const double de = ang * damp * c9;
      const double cik_i = D[(int64_t)i * na + k], cik_k = D[(int64_t)k * na + i];
      const double cjk_j = D[(int64_t)j * na + k], cjk_k = D[(int64_t)k * na + j];
      // 1/cij, 1/cik, 1/cjk from one reciprocal of their product (all > 0 here)
      const double iprod = 1.0 / prod;
      const double icij = cik * cjk * iprod, icik = cij * cjk * iprod, icjk = cij * cik * iprod;
      a_i -= 0.5 * de * (cij_i * icij + cik_i * icik);
      a_j -= 0.5 * de * (cij_j * icij + cjk_j * icjk);
      fix_add(&acn4[k], -0.5 * de * (cik_k * icik + cjk_k * icjk));
    }
    if (grad) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        g_i[c] = warp_sum(g_i[c]);
        g_j[c] = warp_sum(g_j[c]);
      }
      a_i = warp_sum(a_i);
      a_j = warp_sum(a_j);
      if (lane == 0) {
        for (int c = 0; c < 3; ++c) {
          fix_add(&gr[3 * i + c], g_i[c]);
          fix_add(&gr[3 * j + c], g_j[c]);
        }
        fix_add(&acn4[i], a_i);
        fix_add(&acn4[j], a_j);
      }
    }
  }
  eatm = block_sum(eatm, red);
  if (threadIdx.x == 0) {
    if (parts == 1) f.terms[kTermCount * (int64_t)s + kTermAtm] = eatm;
    else f.work[f.work_off[s] + blockIdx.x] = eatm;
  }
  if (!grad) return;
  __syncthreads();
  for (int i = threadIdx.x; i < na; i += blockDim.x) {
    const int64_t g = a0 + i;
    for (int c = 0; c < 3; ++c) fix_merge(&f.grad[3 * g + c], gr[3 * i + c]);
    fix_merge(&f.acn_d4[g], acn4[i]);
  }
}

__global__ void k_atm_combine(ForceArgs f, int parts) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= f.count) return;
  const int s = f.list[idx];
  double e = 0.0;
  for (int q = 0; q < parts; ++q) e += f.work[f.work_off[s] + q];
  f.terms[kTermCount * (int64_t)s + kTermAtm] = e;
}

// GFN1 halogen-bond correction (model/gfn1/halogen.cpp:253-470): every donor
// (Cl, Br, I, At) with an acceptor (N, O, P, S) within 20 bohr takes its
// nearest atom as the bond axis; each acceptor within 20 bohr adds
//   E = xbond_X * ((1 - cos)/2)^6 * (1 - c r^6) / (1 + r^12),
// cos between donor->acceptor and donor->axis, r = R_XA / (1.3 (R_X + R_A)),
// c = 0.44.  A thread per donor; not self-consistent (once after the SCC).
__device__ __forceinline__ bool xb_donor(int z) { return z == 17 || z == 35 || z == 53 || z == 85; }
__device__ __forceinline__ bool xb_acceptor(int z) { return z == 7 || z == 8 || z == 15 || z == 16; }

__global__ void __launch_bounds__(128) k_halogen(ForceArgs f) {
  __shared__ double red[33];
  const DevTopo& t = f.t;
  const int s = f.list[blockIdx.x];
  const int64_t a0 = t.atom_off[s];
  const int na = (int)(t.atom_off[s + 1] - a0);
  constexpr double kCut = 20.0;
  double e = 0.0;
  auto dist = [&](int64_t p, int64_t q, double* d) {
    for (int c = 0; c < 3; ++c) d[c] = t.pos[3 * q + c] - t.pos[3 * p + c];
    return sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  };
  for (int x = threadIdx.x; x < na; x += blockDim.x) {
    const int64_t gx = a0 + x;
    if (!xb_donor(t.Z[gx])) continue;
    bool active = false;
    for (int y = 0; y < na && !active; ++y) {
      double d[3];
      if (xb_acceptor(t.Z[a0 + y]) && dist(gx, a0 + y, d) <= kCut) active = true;
    }
    if (!active) continue;
    int nb = -1;
    double best = DBL_MAX;
    for (int y = 0; y < na; ++y) {   // nearest atom; the lowest index on ties
      double d[3];
      const double r = dist(gx, a0 + y, d);
      if (r > 0.0 && r < best) {
        best = r;
        nb = y;
      }
    }
    if (nb < 0) continue;
    const int64_t gn = a0 + nb;
    double un[3];
    const double rn = dist(gx, gn, un);
    for (int c = 0; c < 3; ++c) un[c] /= rn;
    const double rx = t.m.xb_radius_scale * t.at_rad[gx];
    for (int y = 0; y < na; ++y) {
      const int64_t ga = a0 + y;
      if (!xb_acceptor(t.Z[ga]) || ga == gn) continue;
      double ua[3];
      const double ra = dist(gx, ga, ua);
      if (ra > kCut) continue;
      for (int c = 0; c < 3; ++c) ua[c] /= ra;
      const double cs = ua[0] * un[0] + ua[1] * un[1] + ua[2] * un[2];
      const double ab = 0.5 * (1.0 - cs);
      const double ab2 = ab * ab;
      const double ang = ab2 * ab2 * ab2;
      const double rho = ra / (rx + t.m.xb_radius_scale * t.at_rad[ga]);
      const double rho2 = rho * rho, rho6 = rho2 * rho2 * rho2, rho12 = rho6 * rho6;
      const double den = 1.0 + rho12;
      const double rad = (1.0 - t.m.xb_damping * rho6) / den;
      const double str = t.at_xbond[gx];
      e += str * ang * rad;
      if (!f.want_grad) continue;
      const double drad = 6.0 * rho6 / ra * (t.m.xb_damping * rho12 - 2.0 * rho6 - t.m.xb_damping) / (den * den);
      const double dang = -3.0 * ab2 * ab2 * ab;
      for (int c = 0; c < 3; ++c) {
        const double dca = (un[c] - cs * ua[c]) / ra;
        const double dcn = (ua[c] - cs * un[c]) / rn;
        const double ga_c = str * (rad * dang * dca + ang * drad * ua[c]);
        const double gn_c = str * rad * dang * dcn;
        fix_add(&f.grad[3 * ga + c], ga_c);
        fix_add(&f.grad[3 * gn + c], gn_c);
        fix_add(&f.grad[3 * gx + c], -(ga_c + gn_c));
      }
    }
  }
  e = block_sum(e, red);
  if (threadIdx.x == 0) f.terms[kTermCount * (int64_t)s + kTermXb] = e;
}

void launch_classical(const ForceArgs& f, int max_atoms, int max_shells, cudaStream_t stream) {
  (void)max_shells;
  if (f.count == 0) return;
  const size_t sm = ((size_t)(7 + 2 * kMaxD4Refs) * max_atoms + 48) * sizeof(double);
  const size_t attr = allow_max_dynamic_smem(k_classical);
  const size_t attr_t = allow_max_dynamic_smem(k_atm_table);
  const size_t attr_a = allow_max_dynamic_smem(k_atm);
  (void)attr;
  (void)attr_t;
  (void)attr_a;
  k_classical<<<f.count, 256, sm, stream>>>(f);
  if (f.t.m.gfn1) {   // no three-body dispersion (s9 = 0); the halogen-bond term instead
    k_halogen<<<f.count, 128, 0, stream>>>(f);
    return;
  }
  k_atm_table<<<f.count, 256, (size_t)2 * kMaxD4Refs * max_atoms * sizeof(double), stream>>>(f);
  // few systems: each system's pairs over several CTAs
  const int parts = std::max(1, std::min(16, 2 * sm_count() / f.count));
  k_atm<<<dim3(parts, f.count), 256, (size_t)4 * max_atoms * sizeof(double), stream>>>(f, parts);
  if (parts > 1) k_atm_combine<<<(f.count + 127) / 128, 128, 0, stream>>>(f, parts);
}

// Chain rule through the double-exponential CN (acn) and the D4 CN (acn_d4).
__global__ void __launch_bounds__(256) k_cn_chain(ForceArgs f) {
  const DevTopo& t = f.t;
  const int s = f.list[blockIdx.x];
  const int64_t a0 = t.atom_off[s];
  const int na = (int)(t.atom_off[s + 1] - a0);
  const int64_t npair = (int64_t)na * (na - 1) / 2;
  for (int64_t p = threadIdx.x; p < npair; p += blockDim.x) {
    int64_t ii, jj;
    pair_from_index(p, ii, jj);
    const int64_t gi = a0 + ii, gj = a0 + jj;
    const double d[3] = {t.pos[3 * gi] - t.pos[3 * gj], t.pos[3 * gi + 1] - t.pos[3 * gj + 1],
                         t.pos[3 * gi + 2] - t.pos[3 * gj + 2]};
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double r = sqrt(r2);
    double sc = 0.0;
    if (t.m.gfn1) {
      // d/dr of 1 / (1 + exp(-k (rad / r - 1))) (model/gfn1/coordination.cpp:230-245)
      if (r2 <= 625.0 && r2 > 1e-12) {
        const double rad = t.at_rcov[gi] + t.at_rcov[gj];
        const double fv = logistic(t.m.cn_steepness * (rad / r - 1.0));
        const double dv = -t.m.cn_steepness * rad * fv * (1.0 - fv) / r2;
        sc += (fix_value(f.acn[gi]) + fix_value(f.acn[gj])) * dv / r;
      }
    } else if (r2 <= 625.0) {
      const double rad = t.at_rcov[gi] + t.at_rcov[gj];
      const double f1 = logistic(10.0 * (rad / r - 1.0));
      const double f2 = logistic(20.0 * ((rad + 2.0) / r - 1.0));
      const double dv = -(10.0 * rad * f1 * (1.0 - f1) * f2 + 20.0 * (rad + 2.0) * f2 * (1.0 - f2) * f1) / r2;
      sc += (fix_value(f.acn[gi]) + fix_value(f.acn[gj])) * dv / r;
    }
    if (!t.m.gfn1 && r2 <= 900.0) {
      const int zi = t.Z[gi] - 1, zj = t.Z[gj] - 1;
      const double rc = t.d4_rcov[zi] + t.d4_rcov[zj];
      const double den = fabs(t.d4_en[zi] - t.d4_en[zj]);
      const double enf = 4.10451 * exp(-(den + 19.08857) * (den + 19.08857) / (2.0 * 11.28174 * 11.28174));
      const double x = 7.5 * (r - rc) / rc;
      const double dv = -enf * 7.5 * exp(-x * x) / sqrt(kPi) / rc;
      sc += (fix_value(f.acn_d4[gi]) + fix_value(f.acn_d4[gj])) * dv / r;
    }
    if (sc != 0.0) {
      for (int c = 0; c < 3; ++c) {
        fix_add(&f.grad[3 * gi + c], sc * d[c]);
        fix_add(&f.grad[3 * gj + c], -sc * d[c]);
      }
    }
  }
}

void launch_cn_chain(const ForceArgs& f, int max_atoms, cudaStream_t stream) {
  if (f.count == 0) return;
  (void)max_atoms;
  // onsite shell-level CN adjoints first, then the pair chain rule
  dim3 g1((unsigned)((max_atoms + 127) / 128), f.count);
  k_force_onsite<<<g1, 128, 0, stream>>>(f);
  k_cn_chain<<<f.count, 256, 0, stream>>>(f);
}

}  // namespace xtb
