// Per-iteration SCC kernels: SAD start, potentials (ES2 + ES3 + AES2 + D4),
// Fock build, Mulliken populations with the band trace, and the fused energy
// functional + modified-Broyden mixer + convergence gate.
//
// Restated from model/gfn2/scc_driver.cpp:706-960 (iteration order),
// 2105-2560 (energy functional, potentials), model/gfn2/mulliken_kernels_impl.hpp
// (population and Hamiltonian contractions), model/gfn2/aes2.cpp:451-594
// (AES2 potentials/energy), model/gfn2/d4.cpp:730-980 (self-consistent D4),
// model/gfn2/es3.cpp:190-230 and common/scc_mixer.cpp:559-740 (Broyden).
#include "classical.cuh"
#include "kernels.cuh"

#include <algorithm>
#include <cfloat>

namespace xtb {

__global__ void k_sad_init(SccArgs a) {
  const int s = a.list[blockIdx.x];
  const DevTopo& t = a.t;
  const int64_t a0 = t.atom_off[s], na = t.atom_off[s + 1] - a0;
  const int64_t s0 = t.shell_off[s], ns = t.shell_off[s + 1] - s0;
  const int64_t v0 = t.vec_off[s];
  const double qa = t.qmol[s] / (double)na;
  for (int64_t i = threadIdx.x; i < na; i += blockDim.x) {
    const int64_t g = a0 + i;
    double ref = 0.0;
    for (int sh = t.atom_sh[g]; sh < t.atom_sh[g + 1]; ++sh) ref += t.sh_refocc[sh];
    for (int sh = t.atom_sh[g]; sh < t.atom_sh[g + 1]; ++sh) {
      const double q = t.sh_refocc[sh] / ref * qa;
      a.qsh[sh] = q;
      a.mx_cur[v0 + (sh - s0)] = q;
    }
    for (int c = 0; c < 3; ++c) a.dip[3 * g + c] = 0.0;
    for (int c = 0; c < 6; ++c) a.qp[6 * g + c] = 0.0;
    if (!t.m.gfn1) {
      for (int c = 0; c < 3; ++c) a.mx_cur[v0 + ns + 3 * i + c] = 0.0;
      for (int c = 0; c < 6; ++c) a.mx_cur[v0 + ns + 3 * na + 6 * i + c] = 0.0;
    }
  }
  if (t.nch[s] == 2) {
    // the magnetisation block of the mixed vector starts at zero
    const int64_t d1 = charge_block(t, (int)ns, (int)na);
    for (int64_t i = threadIdx.x; i < d1; i += blockDim.x) a.mx_cur[v0 + d1 + i] = 0.0;
    for (int64_t i = threadIdx.x; i < ns; i += blockDim.x) a.qmag[s0 + i] = 0.0;
  }
  if (threadIdx.x == 0) {
    a.iterations[s] = 0;
    a.converged[s] = 0;
    a.free_energy[s] = 0.0;
  }
}

// WARM start (src/runtime/gfn2_cpu_execution.cpp:1261-1266,1313-1325 of the
// reference): the previous converged state is the first mixed input, the
// mixer starts a new history from it.
__global__ void k_warm_init(SccArgs a) {
  const int s = a.list[blockIdx.x];
  const DevTopo& t = a.t;
  const int64_t a0 = t.atom_off[s], na = t.atom_off[s + 1] - a0;
  const int64_t s0 = t.shell_off[s], ns = t.shell_off[s + 1] - s0;
  const int64_t v0 = t.vec_off[s];
  const bool mp = !t.m.gfn1;   // the mixed vector carries atomic multipoles (GFN2)
  const int64_t d1 = charge_block(t, (int)ns, (int)na);
  for (int64_t i = threadIdx.x; i < ns; i += blockDim.x) {
    const double q = a.ck_qsh[s0 + i];
    a.qsh[s0 + i] = q;
    a.mx_cur[v0 + i] = q;
  }
  for (int64_t i = threadIdx.x; i < 3 * na; i += blockDim.x) {
    const double v = a.ck_dip[3 * a0 + i];
    a.dip[3 * a0 + i] = v;
    if (mp) a.mx_cur[v0 + ns + i] = v;
  }
  for (int64_t i = threadIdx.x; i < 6 * na; i += blockDim.x) {
    const double v = a.ck_qp[6 * a0 + i];
    a.qp[6 * a0 + i] = v;
    if (mp) a.mx_cur[v0 + ns + 3 * na + i] = v;
  }
  if (t.nch[s] == 2) {
    for (int64_t i = threadIdx.x; i < ns; i += blockDim.x) {
      const double m = a.ck_qmag[s0 + i];
      a.qmag[s0 + i] = m;
      a.mx_cur[v0 + d1 + i] = m;
    }
    // magnetisation multipoles: the raw values -pop of the converged iteration
    if (mp) {
      for (int64_t i = threadIdx.x; i < 3 * na; i += blockDim.x)
        a.mx_cur[v0 + d1 + ns + i] = -a.ck_mdip[3 * a0 + i];
      for (int64_t i = threadIdx.x; i < 6 * na; i += blockDim.x)
        a.mx_cur[v0 + d1 + ns + 3 * na + i] = -a.ck_mqp[6 * a0 + i];
    }
  }
  if (threadIdx.x == 0) {
    a.iterations[s] = 0;
    a.converged[s] = 0;
    a.free_energy[s] = 0.0;
  }
}

void launch_warm_init(const SccArgs& a, cudaStream_t stream) {
  if (a.count == 0) return;
  k_warm_init<<<a.count, 128, 0, stream>>>(a);
}

void launch_sad_init(const SccArgs& a, cudaStream_t stream) {
  if (a.count == 0) return;
  k_sad_init<<<a.count, 128, 0, stream>>>(a);
}

// ---------------------------------------------------------------------------
// Potentials from (qsh, dip, qp): vsh = gamma q + g3 q^2 + vat(atom);
// vat, vd, vq from AES2 and the D4 charge response.
// ---------------------------------------------------------------------------
// Per-atom inputs of the pair loop, system-local, in shared memory: atomic
// charges, D4 reference weights and their charge derivatives.
__device__ __forceinline__ void potential_atoms(const SccArgs& a, const double* qsh, int64_t a0,
                                                int na, double* qat, double* w, double* dwq) {
  const DevTopo& t = a.t;
  for (int i = threadIdx.x; i < na; i += blockDim.x) {
    const int64_t g = a0 + i;
    double q = 0.0;
    for (int sh = t.atom_sh[g]; sh < t.atom_sh[g + 1]; ++sh) q += qsh[sh];
    qat[i] = q;
    if (!t.m.gfn1)
      d4_weights(t, t.Z[g], a.cn_d4[g], q, w + kMaxD4Refs * i, nullptr, dwq + kMaxD4Refs * i);
  }
}

// Contribution of partner j to the potentials of atom i (dv = R_i - R_j):
// acc[0] atomic potential (AES2 + D4 charge response), acc[1..3] dipole
// potential, acc[4..9] quadrupole potential.  Each atom gathers over all its
// partners in a fixed order, so the sums are the same in every run and for
// every launch shape.
__device__ __forceinline__ void potential_gather_pair(const SccArgs& a, const double* dip,
                                                      const double* qp, int64_t a0, int i, int j,
                                                      const double* qat, const double* w,
                                                      const double* dwq, double* acc) {
  const DevTopo& t = a.t;
  const int64_t gi = a0 + i, gj = a0 + j;
  const double d[3] = {t.pos[3 * gi] - t.pos[3 * gj], t.pos[3 * gi + 1] - t.pos[3 * gj + 1],
                       t.pos[3 * gi + 2] - t.pos[3 * gj + 2]};
  const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  const double r = sqrt(r2);
  double k3, k5;
  aes2_kernels(r, 0.5 * (a.mrad[gi] + a.mrad[gj]), k3, k5);
  const double* dj = dip + 3 * gj;
  const double* qj = qp + 6 * gj;
  const double sqv[6] = {d[0] * d[0] * k5, 2.0 * d[0] * d[1] * k5, d[1] * d[1] * k5,
                         2.0 * d[0] * d[2] * k5, 2.0 * d[1] * d[2] * k5, d[2] * d[2] * k5};
  const double iso = r2 * k5;
  const double pj = d[0] * dj[0] + d[1] * dj[1] + d[2] * dj[2];
  double v = k3 * pj;
  for (int c = 0; c < 6; ++c) v += sqv[c] * qj[c];
  for (int c = 0; c < 3; ++c) acc[1 + c] += -qat[j] * d[c] * k3 + iso * dj[c] - 3.0 * k5 * d[c] * pj;
  for (int c = 0; c < 6; ++c) acc[4 + c] += qat[j] * sqv[c];
  double damp, ddamp;
  const int zi = t.Z[gi], zj = t.Z[gj];
  d4_pair_damping(t, zi, zj, r2, damp, ddamp);
  if (damp != 0.0) {
    double ci;
    d4_c6(t, zi, zj, w + kMaxD4Refs * i, w + kMaxD4Refs * j, dwq + kMaxD4Refs * i, nullptr, &ci,
          nullptr);
    v -= ci * damp;
  }
  acc[0] += v;
}

// (gamma q)_j = sum_i gamma[i][j] q[i] for the symmetric ns x ns gamma: the
// loads of 16 rows are issued before their products are summed (in row
// order), so a thread waits for memory once per 16 rows.
__device__ __forceinline__ double gamma_column_dot(const double* gam, int ns, int j, const double* q) {
  double acc = 0.0;
  for (int i0 = 0; i0 < ns; i0 += 16) {
    double gv[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) gv[u] = i0 + u < ns ? gam[(int64_t)(i0 + u) * ns + j] : 0.0;
#pragma unroll
    for (int u = 0; u < 16; ++u)
      if (i0 + u < ns) acc = fma(gv[u], q[i0 + u], acc);
  }
  return acc;
}

// Shell potentials of system s from the finished atomic potentials: ES2
// (thread per shell, down its column of the symmetric gamma: coalesced rows,
// independent loads) + ES3 + atomic potential (+ external point charges).
__device__ __forceinline__ void potential_shells(const SccArgs& a, int s, const double* sq,
                                                 const double* vat) {
  const DevTopo& t = a.t;
  const int64_t a0 = t.atom_off[s];
  const int64_t s0 = t.shell_off[s];
  const int ns = (int)(t.shell_off[s + 1] - s0);
  const double* gam = a.gam + t.gam_off[s];
  for (int j = threadIdx.x; j < ns; j += blockDim.x) {
    const double acc = gamma_column_dot(gam, ns, j, sq);
    const int sh = (int)(s0 + j);
    // third order: shell-resolved for GFN2; atom-resolved for GFN1, the
    // potential Gamma_A q_A^2 on every shell of atom A (model/gfn1/es3.cpp:100-125)
    double q = sq[j];
    if (t.m.gfn1) {
      const int at = t.sh_atom[sh];
      q = 0.0;
      for (int k = t.atom_sh[at]; k < t.atom_sh[at + 1]; ++k) q += sq[k - s0];
    }
    a.vsh[sh] = acc + t.sh_g3[sh] * q * q + vat[t.sh_atom[sh] - a0] +
                (t.vpc != nullptr ? t.vpc[sh] : 0.0);
  }
}

// Atomic, dipole and quadrupole potentials: CTA blockIdx.x of gridDim.x for
// system blockIdx.y; warp w of the grid's CTAs of a system gathers atom i for
// i = w, w + warps, ...  vat goes to vat_out (per atom), vd and vq to a.vd, a.vq.
__global__ void __launch_bounds__(256) k_potential_atoms(SccArgs a, const double* qsh,
                                                         const double* dip, const double* qp,
                                                         double* vat_out) {
  extern __shared__ double sm[];
  const DevTopo& t = a.t;
  const int s = a.list[blockIdx.y];
  const int64_t a0 = t.atom_off[s];
  const int na = (int)(t.atom_off[s + 1] - a0);
  const int nw = blockDim.x >> 5;
  const int gw0 = blockIdx.x * nw + (threadIdx.x >> 5), gstride = gridDim.x * nw;
  if (blockIdx.x * nw >= na) return;   // uniform over the block: no atom for this CTA
  double* qat = sm;
  double* w = qat + na;                     // na * 7
  double* dwq = w + kMaxD4Refs * na;        // na * 7
  potential_atoms(a, qsh, a0, na, qat, w, dwq);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const double scl[6] = {1.0, 2.0, 1.0, 2.0, 2.0, 1.0};
  for (int i = gw0; i < na; i += gstride) {
    double acc[10];
#pragma unroll
    for (int c = 0; c < 10; ++c) acc[c] = 0.0;
    // GFN1 has neither atomic multipoles nor self-consistent dispersion
    if (!t.m.gfn1)
      for (int j = lane; j < na; j += 32)
        if (j != i) potential_gather_pair(a, dip, qp, a0, i, j, qat, w, dwq, acc);
    // charge response (b + A q)_i of the mixed charges (reference
    // periodic_embedding.cpp evaluate_system_unchecked)
    if (t.resp_A != nullptr) {
      const double* Ar = t.resp_A + t.resp_off[s] + (int64_t)i * na;
      for (int j = lane; j < na; j += 32) acc[0] = fma(Ar[j], qat[j], acc[0]);
    }
#pragma unroll
    for (int c = 0; c < 10; ++c) acc[c] = warp_sum(acc[c]);
    if (lane == 0) {
      const int64_t g = a0 + i;
      if (t.resp_b != nullptr) acc[0] += t.resp_b[g];
      // uniform field (scc_driver.cpp:2555-2582 of the reference): v_at += -E.R,
      // dipole potential += -E
      const double* ef = t.efield != nullptr ? t.efield + 3 * s : nullptr;
      vat_out[g] = acc[0] - (ef != nullptr ? ef[0] * t.pos[3 * g] + ef[1] * t.pos[3 * g + 1] +
                                                 ef[2] * t.pos[3 * g + 2]
                                           : 0.0);
      const double dk2 = 2.0 * t.at_dk[g], qk2 = 2.0 * t.at_qk[g];
      for (int c = 0; c < 3; ++c)
        a.vd[3 * g + c] = dk2 * dip[3 * g + c] + acc[1 + c] - (ef != nullptr ? ef[c] : 0.0);
      for (int c = 0; c < 6; ++c) a.vq[6 * g + c] = qk2 * scl[c] * qp[6 * g + c] + acc[4 + c];
    }
  }
}

__global__ void __launch_bounds__(256) k_potential_shells(SccArgs a, const double* qsh,
                                                          const double* vat_in) {
  extern __shared__ double sm[];
  const DevTopo& t = a.t;
  const int s = a.list[blockIdx.x];
  const int64_t a0 = t.atom_off[s];
  const int na = (int)(t.atom_off[s + 1] - a0);
  const int64_t s0 = t.shell_off[s];
  const int ns = (int)(t.shell_off[s + 1] - s0);
  double* vat = sm;
  double* sq = vat + na;
  for (int i = threadIdx.x; i < na; i += blockDim.x) vat[i] = vat_in[a0 + i];
  for (int i = threadIdx.x; i < ns; i += blockDim.x) sq[i] = qsh[s0 + i];
  __syncthreads();
  potential_shells(a, s, sq, vat);
  // spin potential v_mag = W m of the atom-local couplings (unrestricted systems)
  if (t.nch[s] == 2) {
    for (int i = threadIdx.x; i < ns; i += blockDim.x) {
      const int64_t sh = s0 + i;
      const int at = t.sh_atom[sh];
      const int f0 = t.atom_sh[at], cnt = t.atom_sh[at + 1] - f0;
      double v = 0.0;
      for (int k = 0; k < cnt; ++k) v = fma(t.sh_spinw[3 * sh + k], a.qmag[f0 + k], v);
      a.vmag[sh] = v;
    }
  }
}

void launch_potential(const SccArgs& a, const double* qsh, const double* dip, const double* qp,
                      int max_atoms, int max_shells, cudaStream_t stream) {
  if (a.count == 0) return;
  const int sms = sm_count();
  // With fewer systems than SMs, each system's atoms are spread over CTAs
  // (at least one atom per warp) so that the whole GPU works on the few
  // systems left; the result does not depend on the split.
  const int parts = a.count * 2 > sms
                        ? 1
                        : std::max(1, std::min((max_atoms + 7) / 8, 2 * sms / a.count));
  const size_t sm1 = ((size_t)(1 + 2 * kMaxD4Refs) * max_atoms + 8) * sizeof(double);
  const size_t attr1 = allow_max_dynamic_smem(k_potential_atoms);
  (void)attr1;
  k_potential_atoms<<<dim3(parts, a.count), 256, sm1, stream>>>(a, qsh, dip, qp, a.pot_acc);
  const size_t sm2 = ((size_t)max_atoms + max_shells + 8) * sizeof(double);
  k_potential_shells<<<a.count, 256, sm2, stream>>>(a, qsh, a.pot_acc);
}

// ---------------------------------------------------------------------------
// Fock build on 32x32 tiles of the upper tile triangle:
//   H = H0 - S (v_mu + v_nu)/2 - (G + G^T)/2,
//   G[x][y] = sum_c D_c[x][y] vd_c(atom y) + Q_c[x][y] vq_c(atom y).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double g_element(const SccArgs& a, int64_t idx, int atom) {
  double g = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) g = fma(a.D[c * a.total_mat + idx], a.vd[3 * atom + c], g);
#pragma unroll
  for (int c = 0; c < 6; ++c) g = fma(a.Q[c * a.total_mat + idx], a.vq[6 * atom + c], g);
  return g;
}

// One spin channel per grid row: the restricted channel (or alpha/beta of an
// unrestricted system, with the spin potential added with sign +1 / -1:
// H_sigma = H0 - S (v + sigma v_mag)_mu,nu / 2 - ...).
__global__ void __launch_bounds__(256) k_fock(SccArgs a) {
  __shared__ double sg[32][33];
  const DevTopo& t = a.t;
  const int ch = a.clist[blockIdx.y];
  const int s = a.ch_sys[ch];
  const double sgn = (double)a.ch_sign[ch];
  const int n = t.nao[s];
  const int T = (n + 31) / 32;
  const int64_t p = blockIdx.x;
  if (p >= (int64_t)T * (T + 1) / 2) return;
  // p -> (ti <= tj): p = tj (tj + 1)/2 + ti
  int tj = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
  while ((int64_t)tj * (tj + 1) / 2 > p) --tj;
  while ((int64_t)(tj + 1) * (tj + 2) / 2 <= p) ++tj;
  const int ti = (int)(p - (int64_t)tj * (tj + 1) / 2);
  const int row0 = ti * 32, col0 = tj * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int64_t mo = t.mat_off[s];
  const int64_t ho = a.ch_mat[ch];   // this channel's Hamiltonian
  const int64_t ao0 = t.ao_off[s];
  // transposed tile: G(col0 + r, row0 + c) -> sg[r][c]
  for (int r = ty; r < 32; r += 8) {
    const int x = col0 + r, y = row0 + tx;
    double g = 0.0;
    if (x < n && y < n) g = g_element(a, mo + (int64_t)x * n + y, t.ao_at[ao0 + y]);
    sg[r][tx] = g;
  }
  __syncthreads();
  double h[4];
  const int y = col0 + tx;
  const bool yin = y < n;
  const double vy =
      yin ? a.vsh[t.ao_sh[ao0 + y]] + (sgn != 0.0 ? sgn * a.vmag[t.ao_sh[ao0 + y]] : 0.0) : 0.0;
  const int aty = yin ? t.ao_at[ao0 + y] : 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int r = ty + 8 * k;
    const int x = row0 + r;
    h[k] = 0.0;
    if (x < n && yin) {
      const int64_t idx = mo + (int64_t)x * n + y;
      const double g1 = g_element(a, idx, aty);
      const int shx = t.ao_sh[ao0 + x];
      const double vx = a.vsh[shx] + (sgn != 0.0 ? sgn * a.vmag[shx] : 0.0);
      h[k] = a.H0[idx] - 0.5 * a.S[idx] * (vx + vy) - 0.5 * (g1 + sg[tx][r]);
      a.H[ho + (int64_t)x * n + y] = h[k];
    }
  }
  if (ti == tj) return;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) sg[tx][ty + 8 * k] = h[k];
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int x = col0 + r, yy = row0 + tx;
    if (x < n && yy < n) a.H[ho + (int64_t)x * n + yy] = sg[r][tx];
  }
}

void launch_fock(const SccArgs& a, int max_n, cudaStream_t stream) {
  if (a.ccount == 0) return;
  const int T = (max_n + 31) / 32;
  dim3 grid((unsigned)(T * (T + 1) / 2), a.ccount);
  k_fock<<<grid, 256, 0, stream>>>(a);
}

// ---------------------------------------------------------------------------
// Mulliken populations (column reductions) and the band trace Tr(P H0).
// ---------------------------------------------------------------------------
// One CTA per system.  The n rows are cut into RP fixed chunks; thread
// (chunk, column) sums its column over its chunk, and the chunks, shells,
// atoms and the trace are then added in a fixed order, so the populations are
// the same in every run.
constexpr int kMullThreads = 512;

__device__ void mulliken_reduce(const SccArgs& a, int s, const double* part, double* out_sh,
                                double* out_dip, double* out_qp);

// Populations of density P (at the system's matrix offset) into the shell,
// dipole and quadrupole arrays; with want_trace, also returns Tr(P H0)
// (block-wide).  part: shared memory of kMullThreads / cw * 10 * n doubles.
__device__ __forceinline__ double mulliken_pass(const SccArgs& a, int s, const double* Pbase,
                                                bool want_trace, double* part, double* red,
                                                double* out_sh, double* out_dip, double* out_qp) {
  const DevTopo& t = a.t;
  const int n = t.nao[s];
  const int64_t mo = t.mat_off[s];
  const int cw = min(kMullThreads, (n + 31) & ~31);   // threads per row chunk
  const int rp = kMullThreads / cw;                    // row chunks
  const int chunk = threadIdx.x / cw, col0 = threadIdx.x - chunk * cw;
  const int rows = (n + rp - 1) / rp;
  const int r0 = min(n, chunk * rows), r1 = min(n, r0 + rows);
  double ph = 0.0;
  if (chunk < rp) {
    for (int col = col0; col < n; col += cw) {
      double v[10];
#pragma unroll
      for (int c = 0; c < 10; ++c) v[c] = 0.0;
      for (int r = r0; r < r1; ++r) {
        const int64_t idx = mo + (int64_t)r * n + col;
        const double pv = Pbase[idx];
        v[0] = fma(pv, a.S[idx], v[0]);
        if (want_trace) ph = fma(pv, a.H0[idx], ph);
#pragma unroll
        for (int c = 0; c < 3; ++c) v[1 + c] = fma(pv, a.D[c * a.total_mat + idx], v[1 + c]);
#pragma unroll
        for (int c = 0; c < 6; ++c) v[4 + c] = fma(pv, a.Q[c * a.total_mat + idx], v[4 + c]);
      }
      double* dst = part + (int64_t)chunk * 10 * n;
#pragma unroll
      for (int c = 0; c < 10; ++c) dst[c * n + col] = v[c];
    }
  }
  const double eb = block_sum(ph, red);   // includes the barrier before the sums below
  // column totals over the chunks (in chunk order), into chunk 0's slots
  for (int idx = threadIdx.x; idx < 10 * n; idx += blockDim.x) {
    double v = part[idx];
    for (int q = 1; q < rp; ++q) v += part[(int64_t)q * 10 * n + idx];
    part[idx] = v;
  }
  __syncthreads();
  mulliken_reduce(a, s, part, out_sh, out_dip, out_qp);
  return eb;
}

// Latency form for few systems: CTA (p, i) sums rows [p rows, (p+1) rows) of
// system i's P S, P D and P Q columns (and of P_alpha - P_beta for
// unrestricted systems) plus its share of Tr(P H0) into the system's
// workspace; k_mulliken_combine adds the parts in part order.
__global__ void __launch_bounds__(256) k_mulliken_part(SccArgs a, int parts) {
  __shared__ double red[33];
  const DevTopo& t = a.t;
  const int s = a.list[blockIdx.y];
  const int p = blockIdx.x;
  const int n = t.nao[s];
  const int64_t mo = t.mat_off[s];
  const int rows = (n + parts - 1) / parts;
  const int r0 = min(n, p * rows), r1 = min(n, r0 + rows);
  const int npass = t.nch[s] == 2 ? 2 : 1;
  for (int pass = 0; pass < npass; ++pass) {
    const double* Pb = pass == 0 ? a.P : a.Pm;
    double* out = a.work + a.work_off[s] + (int64_t)pass * (parts * 10 * (int64_t)n + parts);
    double ph = 0.0;
    for (int col = threadIdx.x; col < n; col += blockDim.x) {
      double v[10];
#pragma unroll
      for (int c = 0; c < 10; ++c) v[c] = 0.0;
      for (int r = r0; r < r1; ++r) {
        const int64_t idx = mo + (int64_t)r * n + col;
        const double pv = Pb[idx];
        v[0] = fma(pv, a.S[idx], v[0]);
        if (pass == 0) ph = fma(pv, a.H0[idx], ph);
#pragma unroll
        for (int c = 0; c < 3; ++c) v[1 + c] = fma(pv, a.D[c * a.total_mat + idx], v[1 + c]);
#pragma unroll
        for (int c = 0; c < 6; ++c) v[4 + c] = fma(pv, a.Q[c * a.total_mat + idx], v[4 + c]);
      }
#pragma unroll
      for (int c = 0; c < 10; ++c) out[((int64_t)p * 10 + c) * n + col] = v[c];
    }
    if (pass == 0) {
      ph = block_sum(ph, red);
      if (threadIdx.x == 0) out[(int64_t)parts * 10 * n + p] = ph;
    }
  }
}

__global__ void __launch_bounds__(kMullThreads) k_mulliken_combine(SccArgs a, int parts) {
  extern __shared__ double sm[];   // 10 n
  const DevTopo& t = a.t;
  const int s = a.list[blockIdx.x];
  const int n = t.nao[s];
  const int npass = t.nch[s] == 2 ? 2 : 1;
  for (int pass = 0; pass < npass; ++pass) {
    const double* in = a.work + a.work_off[s] + (int64_t)pass * (parts * 10 * (int64_t)n + parts);
    for (int idx = threadIdx.x; idx < 10 * n; idx += blockDim.x) {
      double v = in[idx];
      for (int q = 1; q < parts; ++q) v += in[(int64_t)q * 10 * n + idx];
      sm[idx] = v;
    }
    if (pass == 0 && threadIdx.x == 0) {
      double eb = 0.0;
      for (int q = 0; q < parts; ++q) eb += in[(int64_t)parts * 10 * n + q];
      a.e_core[s] = eb;
    }
    __syncthreads();
    if (pass == 0) mulliken_reduce(a, s, sm, a.pop_sh, a.pop_dip, a.pop_qp);
    else mulliken_reduce(a, s, sm, a.pop_mag, a.pop_mdip, a.pop_mqp);
    __syncthreads();
  }
}

// Shell, dipole and quadrupole populations from the column totals part[c n + col].
__device__ void mulliken_reduce(const SccArgs& a, int s, const double* part, double* out_sh,
                                double* out_dip, double* out_qp) {
  const DevTopo& t = a.t;
  const int n = t.nao[s];
  const int64_t s0 = t.shell_off[s], s1 = t.shell_off[s + 1];
  for (int64_t sh = s0 + threadIdx.x; sh < s1; sh += blockDim.x) {
    const int first = t.sh_ao[sh], cnt = 2 * t.sh_l[sh] + 1;
    double v = 0.0;
    for (int k = 0; k < cnt; ++k) v += part[first + k];
    out_sh[sh] = v;
  }
  const int64_t a0 = t.atom_off[s], a1 = t.atom_off[s + 1];
  for (int64_t at = a0 + threadIdx.x; at < a1; at += blockDim.x) {
    double pd[3] = {0, 0, 0}, pq[6] = {0, 0, 0, 0, 0, 0};
    for (int sh = t.atom_sh[at]; sh < t.atom_sh[at + 1]; ++sh) {
      const int first = t.sh_ao[sh], cnt = 2 * t.sh_l[sh] + 1;
      for (int k = 0; k < cnt; ++k) {
        for (int c = 0; c < 3; ++c) pd[c] += part[(1 + c) * n + first + k];
        for (int c = 0; c < 6; ++c) pq[c] += part[(4 + c) * n + first + k];
      }
    }
    for (int c = 0; c < 3; ++c) out_dip[3 * at + c] = pd[c];
    for (int c = 0; c < 6; ++c) out_qp[6 * at + c] = pq[c];
  }
  __syncthreads();   // part is reused by a second pass
}

// One CTA per system.  The n rows are cut into fixed chunks; thread
// (chunk, column) sums its column over its chunk, and the chunks, shells,
// atoms and the trace are then added in a fixed order, so the populations are
// the same in every run.  Unrestricted systems also get the magnetisation
// populations of P_alpha - P_beta.
__global__ void __launch_bounds__(kMullThreads) k_mulliken(SccArgs a) {
  extern __shared__ double sm[];
  __shared__ double red[33];
  const int s = a.list[blockIdx.x];
  const double eb = mulliken_pass(a, s, a.P, true, sm, red, a.pop_sh, a.pop_dip, a.pop_qp);
  if (threadIdx.x == 0) a.e_core[s] = eb;
  if (a.t.nch[s] == 2)
    mulliken_pass(a, s, a.Pm, false, sm, red, a.pop_mag, a.pop_mdip, a.pop_mqp);
}

void launch_mulliken(const SccArgs& a, int max_n, cudaStream_t stream) {
  if (a.count == 0) return;
  // Few systems: each system's rows over several CTAs (one SM alone cannot
  // stream the 11 n^2 doubles fast enough); the workspace holds 16 parts of
  // two passes (2 (160 n + 16) doubles, within its 640 n).
  const int parts = std::min(16, 2 * sm_count() / a.count);
  if (parts >= 2 && a.work != nullptr) {
    const size_t attr_c = allow_max_dynamic_smem(k_mulliken_combine);
    (void)attr_c;
    k_mulliken_part<<<dim3(parts, a.count), 256, 0, stream>>>(a, parts);
    k_mulliken_combine<<<a.count, kMullThreads, (size_t)10 * max_n * sizeof(double), stream>>>(a, parts);
    return;
  }
  // rp(n) * 10 * n doubles: rp * n <= rp * cw = kMullThreads while n <= kMullThreads
  const size_t words = (size_t)10 * std::max(kMullThreads, max_n);
  const size_t attr = allow_max_dynamic_smem(k_mulliken);
  (void)attr;
  k_mulliken<<<a.count, kMullThreads, words * sizeof(double), stream>>>(a);
}

// ---------------------------------------------------------------------------
// Energy functional from the raw populations, Broyden mixing, convergence.
// ---------------------------------------------------------------------------
__device__ bool cholesky_solve_small(double* B, double* c, int n) {
  for (int r = 0; r < n; ++r) {
    for (int col = 0; col <= r; ++col) {
      double v = B[r * 8 + col];
      for (int k = 0; k < col; ++k) v -= B[r * 8 + k] * B[col * 8 + k];
      if (r == col) {
        if (!(v > 0.0)) return false;
        B[r * 8 + col] = sqrt(v);
      } else {
        B[r * 8 + col] = v / B[col * 8 + col];
      }
    }
  }
  for (int r = 0; r < n; ++r) {
    double v = c[r];
    for (int k = 0; k < r; ++k) v -= B[r * 8 + k] * c[k];
    c[r] = v / B[r * 8 + r];
  }
  for (int r = n - 1; r >= 0; --r) {
    double v = c[r];
    for (int k = r + 1; k < n; ++k) v -= B[k * 8 + r] * c[k];
    c[r] = v / B[r * 8 + r];
  }
  return true;
}

__global__ void __launch_bounds__(256) k_energy_mixer(SccArgs a) {
  extern __shared__ double sm[];
  const DevTopo& t = a.t;
  const int s = a.list[blockIdx.x];
  const int64_t a0 = t.atom_off[s];
  const int na = (int)(t.atom_off[s + 1] - a0);
  const int64_t s0 = t.shell_off[s];
  const int ns = (int)(t.shell_off[s + 1] - s0);
  const int d1 = charge_block(t, ns, na);   // charge block
  const bool mp = !t.m.gfn1;                // atomic multipoles in the mixed vector (GFN2)
  const bool uhf = t.nch[s] == 2;
  const int dim = uhf ? 2 * d1 : d1;
  double* raw = sm;                       // dim: [qsh, dip (3na), qp (6na)] (+ the same for m)
  double* qat = raw + dim;                // na
  double* w = qat + na;                   // 7 na
  double* red = w + kMaxD4Refs * na;      // 64 + 8*64
  const int tid = threadIdx.x, bs = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = bs >> 5;
  for (int i = tid; i < ns; i += bs) raw[i] = t.sh_refocc[s0 + i] - a.pop_sh[s0 + i];
  if (mp) {
    for (int i = tid; i < 3 * na; i += bs) raw[ns + i] = -a.pop_dip[3 * a0 + i];
    for (int i = tid; i < 6 * na; i += bs) raw[ns + 3 * na + i] = -a.pop_qp[6 * a0 + i];
  }
  if (uhf) {
    // magnetisation m = pop_beta - pop_alpha (the charge-like sign of the populations)
    for (int i = tid; i < ns; i += bs) raw[d1 + i] = -a.pop_mag[s0 + i];
    if (mp) {
      for (int i = tid; i < 3 * na; i += bs) raw[d1 + ns + i] = -a.pop_mdip[3 * a0 + i];
      for (int i = tid; i < 6 * na; i += bs) raw[d1 + ns + 3 * na + i] = -a.pop_mqp[6 * a0 + i];
    }
  }
  __syncthreads();
  for (int i = tid; i < na; i += bs) {
    const int64_t g = a0 + i;
    double q = 0.0;
    for (int sh = t.atom_sh[g]; sh < t.atom_sh[g + 1]; ++sh) q += raw[sh - s0];
    qat[i] = q;
    if (mp) d4_weights(t, t.Z[g], a.cn_d4[g], q, w + kMaxD4Refs * i, nullptr, nullptr);
  }
  __syncthreads();
  // ES2 and ES3: thread j forms (gamma q)_j down column j of the symmetric
  // gamma (coalesced rows, independent loads)
  double e2 = 0.0, e3 = 0.0, ea = 0.0, ed = 0.0;
  const double* gam = a.gam + t.gam_off[s];
  for (int j = tid; j < ns; j += bs) {
    const double acc = gamma_column_dot(gam, ns, j, raw);
    const double q = raw[j];
    e2 += 0.5 * q * acc;
    if (!t.m.gfn1) e3 += t.sh_g3[s0 + j] * q * q * q / 3.0;
  }
  // GFN1: atom-resolved third order Gamma_A q_A^3 / 3 (model/gfn1/es3.cpp:115-125)
  if (t.m.gfn1)
    for (int i = tid; i < na; i += bs) {
      const double q = qat[i];
      e3 += t.sh_g3[t.atom_sh[a0 + i]] * q * q * q / 3.0;
    }
  // AES2 onsite (GFN2 only: the loops below run for GFN1 with no multipoles)
  const double* rd = raw + ns;
  const double* rq = raw + ns + 3 * na;
  const double scl[6] = {1.0, 2.0, 1.0, 2.0, 2.0, 1.0};
  for (int i = tid; i < (mp ? na : 0); i += bs) {
    const int64_t g = a0 + i;
    double d2 = 0.0, q2 = 0.0;
    for (int c = 0; c < 3; ++c) d2 += rd[3 * i + c] * rd[3 * i + c];
    for (int c = 0; c < 6; ++c) q2 += scl[c] * rq[6 * i + c] * rq[6 * i + c];
    ea += t.at_dk[g] * d2 + t.at_qk[g] * q2;
  }
  // pairs: AES2 and D4 two-body
  const int64_t npair = mp ? (int64_t)na * (na - 1) / 2 : 0;
  for (int64_t p = tid; p < npair; p += bs) {
    int64_t si, fi;
    pair_from_index(p, si, fi);
    const int f = (int)fi, sc = (int)si;
    const int64_t gf = a0 + f, gs = a0 + sc;
    const double d[3] = {t.pos[3 * gf] - t.pos[3 * gs], t.pos[3 * gf + 1] - t.pos[3 * gs + 1],
                         t.pos[3 * gf + 2] - t.pos[3 * gs + 2]};
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double r = sqrt(r2);
    double k3, k5;
    aes2_kernels(r, 0.5 * (a.mrad[gf] + a.mrad[gs]), k3, k5);
    const double* df = rd + 3 * f;
    const double* ds = rd + 3 * sc;
    double pf = 0.0, ps = 0.0, dd = 0.0, cdn = 0.0;
    for (int c = 0; c < 3; ++c) {
      pf += d[c] * df[c];
      ps += d[c] * ds[c];
      dd += df[c] * ds[c];
      cdn += d[c] * (qat[f] * ds[c] - qat[sc] * df[c]);
    }
    const double sqv[6] = {d[0] * d[0] * k5, 2.0 * d[0] * d[1] * k5, d[1] * d[1] * k5,
                           2.0 * d[0] * d[2] * k5, 2.0 * d[1] * d[2] * k5, d[2] * d[2] * k5};
    double tq = 0.0;
    for (int c = 0; c < 6; ++c) tq += qat[f] * sqv[c] * rq[6 * sc + c] + qat[sc] * sqv[c] * rq[6 * f + c];
    ea += k3 * cdn + k5 * (r2 * dd - 3.0 * pf * ps) + tq;
    double damp, ddamp;
    const int zf = t.Z[gf], zs = t.Z[gs];
    d4_pair_damping(t, zf, zs, r2, damp, ddamp);
    if (damp != 0.0) {
      ed -= d4_c6(t, zf, zs, w + kMaxD4Refs * f, w + kMaxD4Refs * sc, nullptr, nullptr, nullptr,
                  nullptr) * damp;
    }
  }
  // uniform field: E_field = sum_A q_A (-E.R_A) + (-E).d_A (raw charges and
  // dipoles; scc_driver.cpp:2212-2232 of the reference)
  double ef = 0.0;
  if (t.efield != nullptr) {
    const double* E = t.efield + 3 * s;
    for (int i = tid; i < na; i += bs) {
      const int64_t g = a0 + i;
      const double vat = -(E[0] * t.pos[3 * g] + E[1] * t.pos[3 * g + 1] + E[2] * t.pos[3 * g + 2]);
      double c = vat * qat[i];
      for (int k = 0; k < 3; ++k) c = fma(-E[k], rd[3 * i + k], c);
      ef += c;
    }
  }
  // charge response: E = q.b + q^T A q / 2 (raw charges)
  double er = 0.0;
  if (t.resp_A != nullptr) {
    const double* A = t.resp_A + t.resp_off[s];
    for (int i = tid; i < na; i += bs) {
      double aq = 0.0;
      for (int j = 0; j < na; ++j) aq = fma(A[(int64_t)i * na + j], qat[j], aq);
      er += qat[i] * (t.resp_b[a0 + i] + 0.5 * aq);
    }
  }
  // spin polarisation: E_spin = 1/2 sum_A m_A^T W_A m_A (raw magnetisation)
  double es = 0.0;
  if (uhf) {
    for (int i = tid; i < ns; i += bs) {
      const int64_t sh = s0 + i;
      const int at = t.sh_atom[sh];
      const int f0 = t.atom_sh[at] - (int)s0, cnt = t.atom_sh[at + 1] - t.atom_sh[at];
      double v = 0.0;
      for (int k = 0; k < cnt; ++k) v = fma(t.sh_spinw[3 * sh + k], raw[d1 + f0 + k], v);
      es = fma(0.5 * raw[d1 + i], v, es);
    }
  }
  // external point charges: E_pc = sum_s q_s V_s (potential fixed by the geometry)
  double ep = 0.0;
  if (t.vpc != nullptr)
    for (int i = tid; i < ns; i += bs) ep += raw[i] * t.vpc[s0 + i];
  e2 = block_sum(e2, red);
  e3 = block_sum(e3, red);
  ea = block_sum(ea, red);
  ed = block_sum(ed, red);
  ep = block_sum(ep, red);
  es = block_sum(es, red);
  ef = block_sum(ef, red);
  er = block_sum(er, red);
  const double ecore = a.e_core[s];
  const int bch = t.beta_ch[s];
  const double ts = -a.kt * (a.entropy[s] + (bch >= 0 ? a.entropy[bch] : 0.0));
  const double F = ecore + e2 + e3 + ea + ed + ep + es + ef + er + ts;

  // ---- modified Broyden (Johnson) ----
  const int64_t v0 = t.vec_off[s];
  const int M = a.memory;
  double* cur = a.mx_cur + v0;
  double* prv = a.mx_prev + v0;
  double* pres = a.mx_res + v0;
  double* dfh = a.mx_df + v0 * M;
  double* uh = a.mx_u + v0 * M;
  double* om = a.mx_omega + (int64_t)s * M;
  const int it = a.iterations[s];
  // residual norm
  double r2p = 0.0;
  for (int i = tid; i < dim; i += bs) {
    const double r = raw[i] - cur[i];
    r2p += r * r;
  }
  const double nrm = sqrt(block_sum(r2p, red));
  const double rms = nrm / sqrt((double)dim);
  __shared__ double s_c[8];
  __shared__ int s_hc, s_ok;
  int hc = 0;
  if (it > 0) {
    double f2p = 0.0;
    for (int i = tid; i < dim; i += bs) {
      const double r = raw[i] - cur[i];
      const double df = r - pres[i];
      f2p += df * df;
    }
    const double inv = 1.0 / fmax(sqrt(block_sum(f2p, red)), DBL_EPSILON);
    const double omega = nrm > 0.01 / 100000.0 ? fmax(1.0, 0.01 / nrm) : 100000.0;
    hc = min(M, it);
    const int new_slot = (it - 1) % M;
    for (int i = tid; i < dim; i += bs) {
      const double r = raw[i] - cur[i];
      const double df = (r - pres[i]) * inv;
      dfh[(int64_t)new_slot * dim + i] = df;
      uh[(int64_t)new_slot * dim + i] = a.damping * df + inv * (cur[i] - prv[i]);
    }
    if (tid == 0) om[new_slot] = omega;
    __syncthreads();
    // dot products: c_h = df_h . res, B_hk = df_h . df_k
    const int first = it - hc + 1;
    int slot[8];
    for (int h = 0; h < 8; ++h) slot[h] = (h < hc) ? (first + h - 1) % M : 0;
    double part[8 + 36];
    for (int q = 0; q < 44; ++q) part[q] = 0.0;
    for (int i = tid; i < dim; i += bs) {
      const double r = raw[i] - cur[i];
      double dv[8];
#pragma unroll
      for (int h = 0; h < 8; ++h) dv[h] = (h < hc) ? dfh[(int64_t)slot[h] * dim + i] : 0.0;
      int q = 8;
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        part[h] += dv[h] * r;
#pragma unroll
        for (int k = 0; k <= h; ++k) part[q++] += dv[h] * dv[k];
      }
    }
    double* wsum = red + 64;   // [nw][44], then the 44 totals
#pragma unroll
    for (int q = 0; q < 44; ++q) {
      const double v = warp_sum(part[q]);
      if (lane == 0) wsum[warp * 44 + q] = v;
    }
    __syncthreads();
    double* totals = red;      // the block sums above are done with red[0..32]
    if (tid < 44) {
      double v = 0.0;
      for (int ww = 0; ww < nw; ++ww) v += wsum[ww * 44 + tid];
      totals[tid] = v;
    }
    __syncthreads();
    if (tid == 0) {
      double tot[44];
      for (int q = 0; q < 44; ++q) tot[q] = totals[q];
      double B[64], c[8];
      int q = 8;
      for (int h = 0; h < 8; ++h) {
        for (int k = 0; k <= h; ++k) {
          if (h < hc && k < hc) {
            const double val = om[slot[h]] * om[slot[k]] * tot[q] + (h == k ? 1e-4 : 0.0);
            B[h * 8 + k] = val;
            B[k * 8 + h] = val;
          }
          ++q;
        }
        if (h < hc) c[h] = om[slot[h]] * tot[h];
      }
      const bool ok = cholesky_solve_small(B, c, hc);
      for (int h = 0; h < 8; ++h) s_c[h] = (h < hc) ? om[slot[h]] * c[h] : 0.0;
      s_ok = ok ? 1 : 0;
      s_hc = hc;
    }
    __syncthreads();
    hc = s_hc;
    if (!s_ok) hc = -1;
  }
  // mixed = cur + damp * res - sum_h omega_h c_h u_h ; shift history
  const double Fold = (it == 0) ? 0.0 : a.free_energy[s];
  const bool exact = a.prec == nullptr || a.prec[s] != 0;   // this iteration ran in FP64
  // The split-precision form reaches the fixed point on another trajectory
  // than the FP64 form, so stopping anywhere inside the gate would leave it
  // as far from the FP64 result as the gate allows (charges ~1e-5 apart):
  // its FP64 iterations continue to a gate kMixedTighten times tighter, so
  // that its result is the fixed point itself.  A system that meets the
  // ordinary gate but not the tighter one within kMixedExtra FP64 iterations
  // (or by the last iteration) stops on the ordinary gate.
  const bool gate = (rms < a.ctol) && (fabs(F - Fold) < a.etol) && hc >= 0 && exact;
  const bool tight = a.prec == nullptr ||
                     ((rms < a.ctol * kMixedTighten) && (fabs(F - Fold) < a.etol * kMixedTighten));
  const int hits = (a.gate_hits != nullptr && gate) ? a.gate_hits[s] + 1 : 0;
  const bool conv = gate && (tight || hits > kMixedExtra || it + 1 >= a.max_iter);
  const bool failed = hc < 0 || !isfinite(F) || !isfinite(nrm);
  const int first = it - (hc > 0 ? hc : 0) + 1;
  for (int i = tid; i < dim; i += bs) {
    const double r = raw[i] - cur[i];
    double mixed = cur[i] + a.damping * r;
    for (int h = 0; h < hc; ++h) {
      const int sl = (first + h - 1) % M;
      mixed -= s_c[h] * uh[(int64_t)sl * dim + i];
    }
    prv[i] = cur[i];
    pres[i] = r;
    cur[i] = mixed;
    const double out = conv ? raw[i] : mixed;
    if (i < ns) {
      a.qsh[s0 + i] = out;
    } else if (i < d1) {   // atomic multipoles (GFN2 only: for GFN1 d1 == ns)
      if (i < ns + 3 * na) a.dip[3 * a0 + (i - ns)] = out;
      else a.qp[6 * a0 + (i - ns - 3 * na)] = out;
    } else if (i < d1 + ns) {
      a.qmag[s0 + (i - d1)] = out;   // magnetisation multipoles live only in the mixer state
    }
  }
  if (tid == 0) {
    a.free_energy[s] = F;
    a.iterations[s] = it + 1;
    double* tm = a.terms + kTermCount * (int64_t)s;
    tm[kTermCore] = ecore;
    tm[kTermEs2] = e2;
    tm[kTermEs3] = e3;
    tm[kTermAes2] = ea;
    tm[kTermD4] = ed;
    tm[kTermEntropy] = ts;
    tm[kTermPc] = ep;
    tm[kTermSpin] = es;
    tm[kTermField] = ef;
    tm[kTermResp] = er;
    if (!exact) {
      a.split_iters[s] += 1;
      // switch once the residual is small, or when split-precision
      // iterations stop making progress (a residual stuck above the switch)
      if (rms < a.prec_switch || a.split_iters[s] >= kMaxSplitIterations) a.prec[s] = 1;
    }
    if (a.gate_hits != nullptr && gate) a.gate_hits[s] = hits;
    if (a.last_rms != nullptr) a.last_rms[s] = rms;
    if (failed) {
      a.status[s] = kInternal;
    } else if (conv) {
      a.converged[s] = 1;
    } else if (it + 1 >= a.max_iter) {
      a.status[s] = kNotConverged;
    }
  }
}

void launch_energy_mixer(const SccArgs& a, int max_atoms, int max_shells, int max_dim,
                         int first_iteration, cudaStream_t stream) {
  (void)first_iteration;
  if (a.count == 0) return;
  const size_t sm = ((size_t)max_dim + (1 + kMaxD4Refs) * max_atoms + 64 + 8 * 44 + 8) * sizeof(double);
  const size_t attr = allow_max_dynamic_smem(k_energy_mixer);
  (void)attr;
  k_energy_mixer<<<a.count, 256, sm, stream>>>(a);
}

// ---------------------------------------------------------------------------
// Active-list compaction in the (cost-descending) system order.
// ---------------------------------------------------------------------------
__global__ void k_compact(const int32_t* order, int nsys, const int32_t* status,
                          const uint8_t* converged, const int32_t* iterations, int max_iter,
                          int32_t* list, int32_t* count) {
  __shared__ int wtot[32];
  __shared__ int base, chunk_total;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c0 = 0; c0 < nsys; c0 += blockDim.x) {
    const int i = c0 + threadIdx.x;
    int sys = -1;
    bool act = false;
    if (i < nsys) {
      sys = order[i];
      act = status[sys] == kOk && converged[sys] == 0 && iterations[sys] < max_iter;
    }
    const unsigned b = __ballot_sync(0xffffffffu, act);
    const int pre = __popc(b & ((1u << lane) - 1u));
    if (lane == 0) wtot[warp] = __popc(b);
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        const int v = wtot[w];
        wtot[w] = acc;
        acc += v;
      }
      chunk_total = acc;
    }
    __syncthreads();
    if (act) list[base + wtot[warp] + pre] = sys;
    __syncthreads();
    if (threadIdx.x == 0) base += chunk_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) count[0] = base;
}

void launch_compact(const int32_t* order, int nsys, const int32_t* status, const uint8_t* converged,
                    const int32_t* iterations, int max_iter, int32_t* list, int32_t* count,
                    cudaStream_t stream) {
  k_compact<<<1, 1024, 0, stream>>>(order, nsys, status, converged, iterations, max_iter, list, count);
}

}  // namespace xtb
