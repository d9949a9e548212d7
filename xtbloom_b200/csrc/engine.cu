// Host orchestration of the batched GFN2-xTB path on one B200.
//
// Per call: validate and stage the ragged batch, build (or reuse) the
// topology on the device, run the geometry setup kernels, build the Loewdin
// orthogonaliser, iterate the SCC with an on-device active list (systems
// leave the launch grid as soon as they converge; the list is ordered by
// decreasing AO count so the largest systems start first), evaluate the
// analytic gradient, and publish into the caller's buffers with quiet-NaN
// slices for failed systems.  Mirrors the reference's CUDA execution flow
// (runtime/gfn2_cuda_execution.cu:8784-10424) with a different kernel design.
#include "engine.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>

#include "kernels.cuh"

namespace xtb {
namespace {

#include "generated/params.inc"

constexpr double kEvToHartree = 1.0 / 27.21138505;
constexpr double kAngstromToBohr = 1.8897261246204404;
constexpr double kPiH = 3.141592653589793238462643383279502884;

// Device bytes held by the engine whose method runs on this thread (the
// workspace a fixed-topology plan reports).
thread_local int64_t* t_ledger = nullptr;

struct Dbuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~Dbuf() {
    if (p) cudaFree(p);
  }
  bool reserve(size_t nbytes) {
    if (nbytes <= bytes && p) return true;
    if (p) cudaFree(p);
    if (t_ledger) *t_ledger -= (int64_t)bytes;
    p = nullptr;
    bytes = 0;
    const size_t want = std::max<size_t>(nbytes, 256);
    if (cudaMalloc(&p, want) != cudaSuccess) return false;
    bytes = want;
    if (t_ledger) *t_ledger += (int64_t)bytes;
    return true;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

template <class T>
bool upload(Dbuf& b, const std::vector<T>& v, cudaStream_t s) {
  if (!b.reserve(v.size() * sizeof(T))) return false;
  if (!v.empty()) cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
  return true;
}

// STO-nG expansion (common/sto.cpp:20-123 of the reference, restated).
bool sto_expand(int n, int l, int ng, double zeta, std::vector<double>& alpha,
                std::vector<double>& coeff) {
  const double* a0 = nullptr;
  const double* c0 = nullptr;
  if (n == 6 && ng == 6) {
    a0 = l == 0 ? kP_sto_alpha6s : kP_sto_alpha6p;
    c0 = l == 0 ? kP_sto_coeff6s : kP_sto_coeff6p;
  } else {
    int typ;
    switch (l) {
      case 0: typ = n - 1; break;
      case 1: typ = n + 3; break;
      case 2: typ = n + 6; break;
      case 3: typ = n + 8; break;
      default: typ = n + 9; break;
    }
    if (typ < 0 || typ >= 15) return false;
    if (ng == 3) { a0 = kP_sto_alpha3 + 3 * typ; c0 = kP_sto_coeff3 + 3 * typ; }
    else if (ng == 4) { a0 = kP_sto_alpha4 + 4 * typ; c0 = kP_sto_coeff4 + 4 * typ; }
    else if (ng == 6) { a0 = kP_sto_alpha6 + 6 * typ; c0 = kP_sto_coeff6 + 6 * typ; }
    else return false;
  }
  const double dfact[5] = {1.0, 1.0, 3.0, 15.0, 105.0};
  alpha.resize(ng);
  coeff.resize(ng);
  for (int i = 0; i < ng; ++i) {
    alpha[i] = a0[i] * zeta * zeta;
    const double norm = std::pow(2.0 / kPiH * alpha[i], 0.75) * std::pow(std::sqrt(4.0 * alpha[i]), l) /
                        std::sqrt(dfact[l]);
    coeff[i] = c0[i] * norm;
  }
  return true;
}

// GFN1 keeps xTB's legacy STO-6G rows for 4s and 4p shells (one exponent
// row, two coefficient rows; model/gfn1/basis.cpp:64-90); every other shell
// is the common Stewart expansion.
bool sto_expand_gfn1(int n, int l, int ng, double zeta, std::vector<double>& alpha,
                     std::vector<double>& coeff) {
  if (!(ng == 6 && n == 4 && l <= 1)) return sto_expand(n, l, ng, zeta, alpha, coeff);
  const double* c0 = l == 0 ? kP_gfn1_sto6_4sp_coeff_s : kP_gfn1_sto6_4sp_coeff_p;
  alpha.resize(6);
  coeff.resize(6);
  for (int i = 0; i < 6; ++i) {
    alpha[i] = kP_gfn1_sto6_4sp_alpha[i] * zeta * zeta;
    const double norm = std::pow(2.0 / kPiH * alpha[i], 0.75) * std::pow(std::sqrt(4.0 * alpha[i]), l);
    coeff[i] = c0[i] * norm;
  }
  return true;
}

void orthogonalize_to_first(const std::vector<double>& a1, const std::vector<double>& c1,
                            std::vector<double>& a, std::vector<double>& c) {
  double ov = 0.0;
  for (size_t i = 0; i < a1.size(); ++i)
    for (size_t j = 0; j < a.size(); ++j) ov += c1[i] * c[j] * std::pow(std::sqrt(kPiH / (a1[i] + a[j])), 3.0);
  const size_t nb = a.size();
  for (size_t i = 0; i < a1.size(); ++i) {
    a.push_back(a1[i]);
    c.push_back(-ov * c1[i]);
  }
  double nrm = 0.0;
  for (size_t i = 0; i < a.size(); ++i)
    for (size_t j = 0; j < a.size(); ++j) nrm += c[i] * c[j] * std::pow(std::sqrt(kPiH / (a[i] + a[j])), 3.0);
  (void)nb;
  const double inv = 1.0 / std::sqrt(nrm);
  for (double& x : c) x *= inv;
}

const char* kGlobalNames[20] = {"wexp", "enscale", "kpol", "pair_scale_default", "rep_kexp",
                                "rep_klight", "es3_s", "es3_p", "es3_d", "mp_dmp3", "mp_dmp5",
                                "mp_kexp", "mp_shift", "mp_rmax", "d4_a1", "d4_a2", "d4_s6",
                                "d4_s8", "d4_s9", "es2_gexp"};

ModelConstants make_constants() {
  ModelConstants m{};
  const double* g = kP_gfn2_globals;
  m.wexp = g[0];
  m.enscale = g[1];
  m.kpol = g[2];
  m.pair_scale_default = g[3];
  for (int i = 0; i < 9; ++i) m.shell_pair_scale[i] = kP_gfn2_shell_pair_scale[i];
  m.rep_kexp = g[4];
  m.rep_klight = g[5];
  m.es3_scale[0] = g[6];
  m.es3_scale[1] = g[7];
  m.es3_scale[2] = g[8];
  m.mp_kexp = g[11];
  m.mp_shift = g[12];
  m.mp_rmax = g[13];
  m.d4_a1 = g[14];
  m.d4_a2 = g[15];
  m.d4_s6 = g[16];
  m.d4_s8 = g[17];
  m.d4_s9 = g[18];
  (void)kGlobalNames;
  return m;
}

// GFN1-xTB constants (tblite export, data/parameters/gfn1.json).
ModelConstants make_constants_gfn1() {
  ModelConstants m{};
  const double* g = kP_gfn1_globals;   // kpol, enscale, rep kexp/klight, d3 a1 a2 s6 s8 s9,
                                       // xb damping, radius scale, CN steepness, cutoff, gexp
  m.gfn1 = 1;
  m.wexp = 0.0;
  m.kpol = g[0];
  m.enscale = g[1];
  m.pair_scale_default = 1.0;
  for (int i = 0; i < 9; ++i) m.shell_pair_scale[i] = kP_gfn1_shell_pair_scale[i];
  m.rep_kexp = g[2];
  m.rep_klight = g[3];
  m.es3_scale[0] = m.es3_scale[1] = m.es3_scale[2] = 1.0;
  m.d3_a1 = g[4];
  m.d3_a2 = g[5];
  m.d3_s6 = g[6];
  m.d3_s8 = g[7];
  m.xb_damping = g[9];
  m.xb_radius_scale = g[10];
  m.cn_steepness = g[11];
  return m;
}

// Optional live kernel timing with CUDA events on the engine stream, grouped
// by pipeline stage; enabled with XTBLOOM_B200_KERNEL_TIMING=1.
enum Stage : int {
  kStSetup, kStLowdin, kStPotential, kStFock, kStTransform, kStTridiag, kStEigvals, kStInvIter,
  kStBacktransform, kStDensity, kStMulliken, kStEnergyMixer, kStCompact, kStForcePairs,
  kStClassical, kStCnChain, kStPublish, kStRefine, kStageCount
};
[[maybe_unused]] const char* kStageNames[kStageCount] = {
    "setup_integrals", "lowdin", "potential", "fock", "gemm_transform", "tridiag", "eigvals",
    "inverse_iteration", "backtransform", "gemm_density", "mulliken", "energy_mixer", "compact",
    "force_pairs", "classical", "cn_chain", "publish", "refine"};

struct Profiler {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  std::vector<std::pair<int, size_t>> marks;   // stage, index of start event (end = +1)
  double total_ms[kStageCount] = {};
  int64_t calls[kStageCount] = {};
  int64_t launches = 0;
  cudaEvent_t next() {
    if (used == pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[used++];
  }
  void begin(int stage, cudaStream_t s) {
    if (!on) return;
    marks.push_back({stage, used});
    cudaEventRecord(next(), s);
  }
  void end(cudaStream_t s) {
    if (!on) return;
    cudaEventRecord(next(), s);
  }
  void collect() {
    for (auto& m : marks) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, pool[m.second], pool[m.second + 1]);
      total_ms[m.first] += ms;
      calls[m.first] += 1;
    }
    marks.clear();
    used = 0;
  }
  ~Profiler() {
    for (auto e : pool) cudaEventDestroy(e);
  }
};

}  // namespace

struct Engine::Impl {
  ModelConstants model = make_constants();   // the model of the current topology
  const ModelConstants model_gfn2 = make_constants();
  const ModelConstants model_gfn1 = make_constants_gfn1();
  // GFN1 tables: element-pair H0 scale, D3 references
  Dbuf kpair, d3_rcnt, d3_roff, d3_ref_cn, d3_c6, d3_r4r2;
  // static parameter tables on the device
  Dbuf d4_rcov, d4_en, d4_zeff, d4_eta, d4_r4r2, d4_roff, d4_rcnt, ref_cn, ref_q, ref_ng, ref_c6;
  bool tables_ready = false;

  // topology (host copies used for caching and sizes)
  HostBatch topo;
  bool topo_valid = false;
  int64_t nsys = 0, natoms = 0, nshells = 0, naos = 0, total_mat = 0, total_gam = 0, total_vec = 0,
          total_scr = 0, total_prim = 0;
  int max_n = 0, max_atoms = 0, max_shells = 0, max_dim = 0;
  int64_t max_pairs = 0;
  std::vector<int32_t> h_nao, h_order;
  std::vector<double> h_nel_a, h_nel_b;

  // device topology arrays
  Dbuf atom_off, shell_off, ao_off, mat_off, gam_off, vec_off, scr_off, nao, nel_a, nel_b, qmol;
  // spin channels: id c < nsys is system c's first (restricted or alpha)
  // channel at the system's own offsets; beta channels have ids nsys + u with
  // storage after the systems' (matrices at total_mat.., vectors at naos..)
  int64_t nchan = 0, nuhf = 0, chan_mat = 0, chan_vec = 0, chan_scr = 0;
  Dbuf nch, beta_ch, sh_spinw, ch_sys, ch_sign, ch_nao, ch_mat, ch_ao, ch_scr, ch_xoff, ch_nel_a,
      ch_nel_b, clist, ccount;
  std::vector<int32_t> h_ch_nao, h_ch_sys;
  std::vector<double> h_ch_nel_a, h_ch_nel_b;
  int32_t* h_clist = nullptr;   // pinned copy of the active channel list
  int64_t h_clist_cap = 0;
  Dbuf Z, atom_sh, pos, at_en, at_rad, at_rcov, at_mprad, at_mpvcn, at_dk, at_qk, at_rep_sa, at_rep_z,
      at_xbond, sh_val;
  Dbuf sh_atom, sh_l, sh_ao, sh_p0, sh_np, sh_level, sh_kcn, sh_shpoly, sh_zeta, sh_eta, sh_g3,
      sh_refocc, p_alpha, p_coeff, ao_sh, ao_at, order;
  // state
  Dbuf list, count, status, iterations, converged, nvec;
  Dbuf cn, cn_d4, mrad, dmrad, gam;
  Dbuf S, D, Q, H0, H, X, T, A, Zv, C, P, W;
  Dbuf d, e, tau, eig, occ, occ_eps, entropy, scratch;
  Dbuf qsh, dip, qp, pop_sh, pop_dip, pop_qp, e_core, vsh, vd, vq;
  Dbuf Pm, qmag, vmag, pop_mag, pop_mdip, pop_mqp;
  Dbuf efield, out_dipoles;
  bool have_field = false;
  // FP64 GEMM tile width chosen by measurement per (product kind, orbital-count
  // bucket of 32, power-of-two class of the system count)
  std::map<uint64_t, int> gemm_width;
  int forced_gemm_width = 0;   // 32 or 64: no timing, every FP64 product at that width
  // side streams for the size buckets of the eigensolver, which run
  // concurrently (small systems fill the SMs that large ones leave free)
  static constexpr int kBucketStreams = 8;
  cudaStream_t bst[kBucketStreams] = {};
  cudaEvent_t bfork = nullptr, bjoin[kBucketStreams] = {};
  // per bucket stream: a second stream for the WY T factors, which need only
  // the reflectors and run beside the eigenvalues and the inverse iteration
  cudaStream_t fst[kBucketStreams] = {};
  cudaEvent_t ffork[kBucketStreams] = {}, wydone[kBucketStreams] = {};
  bool bstreams = false;
  bool ensure_bucket_streams() {
    if (bstreams) return true;
    if (cudaEventCreateWithFlags(&bfork, cudaEventDisableTiming) != cudaSuccess) return false;
    for (int i = 0; i < kBucketStreams; ++i)
      if (cudaStreamCreateWithFlags(&bst[i], cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&bjoin[i], cudaEventDisableTiming) != cudaSuccess ||
          cudaStreamCreateWithFlags(&fst[i], cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&ffork[i], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&wydone[i], cudaEventDisableTiming) != cudaSuccess)
        return false;
    bstreams = true;
    return true;
  }
  Dbuf resp_b, resp_A, resp_off;
  bool have_resp = false;
  Dbuf free_energy, terms;
  Dbuf mx_cur, mx_prev, mx_res, mx_df, mx_u, mx_omega;
  Dbuf grad, acn, acn_d4, pot_acc;
  Dbuf out_energy, out_forces, out_charges;
  // external point charges of the current call
  Dbuf pc_off, pc_pos, pc_q, pc_gam, vpc, pc_grad, pc_dq, out_pcf;
  bool have_pc = false;
  int64_t npc = 0;
  std::vector<int64_t> h_pc_off;
  int32_t* h_count = nullptr;   // pinned
  int32_t* h_list = nullptr;    // pinned copy of the active list
  int64_t h_list_cap = 0;
  int last_memory = 0;
  bool have_results = false;
  int64_t ledger = 0;          // device bytes of every Dbuf above
  bool trace = false;
  bool tridiag_smem = false;   // use the shared-memory tridiagonalisation for every size
  bool mixed = false;          // split-precision GEMMs until the precision switch
  double prec_switch = 1e-5;
  bool graphs = false;
  Dbuf prec, split_iters, gate_hits, last_rms;
  // warm-started refinement of the SCC eigenvectors (k_refine.cu): the
  // eigenvector columns V and the product buffer of a step per channel, and
  // the per-channel phases and masks that route channels between the
  // refinement and the Householder path
  Dbuf Vw, Vt, wstate, wphase, m_step, m_apply, m_cold, m_warm, w_emax, w_fail, w_arrive, w_bounds,
      w_stats;
  // refinement steps per SCC iteration; 0 (the default) = the Householder path
  // in every iteration.  The warm-started refinement is an opt-in
  // (XTBLOOM_B200_REFINE_STEPS): on the hetero-alkane workload too many
  // channels fall back to the Householder path (near-degenerate levels inside
  // the occupied and virtual blocks keep the block bounds loose) for it to
  // pay (1356 vs 1037 ms per 4096-system step, both FP64, same results).
  int refine_steps = 0;
  int refine_from = 1;       // first SCC iteration that refines
  // max |E| that ends a channel's refinement: split-precision iterations,
  // FP64 iterations, FP64 iterations once the residual is below
  // refine_final_factor x the charge tolerance (the result must then be as
  // exact as a direct solve: the gate compares energies to 1e-8 Eh or less)
  double refine_theta_split = 1e-5, refine_theta = 1e-7, refine_theta_final = 1e-11;
  double refine_final_factor = 100.0;
  // strict WARM start: the converged state of the latest fully converged call
  // and that call's identity (topology, charges, spin, point-charge layout,
  // requested properties and SCC settings)
  Dbuf ck_qsh, ck_dip, ck_qp, ck_qmag, ck_mdip, ck_mqp;
  bool ck_valid = false;
  struct CallIdentity {
    HostBatch topo;
    uint32_t flags = 0;
    int32_t max_iter = 0, memory = 0;
    double ctol = 0, etol = 0, kt = 0, damping = 0;
    std::vector<int64_t> pc_off;
    std::vector<uint8_t> field_attached;
    std::vector<double> field;
    std::vector<int64_t> resp_off;   // charge-response structure (present: nsys + 1 offsets)
    bool operator==(const CallIdentity& o) const {
      return topo.nsys == o.topo.nsys && topo.atom_off == o.topo.atom_off && topo.Z == o.topo.Z &&
             topo.qmol == o.topo.qmol && topo.uhf == o.topo.uhf && topo.nch == o.topo.nch &&
             topo.model == o.topo.model &&
             flags == o.flags && max_iter == o.max_iter && memory == o.memory && ctol == o.ctol &&
             etol == o.etol && kt == o.kt && damping == o.damping && pc_off == o.pc_off &&
             field_attached == o.field_attached && field == o.field && resp_off == o.resp_off;
    }
  } ck_id;
  Dbuf fdone;
  Dbuf umma_fault;   // int32: a tensor-core wait of the split-precision tiles ran out
  Profiler prof;

  DevTopo devtopo() const {
    DevTopo t{};
    t.m = model;
    t.nsys = (int32_t)nsys;
    t.total_atoms = natoms;
    t.total_shells = nshells;
    t.total_aos = naos;
    t.atom_off = atom_off.as<int64_t>();
    t.shell_off = shell_off.as<int64_t>();
    t.ao_off = ao_off.as<int64_t>();
    t.mat_off = mat_off.as<int64_t>();
    t.gam_off = gam_off.as<int64_t>();
    t.vec_off = vec_off.as<int64_t>();
    t.nao = nao.as<int32_t>();
    t.nel_a = nel_a.as<double>();
    t.nel_b = nel_b.as<double>();
    t.qmol = qmol.as<double>();
    t.nch = nch.as<int32_t>();
    t.beta_ch = beta_ch.as<int32_t>();
    t.sh_spinw = sh_spinw.as<double>();
    t.efield = have_field ? efield.as<double>() : nullptr;
    t.resp_b = have_resp ? resp_b.as<double>() : nullptr;
    t.resp_A = have_resp ? resp_A.as<double>() : nullptr;
    t.resp_off = have_resp ? resp_off.as<int64_t>() : nullptr;
    t.Z = Z.as<int32_t>();
    t.atom_sh = atom_sh.as<int32_t>();
    t.pos = pos.as<double>();
    t.at_en = at_en.as<double>();
    t.at_rad = at_rad.as<double>();
    t.at_rcov = at_rcov.as<double>();
    t.at_mprad = at_mprad.as<double>();
    t.at_mpvcn = at_mpvcn.as<double>();
    t.at_dk = at_dk.as<double>();
    t.at_qk = at_qk.as<double>();
    t.at_rep_sa = at_rep_sa.as<double>();
    t.at_rep_z = at_rep_z.as<double>();
    t.d4_rcov = d4_rcov.as<double>();
    t.d4_en = d4_en.as<double>();
    t.d4_zeff = d4_zeff.as<double>();
    t.d4_eta = d4_eta.as<double>();
    t.d4_r4r2 = d4_r4r2.as<double>();
    t.d4_roff = d4_roff.as<int32_t>();
    t.d4_rcnt = d4_rcnt.as<int32_t>();
    t.at_xbond = at_xbond.as<double>();
    t.kpair = kpair.as<double>();
    t.d3_rcnt = d3_rcnt.as<int32_t>();
    t.d3_roff = d3_roff.as<int32_t>();
    t.d3_ref_cn = d3_ref_cn.as<double>();
    t.d3_c6 = d3_c6.as<double>();
    t.d3_r4r2 = d3_r4r2.as<double>();
    t.sh_val = sh_val.as<int32_t>();
    t.sh_atom = sh_atom.as<int32_t>();
    t.sh_l = sh_l.as<int32_t>();
    t.sh_ao = sh_ao.as<int32_t>();
    t.sh_p0 = sh_p0.as<int32_t>();
    t.sh_np = sh_np.as<int32_t>();
    t.sh_level = sh_level.as<double>();
    t.sh_kcn = sh_kcn.as<double>();
    t.sh_shpoly = sh_shpoly.as<double>();
    t.sh_zeta = sh_zeta.as<double>();
    t.sh_eta = sh_eta.as<double>();
    t.pc_off = have_pc ? pc_off.as<int64_t>() : nullptr;
    t.pc_pos = have_pc ? pc_pos.as<double>() : nullptr;
    t.pc_q = have_pc ? pc_q.as<double>() : nullptr;
    t.pc_gam = have_pc ? pc_gam.as<double>() : nullptr;
    t.vpc = have_pc ? vpc.as<double>() : nullptr;
    t.sh_g3 = sh_g3.as<double>();
    t.sh_refocc = sh_refocc.as<double>();
    t.p_alpha = p_alpha.as<double>();
    t.p_coeff = p_coeff.as<double>();
    t.ao_sh = ao_sh.as<int32_t>();
    t.ao_at = ao_at.as<int32_t>();
    t.ref_cn = ref_cn.as<double>();
    t.ref_q = ref_q.as<double>();
    t.ref_ng = ref_ng.as<int32_t>();
    t.ref_c6 = ref_c6.as<double>();
    t.ref_count = 262;
    return t;
  }
};

Engine::Engine(int device, cudaStream_t stream) : impl_(new Impl), device_(device), stream_(stream) {
  cudaMallocHost(&impl_->h_count, 4 * sizeof(int32_t));
  const char* env = std::getenv("XTBLOOM_B200_KERNEL_TIMING");
  impl_->prof.on = env != nullptr && env[0] == '1';
  const char* tr = std::getenv("XTBLOOM_B200_TRACE");
  impl_->trace = tr != nullptr && tr[0] == '1';
  const char* td = std::getenv("XTBLOOM_B200_TRIDIAG");
  impl_->tridiag_smem = td != nullptr && std::strcmp(td, "smem") == 0;
  // XTBLOOM_B200_GEMM_WIDTH=32|64 fixes the FP64 tile width of every product
  // instead of timing both (a check that the widths form identical elements).
  // XTBLOOM_B200_REFINE_STEPS=k: refinement steps per SCC iteration (k > 0
  // turns the warm-started eigensolver on; 0 keeps the Householder path).
  const char* rs = std::getenv("XTBLOOM_B200_REFINE_STEPS");
  if (rs != nullptr && rs[0] >= '0' && rs[0] <= '9') impl_->refine_steps = std::min(8, std::atoi(rs));
  const char* gw = std::getenv("XTBLOOM_B200_GEMM_WIDTH");
  if (gw != nullptr && (std::strcmp(gw, "32") == 0 || std::strcmp(gw, "64") == 0))
    impl_->forced_gemm_width = std::atoi(gw);
}

void Engine::set_execution(int precision, double switch_residual, bool graphs) {
  impl_->mixed = precision == 1;
  impl_->prec_switch = switch_residual;
  impl_->graphs = graphs;
}

Engine::~Engine() {
  for (int i = 0; i < Impl::kBucketStreams; ++i) {
    if (impl_->bst[i]) cudaStreamDestroy(impl_->bst[i]);
    if (impl_->bjoin[i]) cudaEventDestroy(impl_->bjoin[i]);
    if (impl_->fst[i]) cudaStreamDestroy(impl_->fst[i]);
    if (impl_->ffork[i]) cudaEventDestroy(impl_->ffork[i]);
    if (impl_->wydone[i]) cudaEventDestroy(impl_->wydone[i]);
  }
  if (impl_->bfork) cudaEventDestroy(impl_->bfork);
  if (impl_->h_count) cudaFreeHost(impl_->h_count);
  if (impl_->h_list) cudaFreeHost(impl_->h_list);
  if (impl_->h_clist) cudaFreeHost(impl_->h_clist);
  delete impl_;
}

namespace {

// Times one product at both FP64 tile widths (each twice, best of two) and
// returns the faster width, or 0 when the events cannot be made.  The product
// is out of place, so running it several times leaves the same result.
int tune_gemm_width(const GemmArgs& g, bool ta, bool weighted, int tiles, int count, cudaStream_t st) {
  cudaEvent_t ev[5] = {};
  bool ok = true;
  for (auto& e : ev) ok = ok && cudaEventCreate(&e) == cudaSuccess;
  int width = 0;
  if (ok) {
    const int order[4] = {64, 32, 64, 32};
    cudaEventRecord(ev[0], st);
    for (int q = 0; q < 4; ++q) {
      launch_gemm(g, ta, weighted, tiles, count, st, order[q]);
      cudaEventRecord(ev[q + 1], st);
    }
    float t[4] = {0.f, 0.f, 0.f, 0.f};
    if (cudaEventSynchronize(ev[4]) == cudaSuccess) {
      bool timed = true;
      for (int q = 0; q < 4; ++q) timed = timed && cudaEventElapsedTime(&t[q], ev[q], ev[q + 1]) == cudaSuccess;
      if (timed) width = std::min(t[1], t[3]) < std::min(t[0], t[2]) ? 32 : 64;
    }
  }
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  return width;
}

bool ensure_tables(Engine::Impl& m, cudaStream_t s) {
  if (m.tables_ready) return true;
  auto upd = [&](Dbuf& b, const double* src, size_t n) {
    return b.reserve(n * sizeof(double)) &&
           cudaMemcpyAsync(b.p, src, n * sizeof(double), cudaMemcpyHostToDevice, s) == cudaSuccess;
  };
  auto upi = [&](Dbuf& b, const int* src, size_t n) {
    return b.reserve(n * sizeof(int)) &&
           cudaMemcpyAsync(b.p, src, n * sizeof(int), cudaMemcpyHostToDevice, s) == cudaSuccess;
  };
  bool ok = upd(m.d4_rcov, kP_d4_rcov, 86) && upd(m.d4_en, kP_d4_en, 86) &&
            upd(m.d4_zeff, kP_d4_zeff, 86) && upd(m.d4_eta, kP_d4_eta, 86) &&
            upd(m.d4_r4r2, kP_d4_r4r2, 86) && upi(m.d4_roff, kP_d4_ref_offset, 86) &&
            upi(m.d4_rcnt, kP_d4_ref_count, 86) && upd(m.ref_cn, kP_d4_ref_cn, 262) &&
            upd(m.ref_q, kP_d4_ref_q, 262) && upi(m.ref_ng, kP_d4_ref_ngauss, 262) &&
            upd(m.ref_c6, kP_d4_ref_c6, 262 * 262) && upd(m.kpair, kP_gfn1_kpair, 86 * 86) &&
            upi(m.d3_rcnt, kP_d3_ref_count, 86) && upi(m.d3_roff, kP_d3_ref_offset, 86) &&
            upd(m.d3_ref_cn, kP_d3_ref_cn, kD3Refs) && upd(m.d3_c6, kP_d3_ref_c6, kD3Refs * kD3Refs) &&
            upd(m.d3_r4r2, kP_d3_r4r2, 86);
  m.tables_ready = ok;
  return ok;
}

bool same_topology(const HostBatch& a, const HostBatch& b) {
  return a.nsys == b.nsys && a.atom_off == b.atom_off && a.Z == b.Z && a.qmol == b.qmol &&
         a.uhf == b.uhf && a.nch == b.nch && a.model == b.model;
}

xtbloom_status_t build_topology(Engine::Impl& m, const HostBatch& hb, cudaStream_t s,
                                std::string& error) {
  const int64_t B = hb.nsys;
  const int64_t N = hb.atom_off[B];
  std::vector<int64_t> atom_off = hb.atom_off, shell_off(B + 1), ao_off(B + 1), mat_off(B + 1),
                       gam_off(B + 1), vec_off(B + 1), scr_off(B + 1);
  std::vector<int32_t> nao(B), Zv(hb.Z.begin(), hb.Z.end()), atom_sh(N + 1);
  std::vector<double> nel_a(B), nel_b(B), qmol(hb.qmol.begin(), hb.qmol.end());
  std::vector<double> at_en(N), at_rad(N), at_rcov(N), at_mprad(N), at_mpvcn(N), at_dk(N), at_qk(N),
      at_rep_sa(N), at_rep_z(N), at_xbond(N, 0.0);
  std::vector<int32_t> sh_atom, sh_l, sh_ao, sh_p0, sh_np, ao_sh, ao_at, sh_val;
  // GFN1 (model/gfn1/basis.cpp, h0.cpp, es2.cpp, es3.cpp, repulsion.cpp,
  // coordination.cpp, halogen.cpp) or GFN2 element and shell parameters
  const bool g1 = hb.model == XTBLOOM_MODEL_GFN1_XTB;
  std::vector<double> sh_level, sh_kcn, sh_shpoly, sh_zeta, sh_eta, sh_g3, sh_refocc, p_alpha, p_coeff,
      sh_spinw;
  int64_t shell = 0;
  int max_n = 0, max_atoms = 0, max_shells = 0, max_dim = 0;
  int64_t max_pairs = 0;
  for (int64_t sy = 0; sy < B; ++sy) {
    shell_off[sy] = shell;
    ao_off[sy] = (int64_t)ao_sh.size();
    int ao_local = 0;
    double nel = 0.0;
    for (int64_t a = atom_off[sy]; a < atom_off[sy + 1]; ++a) {
      const int z = Zv[a];
      const int zi = z - 1;
      atom_sh[a] = (int32_t)shell;
      if (g1) {
        at_en[a] = kP_gfn1_en[zi];
        at_rad[a] = kP_gfn1_atomic_radius[zi];
        at_rcov[a] = kP_gfn1_covalent_radius[zi];
        at_mprad[a] = at_mpvcn[a] = at_dk[a] = at_qk[a] = 0.0;
        at_rep_sa[a] = std::sqrt(kP_gfn1_arep[zi]);
        at_rep_z[a] = kP_gfn1_zeff[zi];
        at_xbond[a] = kP_gfn1_xbond[zi];
      } else {
        at_en[a] = kP_gfn2_en[zi];
        at_rad[a] = kP_atomic_radii_angstrom[zi] * kAngstromToBohr;
        at_rcov[a] = (4.0 / 3.0) * kAngstromToBohr * kP_covalent_radii_angstrom[zi];
        at_mprad[a] = kP_gfn2_mprad[zi];
        at_mpvcn[a] = kP_gfn2_mpvcn[zi];
        at_dk[a] = kP_gfn2_dkernel[zi];
        at_qk[a] = kP_gfn2_qkernel[zi];
        at_rep_sa[a] = std::sqrt(kP_gfn2_arep[zi]);
        at_rep_z[a] = kP_gfn2_zeff[zi];
      }
      const int nsh = g1 ? kP_gfn1_nshell[zi] : kP_gfn2_nshell[zi];
      int first_of_l[5] = {-1, -1, -1, -1, -1};
      for (int k = 0; k < nsh; ++k) {
        const int l = g1 ? kP_gfn1_shell_l[3 * zi + k] : kP_gfn2_shell_l[3 * zi + k];
        const int pn = g1 ? kP_gfn1_shell_n[3 * zi + k] : kP_gfn2_shell_n[3 * zi + k];
        const int ng = g1 ? kP_gfn1_shell_ngauss[3 * zi + k] : kP_gfn2_shell_ngauss[3 * zi + k];
        const double zeta = g1 ? kP_gfn1_shell_slater[3 * zi + k] : kP_gfn2_shell_slater[3 * zi + k];
        std::vector<double> al, co;
        if (!(g1 ? sto_expand_gfn1(pn, l, ng, zeta, al, co) : sto_expand(pn, l, ng, zeta, al, co))) {
          error = "unsupported STO-nG shell in the parameter tables";
          return XTBLOOM_STATUS_INTERNAL_ERROR;
        }
        if (first_of_l[l] >= 0) {
          const int f = first_of_l[l];
          std::vector<double> a1(p_alpha.begin() + sh_p0[f], p_alpha.begin() + sh_p0[f] + sh_np[f]);
          std::vector<double> c1(p_coeff.begin() + sh_p0[f], p_coeff.begin() + sh_p0[f] + sh_np[f]);
          orthogonalize_to_first(a1, c1, al, co);
        } else {
          first_of_l[l] = (int)shell;
        }
        sh_atom.push_back((int32_t)a);
        sh_l.push_back(l);
        sh_ao.push_back(ao_local);
        sh_p0.push_back((int32_t)p_alpha.size());
        sh_np.push_back((int32_t)al.size());
        p_alpha.insert(p_alpha.end(), al.begin(), al.end());
        p_coeff.insert(p_coeff.end(), co.begin(), co.end());
        if (g1) {
          // GFN1: levels and CN scales in eV (xTB's 27.21138505 conversion);
          // third order per atom (no shell scaling)
          sh_level.push_back(kP_gfn1_shell_level[3 * zi + k] * kEvToHartree);
          sh_kcn.push_back(kP_gfn1_shell_kcn[3 * zi + k] * kEvToHartree);
          sh_shpoly.push_back(kP_gfn1_shell_shpoly[3 * zi + k]);
          sh_eta.push_back(kP_gfn1_gam[zi] * kP_gfn1_shell_hubbard_scale[3 * zi + k]);
          sh_g3.push_back(kP_gfn1_gam3[zi]);
          sh_val.push_back(kP_gfn1_shell_valence[3 * zi + k]);
        } else {
          sh_level.push_back(kP_gfn2_shell_level[3 * zi + k] * kEvToHartree);
          sh_kcn.push_back(kP_gfn2_shell_kcn[3 * zi + k] * kEvToHartree);
          sh_shpoly.push_back(kP_gfn2_shell_shpoly[3 * zi + k]);
          sh_eta.push_back(kP_gfn2_gam[zi] * kP_gfn2_shell_hubbard_scale[3 * zi + k]);
          sh_g3.push_back(kP_gfn2_gam3[zi] * m.model_gfn2.es3_scale[l]);
          sh_val.push_back(1);
        }
        sh_zeta.push_back(zeta);
        const double ro = g1 ? kP_gfn1_shell_refocc[3 * zi + k] : kP_gfn2_shell_refocc[3 * zi + k];
        sh_refocc.push_back(ro);
        nel += ro;
        for (int q = 0; q < 2 * l + 1; ++q) {
          ao_sh.push_back((int32_t)shell);
          ao_at.push_back((int32_t)a);
        }
        ao_local += 2 * l + 1;
        ++shell;
      }
      // atom-local spin couplings W(l_row, l_col) (tblite element constants,
      // ss sp pp sd pd dd), 3 per shell
      for (int64_t r = atom_sh[a]; r < shell; ++r) {
        for (int k = 0; k < 3; ++k) {
          double wv = 0.0;
          if (atom_sh[a] + k < shell) {
            int l1 = sh_l[r], l2 = sh_l[atom_sh[a] + k];
            if (l1 > l2) std::swap(l1, l2);
            const int idx = l1 == 0 ? (l2 == 0 ? 0 : (l2 == 1 ? 1 : 3)) : (l1 == 1 ? (l2 == 1 ? 2 : 4) : 5);
            wv = kP_spin_constants[6 * zi + idx];
          }
          sh_spinw.push_back(wv);
        }
      }
    }
    const int na = (int)(atom_off[sy + 1] - atom_off[sy]);
    const int ns = (int)(shell - shell_off[sy]);
    nao[sy] = ao_local;
    nel -= qmol[sy];
    const double u = hb.uhf[sy];
    if (!(nel >= 0.0) || u < 0 || u > nel + 1e-12) {
      error = "molecular charge or unpaired electrons are incompatible with the electron count";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    nel_a[sy] = 0.5 * (nel + u);
    nel_b[sy] = 0.5 * (nel - u);
    max_n = std::max(max_n, ao_local);
    max_atoms = std::max(max_atoms, na);
    max_shells = std::max(max_shells, ns);
    max_dim = std::max(max_dim, hb.nch[sy] * (g1 ? ns : ns + 9 * na));
    max_pairs = std::max<int64_t>(max_pairs, (int64_t)na * (na + 1) / 2);
  }
  shell_off[B] = shell;
  ao_off[B] = (int64_t)ao_sh.size();
  atom_sh[N] = (int32_t)shell;
  mat_off[0] = gam_off[0] = vec_off[0] = scr_off[0] = 0;
  for (int64_t sy = 0; sy < B; ++sy) {
    const int64_t n = nao[sy];
    const int64_t k = shell_off[sy + 1] - shell_off[sy];
    const int64_t na = atom_off[sy + 1] - atom_off[sy];
    mat_off[sy + 1] = mat_off[sy] + n * n;
    gam_off[sy + 1] = gam_off[sy] + k * k;
    vec_off[sy + 1] = vec_off[sy] + hb.nch[sy] * (g1 ? k : k + 9 * na);
    scr_off[sy + 1] = scr_off[sy] + eig_scratch(n);
  }
  // largest systems first
  std::vector<int32_t> order(B);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return nao[a] > nao[b]; });

  m.nsys = B;
  m.natoms = N;
  m.nshells = shell;
  m.naos = ao_off[B];
  m.total_mat = mat_off[B];
  m.total_gam = gam_off[B];
  m.total_vec = vec_off[B];
  m.total_scr = scr_off[B];
  m.total_prim = (int64_t)p_alpha.size();
  m.max_n = max_n;
  m.max_atoms = max_atoms;
  m.max_shells = max_shells;
  m.max_dim = max_dim;
  m.max_pairs = max_pairs;
  m.h_nao = nao;
  m.h_order = order;
  m.h_nel_a = nel_a;
  m.h_nel_b = nel_b;

  // spin channels (see Impl): restricted channel c = s holds both electron
  // counts (occupation <= 2); unrestricted alpha (c = s) and beta
  // (c = B + u) hold one count each (occupation <= 1)
  std::vector<int32_t> nchv(hb.nch.begin(), hb.nch.end()), beta(B, -1);
  int64_t nU = 0;
  for (int64_t sy = 0; sy < B; ++sy) nU += nchv[sy] == 2 ? 1 : 0;
  const int64_t NC = B + nU;
  std::vector<int32_t> ch_sys(NC), ch_sign(NC), ch_nao(NC);
  std::vector<int64_t> ch_mat(NC), ch_ao(NC), ch_scr(NC), ch_xoff(NC);
  std::vector<double> ch_nel_a(NC), ch_nel_b(NC);
  int64_t xm = 0, xv = 0, xs = 0, u = 0;
  for (int64_t sy = 0; sy < B; ++sy) {
    const bool un = nchv[sy] == 2;
    ch_sys[sy] = (int32_t)sy;
    ch_sign[sy] = un ? 1 : 0;
    ch_nao[sy] = nao[sy];
    ch_mat[sy] = mat_off[sy];
    ch_ao[sy] = ao_off[sy];
    ch_scr[sy] = scr_off[sy];
    ch_xoff[sy] = mat_off[sy];
    ch_nel_a[sy] = nel_a[sy];
    ch_nel_b[sy] = un ? 0.0 : nel_b[sy];
    if (un) {
      const int64_t c = B + u++;
      const int64_t n = nao[sy];
      beta[sy] = (int32_t)c;
      ch_sys[c] = (int32_t)sy;
      ch_sign[c] = -1;
      ch_nao[c] = (int32_t)n;
      ch_mat[c] = mat_off[B] + xm;
      ch_ao[c] = ao_off[B] + xv;
      ch_scr[c] = scr_off[B] + xs;
      ch_xoff[c] = mat_off[sy];
      ch_nel_a[c] = nel_b[sy];
      ch_nel_b[c] = 0.0;
      xm += n * n;
      xv += n;
      xs += eig_scratch(n);
    }
  }
  m.nchan = NC;
  m.nuhf = nU;
  m.chan_mat = xm;
  m.chan_vec = xv;
  m.chan_scr = xs;
  m.h_ch_nao = ch_nao;
  m.h_ch_sys = ch_sys;
  m.h_ch_nel_a = ch_nel_a;
  m.h_ch_nel_b = ch_nel_b;
  if (m.h_clist_cap < NC) {
    if (m.h_clist) cudaFreeHost(m.h_clist);
    m.h_clist = nullptr;
    if (cudaMallocHost(&m.h_clist, NC * sizeof(int32_t)) != cudaSuccess) {
      error = "pinned host allocation failed";
      return XTBLOOM_STATUS_ALLOCATION_FAILED;
    }
    m.h_clist_cap = NC;
  }
  if (!upload(m.nch, nchv, s) || !upload(m.beta_ch, beta, s) || !upload(m.sh_spinw, sh_spinw, s) ||
      !upload(m.ch_sys, ch_sys, s) || !upload(m.ch_sign, ch_sign, s) || !upload(m.ch_nao, ch_nao, s) ||
      !upload(m.ch_mat, ch_mat, s) || !upload(m.ch_ao, ch_ao, s) || !upload(m.ch_scr, ch_scr, s) ||
      !upload(m.ch_xoff, ch_xoff, s) || !upload(m.ch_nel_a, ch_nel_a, s) ||
      !upload(m.ch_nel_b, ch_nel_b, s) || !m.clist.reserve((size_t)NC * 4) || !m.ccount.reserve(16)) {
    error = "device allocation for the spin channels failed";
    return XTBLOOM_STATUS_ALLOCATION_FAILED;
  }
  // the host vectors above must outlive their asynchronous uploads
  cudaStreamSynchronize(s);

  bool ok = upload(m.atom_off, atom_off, s) && upload(m.shell_off, shell_off, s) &&
            upload(m.ao_off, ao_off, s) && upload(m.mat_off, mat_off, s) &&
            upload(m.gam_off, gam_off, s) && upload(m.vec_off, vec_off, s) &&
            upload(m.scr_off, scr_off, s) && upload(m.nao, nao, s) && upload(m.nel_a, nel_a, s) &&
            upload(m.nel_b, nel_b, s) && upload(m.qmol, qmol, s) && upload(m.Z, Zv, s) &&
            upload(m.atom_sh, atom_sh, s) && upload(m.at_en, at_en, s) &&
            upload(m.at_rad, at_rad, s) && upload(m.at_rcov, at_rcov, s) &&
            upload(m.at_mprad, at_mprad, s) && upload(m.at_mpvcn, at_mpvcn, s) &&
            upload(m.at_dk, at_dk, s) && upload(m.at_qk, at_qk, s) &&
            upload(m.at_rep_sa, at_rep_sa, s) && upload(m.at_rep_z, at_rep_z, s) &&
            upload(m.at_xbond, at_xbond, s) && upload(m.sh_val, sh_val, s) &&
            upload(m.sh_atom, sh_atom, s) && upload(m.sh_l, sh_l, s) && upload(m.sh_ao, sh_ao, s) &&
            upload(m.sh_p0, sh_p0, s) && upload(m.sh_np, sh_np, s) &&
            upload(m.sh_level, sh_level, s) && upload(m.sh_kcn, sh_kcn, s) &&
            upload(m.sh_shpoly, sh_shpoly, s) && upload(m.sh_zeta, sh_zeta, s) &&
            upload(m.sh_eta, sh_eta, s) && upload(m.sh_g3, sh_g3, s) &&
            upload(m.sh_refocc, sh_refocc, s) && upload(m.p_alpha, p_alpha, s) &&
            upload(m.p_coeff, p_coeff, s) && upload(m.ao_sh, ao_sh, s) &&
            upload(m.ao_at, ao_at, s) && upload(m.order, order, s);
  const size_t d8 = sizeof(double);
  const size_t mat = (size_t)m.total_mat * d8;
  const size_t cmat = (size_t)(m.total_mat + m.chan_mat) * d8;     // channel matrices
  const size_t cvec = (size_t)(m.naos + m.chan_vec) * d8;          // channel vectors
  ok = ok && m.pos.reserve((size_t)N * 3 * d8) && m.list.reserve((size_t)B * 4) &&
       m.count.reserve(16) && m.status.reserve((size_t)B * 4) && m.iterations.reserve((size_t)B * 4) &&
       m.converged.reserve((size_t)B) && m.prec.reserve((size_t)B) &&
       m.fdone.reserve((size_t)B) && m.umma_fault.reserve(4) &&
       m.split_iters.reserve((size_t)B * 4) && m.gate_hits.reserve((size_t)B * 4) && m.last_rms.reserve((size_t)B * 8) && m.nvec.reserve((size_t)NC * 4) && m.cn.reserve(N * d8) &&
       m.cn_d4.reserve(N * d8) && m.mrad.reserve(N * d8) && m.dmrad.reserve(N * d8) &&
       m.gam.reserve((size_t)m.total_gam * d8) && m.S.reserve(mat) && m.D.reserve(3 * mat) &&
       m.Q.reserve(6 * mat) && m.H0.reserve(mat) && m.H.reserve(cmat) && m.X.reserve(mat) &&
       m.T.reserve(cmat) && m.A.reserve(cmat) && m.Zv.reserve(cmat) && m.C.reserve(cmat) &&
       m.P.reserve(cmat) && m.W.reserve(cmat) && m.Vw.reserve(cmat) && m.Vt.reserve(cmat) &&
       m.wstate.reserve((size_t)NC) && m.wphase.reserve((size_t)NC) && m.m_step.reserve((size_t)NC) &&
       m.m_apply.reserve((size_t)NC) && m.m_cold.reserve((size_t)NC) && m.m_warm.reserve((size_t)NC) &&
       m.w_emax.reserve((size_t)NC * 8) && m.w_fail.reserve((size_t)NC * 4) &&
       m.w_arrive.reserve((size_t)NC * 4) && m.w_stats.reserve(256 * 8 * 4) &&
       m.w_bounds.reserve((size_t)NC * kRefineMaxParts * 9 * d8) &&
       m.d.reserve(cvec) && m.e.reserve(cvec) &&
       m.tau.reserve(cvec) && m.eig.reserve(cvec) && m.occ.reserve(cvec) &&
       m.occ_eps.reserve(cvec) && m.entropy.reserve(NC * d8) &&
       m.scratch.reserve((size_t)(m.total_scr + m.chan_scr) * d8) && m.qsh.reserve(shell * d8) &&
       m.Pm.reserve(nU > 0 ? mat : 8) && m.qmag.reserve(shell * d8) && m.vmag.reserve(shell * d8) &&
       m.pop_mag.reserve(shell * d8) && m.pop_mdip.reserve(3 * N * d8) &&
       m.pop_mqp.reserve(6 * N * d8) &&
       m.dip.reserve(3 * N * d8) && m.qp.reserve(6 * N * d8) && m.pop_sh.reserve(shell * d8) &&
       m.pop_dip.reserve(3 * N * d8) && m.pop_qp.reserve(6 * N * d8) && m.e_core.reserve(B * d8) &&
       m.vsh.reserve(shell * d8) && m.vd.reserve(3 * N * d8) && m.vq.reserve(6 * N * d8) &&
       m.free_energy.reserve(B * d8) && m.terms.reserve(kTermCount * B * d8) &&
       m.mx_cur.reserve((size_t)m.total_vec * d8) && m.mx_prev.reserve((size_t)m.total_vec * d8) &&
       m.mx_res.reserve((size_t)m.total_vec * d8) && m.grad.reserve(3 * N * d8) &&
       m.acn.reserve(N * d8) && m.acn_d4.reserve(N * d8) && m.pot_acc.reserve(10 * N * d8) &&
       cudaMemsetAsync(m.pot_acc.p, 0, 10 * N * d8, s) == cudaSuccess && m.out_energy.reserve(B * d8) &&
       m.out_forces.reserve(3 * N * d8) && m.out_charges.reserve(N * d8);
  if (!ok) {
    error = "device allocation for the batch failed";
    return XTBLOOM_STATUS_ALLOCATION_FAILED;
  }
  return XTBLOOM_STATUS_SUCCESS;
}

bool read_input(const xtbloom_const_buffer_t& b, void* dst, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return true;
  const cudaMemcpyKind kind =
      b.memory_space == XTBLOOM_MEMORY_CUDA_DEVICE ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
  if (kind == cudaMemcpyHostToHost) {
    std::memcpy(dst, b.data, bytes);
    return true;
  }
  return cudaMemcpyAsync(dst, b.data, bytes, kind, s) == cudaSuccess && cudaStreamSynchronize(s) == cudaSuccess;
}

// Per system: energy, forces (with the explicit field force q_A E of a
// uniform field, gfn2_cpu_execution.cpp:1588-1597 of the reference), charges
// and the dipole moment sum_A q_A R_A + d_A (gfn2_cpu_execution.cpp:1497-1508).
__global__ void k_publish(DevTopo t, const int32_t* status, const double* free_energy,
                          const double* terms, const double* grad, const double* qsh,
                          const double* dip, double* energy, double* forces, double* charges,
                          double* dipoles) {
  __shared__ double red[33];
  const int s = blockIdx.x;
  const bool ok = status[s] == kOk;
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  const int64_t a0 = t.atom_off[s], a1 = t.atom_off[s + 1];
  const double* ef = t.efield != nullptr ? t.efield + 3 * s : nullptr;
  if (threadIdx.x == 0)
    energy[s] = ok ? free_energy[s] + terms[kTermCount * (int64_t)s + kTermRep] +
                         terms[kTermCount * (int64_t)s + kTermAtm] +
                         terms[kTermCount * (int64_t)s + kTermDisp3] +
                         terms[kTermCount * (int64_t)s + kTermXb]
               : nan;
  double mu[3] = {0.0, 0.0, 0.0};
  for (int64_t a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    double q = 0.0;
    for (int sh = t.atom_sh[a]; sh < t.atom_sh[a + 1]; ++sh) q += qsh[sh];
    charges[a] = ok ? q : nan;
    for (int c = 0; c < 3; ++c) {
      forces[3 * a + c] = ok ? -fix_value(grad[3 * a + c]) + (ef != nullptr ? q * ef[c] : 0.0) : nan;
      mu[c] += q * t.pos[3 * a + c] + dip[3 * a + c];
    }
  }
  for (int c = 0; c < 3; ++c) {
    const double m = block_sum(mu[c], red);
    if (threadIdx.x == 0) dipoles[3 * s + c] = ok ? m : nan;
  }
}

__global__ void k_finalize_status(int nsys, int32_t* status, const uint8_t* converged) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nsys && status[i] == kOk && !converged[i]) status[i] = kNotConverged;
}

// Channel list of a system list: every system's first channel (id = system)
// followed, for unrestricted systems, by its beta channel; order preserved.
// One block of 1024 threads; count is read on the device.
__global__ void k_channels(const int32_t* list, const int32_t* count, const int32_t* beta_ch,
                           int32_t* clist, int32_t* ccount) {
  __shared__ int wtot[32];
  __shared__ int base, chunk_total;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const int n = count[0];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c0 = 0; c0 < n; c0 += blockDim.x) {
    const int i = c0 + threadIdx.x;
    const int sys = i < n ? list[i] : -1;
    const int bc = sys >= 0 ? beta_ch[sys] : -1;
    const int w = sys < 0 ? 0 : (bc >= 0 ? 2 : 1);
    int incl = w;   // inclusive warp scan
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) wtot[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
        const int v = wtot[q];
        wtot[q] = acc;
        acc += v;
      }
      chunk_total = acc;
    }
    __syncthreads();
    const int pos = base + wtot[warp] + incl - w;
    if (w >= 1) clist[pos] = sys;
    if (w == 2) clist[pos + 1] = bc;
    __syncthreads();
    if (threadIdx.x == 0) base += chunk_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) ccount[0] = base;
}

// Unrestricted systems of the list: the alpha-channel matrix (at the system's
// offset) becomes the total alpha + beta; with Pm, also P_alpha - P_beta.
__global__ void k_combine_spin(const int32_t* list, const int32_t* beta_ch, const int32_t* nao,
                               const int64_t* mat_off, const int64_t* ch_mat, double* M,
                               double* Pm) {
  const int s = list[blockIdx.y];
  const int bc = beta_ch[s];
  if (bc < 0) return;
  const int64_t n2 = (int64_t)nao[s] * nao[s];
  double* a = M + mat_off[s];
  const double* b = M + ch_mat[bc];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n2;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double va = a[i], vb = b[i];
    a[i] = va + vb;
    if (Pm != nullptr) Pm[mat_off[s] + i] = va - vb;
  }
}

// Converged systems (status ok) whose energy and force terms are not yet
// formed, in cost order; marks them formed.  One block of 1024 threads (an
// ordered compaction, like the active list).
__global__ void k_list_ready(const int32_t* order, int nsys, const int32_t* status,
                             const uint8_t* converged, uint8_t* done, int32_t* list, int32_t* count) {
  __shared__ int wtot[32];
  __shared__ int base, chunk_total;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c0 = 0; c0 < nsys; c0 += blockDim.x) {
    const int i = c0 + threadIdx.x;
    int sys = -1;
    bool take = false;
    if (i < nsys) {
      sys = order[i];
      take = status[sys] == kOk && converged[sys] != 0 && done[sys] == 0;
    }
    const unsigned b = __ballot_sync(0xffffffffu, take);
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
    if (take) {
      list[base + wtot[warp] + pre] = sys;
      done[sys] = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) base += chunk_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) count[0] = base;
}

}  // namespace

void Engine::invalidate_checkpoint() { impl_->ck_valid = false; }

size_t Engine::device_bytes() const { return (size_t)std::max<int64_t>(0, impl_->ledger); }

size_t Engine::host_bytes() const {
  return 4 * sizeof(int32_t) + (size_t)impl_->h_list_cap * sizeof(int32_t) +
         (size_t)impl_->h_clist_cap * sizeof(int32_t);
}

xtbloom_status_t Engine::compute(const ComputeRequest& req, std::string& error) {
  Impl& m = *impl_;
  // every device buffer this call grows is counted in the engine's ledger
  struct LedgerScope {
    int64_t* prev;
    explicit LedgerScope(int64_t* l) : prev(t_ledger) { t_ledger = l; }
    ~LedgerScope() { t_ledger = prev; }
  } ledger_scope(&m.ledger);
  cudaStream_t s = stream_;
  cudaSetDevice(device_);
  const auto t_start = std::chrono::steady_clock::now();
  const xtbloom_batch_t& b = *req.batch;
  const int64_t B = b.batch_size;
  const int64_t N = b.total_atoms;
  if (!ensure_tables(m, s)) {
    error = "failed to upload parameter tables";
    return XTBLOOM_STATUS_ALLOCATION_FAILED;
  }
  // ---- stage topology descriptors on the host ----
  HostBatch hb;
  hb.nsys = B;
  hb.atom_off.resize(B + 1);
  hb.Z.resize(N);
  hb.qmol.resize(B);
  hb.uhf.resize(B, 0);
  hb.nch.assign(B, 1);
  if (!read_input(b.atom_offsets, hb.atom_off.data(), (B + 1) * 8, s) ||
      !read_input(b.atomic_numbers, hb.Z.data(), N * 4, s) ||
      !read_input(b.molecular_charges, hb.qmol.data(), B * 8, s) ||
      (b.unpaired_electrons.data && !read_input(b.unpaired_electrons, hb.uhf.data(), B * 4, s)) ||
      (req.spin_channels && b.spin_channels.data &&
       !read_input(b.spin_channels, hb.nch.data(), B * 4, s))) {
    error = "failed to read the batch descriptors";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (hb.atom_off[0] != 0 || hb.atom_off[B] != N) {
    error = "atom_offsets must start at zero and end at total_atoms";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  for (int64_t i = 0; i < B; ++i) {
    if (hb.atom_off[i + 1] <= hb.atom_off[i]) {
      error = "atom_offsets must be strictly increasing (every system needs an atom)";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    if (!std::isfinite(hb.qmol[i])) {
      error = "molecular_charges must be finite";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    if (hb.uhf[i] < 0) {
      error = "unpaired_electrons must be nonnegative";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    if (hb.nch[i] != 1 && hb.nch[i] != 2) {
      error = "spin_channels values must be one or two";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
  }
  for (int64_t a = 0; a < N; ++a) {
    if (hb.Z[a] < 1 || hb.Z[a] > 86) {
      error = "atomic_numbers must be in [1, 86]";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
  }
  hb.model = req.model;
  m.model = hb.model == XTBLOOM_MODEL_GFN1_XTB ? m.model_gfn1 : m.model_gfn2;
  if (!m.topo_valid || !same_topology(m.topo, hb)) {
    m.topo_valid = false;
    xtbloom_status_t st = build_topology(m, hb, s, error);
    if (st != XTBLOOM_STATUS_SUCCESS) return st;
    m.topo = hb;
    m.topo_valid = true;
  }
  // ---- positions ----
  {
    const cudaMemcpyKind kind = b.positions.memory_space == XTBLOOM_MEMORY_CUDA_DEVICE
                                    ? cudaMemcpyDeviceToDevice
                                    : cudaMemcpyHostToDevice;
    if (cudaMemcpyAsync(m.pos.p, b.positions.data, (size_t)N * 3 * 8, kind, s) != cudaSuccess) {
      error = "failed to stage positions";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
  }
  // ---- external point charges (validated here, before any output is touched) ----
  {
    const int64_t P = b.total_point_charges;
    m.have_pc = P > 0;
    m.npc = P;
    if (P > 0) {
      m.h_pc_off.assign(B + 1, 0);
      std::vector<double> ppos(3 * P), pq(P), pg(P);
      if (!read_input(b.point_charge_offsets, m.h_pc_off.data(), (B + 1) * 8, s) ||
          !read_input(b.point_charge_positions, ppos.data(), 3 * P * 8, s) ||
          !read_input(b.point_charge_values, pq.data(), P * 8, s) ||
          !read_input(b.point_charge_gammas, pg.data(), P * 8, s)) {
        error = "failed to read the point-charge inputs";
        return XTBLOOM_STATUS_INVALID_ARGUMENT;
      }
      if (m.h_pc_off[0] != 0 || m.h_pc_off[B] != P) {
        error = "point_charge_offsets must start at zero and end at total_point_charges";
        return XTBLOOM_STATUS_INVALID_ARGUMENT;
      }
      for (int64_t i = 0; i < B; ++i)
        if (m.h_pc_off[i + 1] < m.h_pc_off[i]) {
          error = "point_charge_offsets must be nondecreasing";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
      for (int64_t i = 0; i < 3 * P; ++i)
        if (!std::isfinite(ppos[i])) {
          error = "external point-charge positions contain NaN or infinity";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
      for (int64_t i = 0; i < P; ++i)
        if (!std::isfinite(pq[i]) || !(pg[i] > 0.0) || !std::isfinite(pg[i])) {
          error = "external point-charge values must be finite and hardnesses must be finite positive";
          return XTBLOOM_STATUS_INVALID_ARGUMENT;
        }
      if (!upload(m.pc_off, m.h_pc_off, s) || !upload(m.pc_pos, ppos, s) || !upload(m.pc_q, pq, s) ||
          !upload(m.pc_gam, pg, s) || !m.vpc.reserve((size_t)m.nshells * 8) ||
          !m.pc_grad.reserve((size_t)P * 24) || !m.pc_dq.reserve((size_t)P * 8) ||
          !m.out_pcf.reserve((size_t)P * 24)) {
        error = "device allocation for the point charges failed";
        return XTBLOOM_STATUS_ALLOCATION_FAILED;
      }
      cudaMemsetAsync(m.pc_grad.p, 0, (size_t)P * 24, s);
      cudaMemsetAsync(m.pc_dq.p, 0, (size_t)P * 8, s);
      // the host vectors must outlive the asynchronous uploads
      cudaStreamSynchronize(s);
    }
  }
  // ---- uniform electric fields of the attachments ----
  m.have_field = false;
  for (int64_t i = 0; i < B; ++i) m.have_field = m.have_field || req.field_attached[i] != 0;
  if (!m.out_dipoles.reserve((size_t)B * 24)) {
    error = "device allocation for the dipole moments failed";
    return XTBLOOM_STATUS_ALLOCATION_FAILED;
  }
  if (m.have_field) {
    if (!upload(m.efield, req.field, s)) {
      error = "device allocation for the electric fields failed";
      return XTBLOOM_STATUS_ALLOCATION_FAILED;
    }
    cudaStreamSynchronize(s);   // req.field outlives the upload either way; keep order simple
  }
  // ---- charge response b + A q ----
  m.have_resp = req.have_response;
  if (m.have_resp) {
    if (!upload(m.resp_b, req.resp_b, s) || !upload(m.resp_off, req.resp_off, s) ||
        !upload(m.resp_A, req.resp_A, s)) {
      error = "device allocation for the charge response failed";
      return XTBLOOM_STATUS_ALLOCATION_FAILED;
    }
    cudaStreamSynchronize(s);
  }
  // ---- strict WARM policy (reference include/xtbloom/xtbloom.h:502-523): a
  // WARM call needs the checkpoint of the latest fully converged call with the
  // same identity; every accepted call consumes the checkpoint ----
  Impl::CallIdentity ident;
  ident.topo = hb;
  ident.flags = req.flags;
  ident.max_iter = req.max_iter;
  ident.memory = req.memory;
  ident.ctol = req.ctol;
  ident.etol = req.etol;
  ident.kt = req.kt;
  ident.damping = req.damping;
  if (m.have_pc) ident.pc_off = m.h_pc_off;
  ident.field_attached = req.field_attached;
  ident.field = req.field;
  if (req.have_response) ident.resp_off = req.resp_off;
  if (req.warm && !(m.ck_valid && ident == m.ck_id)) {
    error = "WARM start requires the checkpoint of a fully converged call with the same topology, "
            "charges, spin settings, point-charge layout, requested properties and SCC settings";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  const bool warm = req.warm;
  m.ck_valid = false;
  // Broyden history sized by the requested memory
  const int M = req.memory;
  if (!m.mx_df.reserve((size_t)m.total_vec * M * 8) || !m.mx_u.reserve((size_t)m.total_vec * M * 8) ||
      !m.mx_omega.reserve((size_t)B * M * 8)) {
    error = "device allocation for the mixer history failed";
    return XTBLOOM_STATUS_ALLOCATION_FAILED;
  }
  const DevTopo t = m.devtopo();
  const int nsys = (int)B;
  int32_t* list = m.list.as<int32_t>();
  int32_t* dcount = m.count.as<int32_t>();
  int32_t* status = m.status.as<int32_t>();
  const int32_t* order = m.order.as<int32_t>();
  cudaMemsetAsync(status, 0, B * 4, s);
  cudaMemsetAsync(m.converged.p, 0, B, s);
  cudaMemsetAsync(m.iterations.p, 0, B * 4, s);
  cudaMemsetAsync(m.terms.p, 0, kTermCount * B * 8, s);
  cudaMemsetAsync(m.pot_acc.p, 0, 10 * N * 8, s);
  cudaMemsetAsync(m.prec.p, m.mixed ? 0 : 1, B, s);
  cudaMemsetAsync(m.split_iters.p, 0, B * 4, s);
  cudaMemsetAsync(m.gate_hits.p, 0, B * 4, s);
  cudaMemsetAsync(m.last_rms.p, 0x7f, B * 8, s);   // 1.4e306: no residual yet
  // no channel has eigenvectors to refine from yet
  cudaMemsetAsync(m.wstate.p, 0, (size_t)m.nchan, s);
  cudaMemsetAsync(m.w_stats.p, 0, 256 * 8 * 4, s);
  cudaMemsetAsync(m.fdone.p, 0, B, s);
  cudaMemsetAsync(m.umma_fault.p, 0, 4, s);
  cudaMemsetAsync(m.grad.p, 0, 3 * N * 8, s);
  cudaMemsetAsync(m.acn.p, 0, N * 8, s);
  cudaMemsetAsync(m.acn_d4.p, 0, N * 8, s);
  cudaMemcpyAsync(list, order, B * 4, cudaMemcpyDeviceToDevice, s);

  // first launch failure of any stage (a launch that fails does not run and
  // leaves its outputs unwritten, so the call must fail)
  cudaError_t launch_error = cudaSuccess;
#define XTB_STAGE(id, nk, ...) XTB_STAGE_ON(s, id, nk, __VA_ARGS__)
#define XTB_STAGE_ON(st, id, nk, ...)                                              \
  do {                                                                             \
    m.prof.begin(id, st);                                                          \
    __VA_ARGS__;                                                                   \
    m.prof.end(st);                                                                \
    m.prof.launches += (nk);                                                       \
    if (const cudaError_t le_ = cudaGetLastError(); le_ != cudaSuccess && !launch_error) \
      launch_error = le_;                                                          \
  } while (0)
  // ---- geometry setup ----
  XTB_STAGE(kStSetup, 3,
            launch_setup(t, list, nsys, m.max_atoms, m.max_pairs, m.max_shells, m.cn.as<double>(),
                         m.cn_d4.as<double>(), m.mrad.as<double>(), m.dmrad.as<double>(),
                         m.S.as<double>(), m.D.as<double>(), m.Q.as<double>(), m.H0.as<double>(),
                         m.gam.as<double>(), m.total_mat, s);
            if (m.have_pc) launch_pc_potential(t, list, nsys, m.vpc.as<double>(), s));

  // Eigensolver and GEMM arguments are indexed by spin channel; channel c < B
  // is system c at its own offsets, so system lists work for them as well.
  const int32_t* dch_nao = m.ch_nao.as<int32_t>();
  const int64_t* dch_mat = m.ch_mat.as<int64_t>();
  const int64_t* dch_ao = m.ch_ao.as<int64_t>();
  const int64_t* dch_xoff = m.ch_xoff.as<int64_t>();
  EigArgs eg{};
  eg.list = list;
  eg.nao = dch_nao;
  eg.mat_off = dch_mat;
  eg.ao_off = dch_ao;
  eg.A = m.A.as<double>();
  eg.d = m.d.as<double>();
  eg.e = m.e.as<double>();
  eg.tau = m.tau.as<double>();
  eg.eig = m.eig.as<double>();
  eg.occ = m.occ.as<double>();
  eg.occ_eps = m.occ_eps.as<double>();
  eg.entropy = m.entropy.as<double>();
  eg.nvec = m.nvec.as<int32_t>();
  eg.Z = m.Zv.as<double>();
  eg.scratch = m.scratch.as<double>();
  eg.scratch_off = m.ch_scr.as<int64_t>();
  eg.nel_a = m.ch_nel_a.as<double>();
  eg.nel_b = m.ch_nel_b.as<double>();
  const int tiles = ((m.max_n + 63) / 64) * ((m.max_n + 63) / 64);
  // C = op(A) diag(w) B over the entries of glist (systems or channels); each
  // operand has its own offset array (channel matrices at ch_mat, the
  // system-level orthogonaliser at ch_xoff).
  auto gemm = [&](const int32_t* glist, const double* A, const int64_t* offA, const double* Bm,
                  const int64_t* offB, double* C, const int32_t* dm, const int32_t* dn,
                  const int32_t* dk, bool ta, const double* w, int count, bool sym = false,
                  const uint8_t* prec = nullptr, cudaStream_t st = nullptr,
                  const uint8_t* only = nullptr) {
    GemmArgs g{};
    g.fault = m.umma_fault.as<int32_t>();
    g.sym = sym ? 1 : 0;
    g.only = only;
    g.prec = prec;
    g.prec_of = m.ch_sys.as<int32_t>();
    g.list = glist;
    g.nao = dch_nao;
    g.dm = dm;
    g.dn = dn;
    g.dk = dk;
    g.A = A;
    g.offA = offA;
    g.B = Bm;
    g.offB = offB;
    g.C = C;
    g.offC = dch_mat;
    g.w = w;
    g.offW = dch_ao;
    cudaStream_t gs = st != nullptr ? st : s;
    // Tile width autotuner (FP64 products only: the two widths form every
    // element identically, so the choice never changes a result).  The first
    // product of each kind, size bucket and count class in an eager
    // iteration runs both widths twice, timed by events, and the faster one
    // is kept for this context; captured iterations only reuse choices.
    int width = 0;
    if (prec == nullptr && m.forced_gemm_width != 0) {
      width = m.forced_gemm_width;
    } else if (prec == nullptr && count > 0) {
      const int lg = 31 - __builtin_clz((unsigned)count);
      const int32_t* nv = m.nvec.as<int32_t>();
      const uint64_t key = ((uint64_t)((m.max_n + 31) / 32) << 32) | ((uint64_t)lg << 8) |
                           (uint64_t)(ta ? 1 : 0) | ((uint64_t)(w != nullptr) << 1) |
                           ((uint64_t)(sym ? 1 : 0) << 2) | ((uint64_t)(dk == nv) << 3) |
                           ((uint64_t)(dm == nv) << 4);
      const auto it = m.gemm_width.find(key);
      if (it != m.gemm_width.end()) {
        width = it->second;
      } else {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(gs, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
          width = tune_gemm_width(g, ta, w != nullptr, tiles, count, gs);
          if (width != 0) m.gemm_width.emplace(key, width);
        }
      }
    }
    launch_gemm(g, ta, w != nullptr, tiles, count, gs, width);
  };
  const int32_t* dnao = dch_nao;
  const int32_t* dnvec = m.nvec.as<int32_t>();

  // AO-count buckets of the (n-descending) active list: each bucket gets its
  // own launch geometry and shared-memory footprint.
  if (m.h_list_cap < B) {
    if (m.h_list) cudaFreeHost(m.h_list);
    cudaMallocHost(&m.h_list, B * sizeof(int32_t));
    m.h_list_cap = B;
  }
  struct Bucket {
    int start, count, max_n, max_m;
  };
  auto buckets = [&](const int32_t* hl, int count) {
    static const int kEdges[] = {230, 192, 160, 128, 96, 64, 0};
    std::vector<Bucket> out;
    int i = 0;
    if (count <= 296) {
      // at most two waves: one launch, so few large systems run concurrently
      Bucket bk{0, count, count > 0 ? m.h_ch_nao[hl[0]] : 0, 0};
      for (int k = 0; k < count; ++k) {
        const int c = hl[k];
        bk.max_m = std::max(bk.max_m, (int)std::ceil(std::max(m.h_ch_nel_a[c], m.h_ch_nel_b[c])) + 4);
      }
      if (count > 0) out.push_back(bk);
      return out;
    }
    while (i < count) {
      const int n0 = m.h_ch_nao[hl[i]];
      int lo_edge = 0;
      for (int e : kEdges)
        if (n0 > e) { lo_edge = e; break; }
      Bucket bk{i, 0, n0, 0};
      while (i < count && m.h_ch_nao[hl[i]] > lo_edge) {
        const int c = hl[i];
        bk.max_m = std::max(bk.max_m, (int)std::ceil(std::max(m.h_ch_nel_a[c], m.h_ch_nel_b[c])) + 4);
        ++bk.count;
        ++i;
      }
      out.push_back(bk);
    }
    return out;
  };
  // tridiagonalise, eigenvalues (+ occupations), eigenvectors, back-transform
  // over the entries of dl (device) / hl (its host copy), systems or channels
  // mode 0: SCC, the occupied vectors; 1: all vectors, no occupations
  // (overlap); 2: SCC, all vectors (they seed the warm-started refinement).
  // only: per-channel mask of the entries to solve (NULL: every entry).
  auto eigensolve = [&](const int32_t* dl, const int32_t* hl, int count, int mode, double kt,
                        double ortol_rel, int stage_base, const uint8_t* only = nullptr) {
    const std::vector<Bucket> bks = buckets(hl, count);
    auto sub = [&](const Bucket& bk) {
      EigArgs gb = eg;
      gb.list = dl + bk.start;
      gb.only = only;
      gb.all_vectors = mode != 0 ? 1 : 0;
      return gb;
    };
    auto tridiag = [&](const Bucket& bk, cudaStream_t st) {
      const EigArgs gb = sub(bk);
      // few systems: register-resident cluster kernel (latency); many: the
      // shared-memory kernel, one CTA per system (throughput)
      if (bk.max_n <= tridiag_reg_max_n() && bk.count * 8 <= sm_count() && !m.tridiag_smem)
        launch_tridiag_reg(gb, gb.list, bk.count, bk.max_n, st);
      else
        launch_tridiag_smem(gb, gb.list, bk.count, bk.max_n, st);
    };
    auto eigvals = [&](const Bucket& bk, cudaStream_t st) {
      // levels_needed: ceil(max(nel_a, nel_b)) + 8 = bk.max_m + 4
      launch_eigvals(sub(bk), mode, kt, bk.count, bk.max_n, bk.max_m + 4, st);
    };
    auto invit = [&](const Bucket& bk, cudaStream_t st) {
      launch_inverse_iteration(sub(bk), bk.count, bk.max_n,
                               mode != 0 ? bk.max_n : std::min(bk.max_m + 4, bk.max_n), ortol_rel, st);
    };
    auto wy_cap = [&](const Bucket& bk) {
      const int want = mode != 0 ? bk.max_n : std::min(bk.max_m, bk.max_n);
      const long budget = 220L * 1024 / 8 - (long)bk.max_n * 33 - 32 * 33 - 8;
      return (int)std::min<long>(want, budget / 32);
    };
    // factored: the T factors were launched already (launch_wy_factor)
    auto backtransform = [&](const Bucket& bk, cudaStream_t st, bool factored = false) {
      const EigArgs gb = sub(bk);
      const int want = mode != 0 ? bk.max_n : std::min(bk.max_m, bk.max_n);
      const int wcap = wy_cap(bk);
      if (wcap >= 8) {
        launch_backtransform_wy(gb, bk.count, bk.max_n, wcap, want, st, factored);
      } else {
        // a block of reflectors no longer fits in shared memory: row chunks
        launch_backtransform_rows(gb, bk.count, bk.max_n, want, st);
      }
    };
    if (!bks.empty() && !m.prof.on && m.ensure_bucket_streams()) {
      // Each bucket runs its whole chain on its own side stream, forked from
      // and joined back into the call's stream (also inside graph capture);
      // its WY T factors run on a second stream from the tridiagonalisation
      // on, beside the eigenvalues and the inverse iteration, and join before
      // the back-transform.
      cudaEventRecord(m.bfork, s);
      const int ns = std::min<int>((int)bks.size(), Impl::kBucketStreams);
      for (int i = 0; i < ns; ++i) cudaStreamWaitEvent(m.bst[i], m.bfork, 0);
      for (size_t i = 0; i < bks.size(); ++i) {
        const int k = (int)(i % Impl::kBucketStreams);
        cudaStream_t st = m.bst[k];
        tridiag(bks[i], st);
        const bool fork = wy_cap(bks[i]) >= 8;
        if (fork) {
          cudaEventRecord(m.ffork[k], st);
          cudaStreamWaitEvent(m.fst[k], m.ffork[k], 0);
          launch_wy_factor(sub(bks[i]), bks[i].count, bks[i].max_n, m.fst[k]);
          cudaEventRecord(m.wydone[k], m.fst[k]);
        }
        eigvals(bks[i], st);
        invit(bks[i], st);
        if (fork) cudaStreamWaitEvent(st, m.wydone[k], 0);
        backtransform(bks[i], st, fork);
      }
      for (int i = 0; i < ns; ++i) {
        cudaEventRecord(m.bjoin[i], m.bst[i]);
        cudaStreamWaitEvent(s, m.bjoin[i], 0);
      }
      m.prof.launches += 4 * (int)bks.size();
      if (const cudaError_t le = cudaGetLastError(); le != cudaSuccess && !launch_error) launch_error = le;
      return;
    }
    XTB_STAGE(stage_base == kStLowdin ? kStLowdin : kStTridiag, (int)bks.size(),
              for (const Bucket& bk : bks) tridiag(bk, s));
    XTB_STAGE(stage_base == kStLowdin ? kStLowdin : kStEigvals, (int)bks.size(),
              for (const Bucket& bk : bks) eigvals(bk, s));
    XTB_STAGE(stage_base == kStLowdin ? kStLowdin : kStInvIter, (int)bks.size(),
              for (const Bucket& bk : bks) invit(bk, s));
    XTB_STAGE(stage_base == kStLowdin ? kStLowdin : kStBacktransform, (int)bks.size(),
              for (const Bucket& bk : bks) backtransform(bk, s));
  };

  // ---- Loewdin orthogonaliser X = U s^-1/2 U^T ----
  cudaMemcpyAsync(m.A.p, m.S.p, (size_t)m.total_mat * 8, cudaMemcpyDeviceToDevice, s);
  std::memcpy(m.h_list, m.h_order.data(), B * sizeof(int32_t));
  eigensolve(list, m.h_list, nsys, 1, 0.0, 2e-6, kStLowdin);
  XTB_STAGE(kStLowdin, 2, launch_lowdin_weights(eg, status, nsys, s);
            gemm(list, m.Zv.as<double>(), dch_mat, m.Zv.as<double>(), dch_mat, m.X.as<double>(),
                 dnao, dnao, dnao, true, m.occ.as<double>(), nsys, true));

  // ---- SCC ----
  SccArgs a{};
  a.t = t;
  a.list = list;
  a.qsh = m.qsh.as<double>();
  a.dip = m.dip.as<double>();
  a.qp = m.qp.as<double>();
  a.pop_sh = m.pop_sh.as<double>();
  a.pop_dip = m.pop_dip.as<double>();
  a.pop_qp = m.pop_qp.as<double>();
  a.e_core = m.e_core.as<double>();
  a.vsh = m.vsh.as<double>();
  a.vd = m.vd.as<double>();
  a.vq = m.vq.as<double>();
  a.gam = m.gam.as<double>();
  a.mrad = m.mrad.as<double>();
  a.cn_d4 = m.cn_d4.as<double>();
  a.S = m.S.as<double>();
  a.D = m.D.as<double>();
  a.Q = m.Q.as<double>();
  a.H0 = m.H0.as<double>();
  a.H = m.H.as<double>();
  a.P = m.P.as<double>();
  a.total_mat = m.total_mat;
  a.pot_acc = m.pot_acc.as<double>();
  a.entropy = m.entropy.as<double>();
  a.free_energy = m.free_energy.as<double>();
  a.terms = m.terms.as<double>();
  a.iterations = m.iterations.as<int32_t>();
  a.status = status;
  a.converged = m.converged.as<uint8_t>();
  a.mx_cur = m.mx_cur.as<double>();
  a.mx_prev = m.mx_prev.as<double>();
  a.mx_res = m.mx_res.as<double>();
  a.mx_df = m.mx_df.as<double>();
  a.mx_u = m.mx_u.as<double>();
  a.mx_omega = m.mx_omega.as<double>();
  a.memory = M;
  a.damping = req.damping;
  a.ctol = req.ctol;
  a.etol = req.etol;
  a.kt = req.kt;
  a.max_iter = req.max_iter;
  a.prec = m.mixed ? m.prec.as<uint8_t>() : nullptr;
  a.prec_switch = m.prec_switch;
  a.split_iters = m.split_iters.as<int32_t>();
  a.gate_hits = m.mixed ? m.gate_hits.as<int32_t>() : nullptr;
  a.last_rms = m.last_rms.as<double>();
  const uint8_t* sprec = a.prec;   // split-precision selector of the SCC GEMMs
  a.qmag = m.qmag.as<double>();
  a.vmag = m.vmag.as<double>();
  a.pop_mag = m.pop_mag.as<double>();
  a.pop_mdip = m.pop_mdip.as<double>();
  a.pop_mqp = m.pop_mqp.as<double>();
  a.Pm = m.Pm.as<double>();
  a.work = m.scratch.as<double>();
  a.work_off = m.ch_scr.as<int64_t>();
  a.ch_sys = m.ch_sys.as<int32_t>();
  a.ch_sign = m.ch_sign.as<int32_t>();
  a.ch_mat = dch_mat;
  // Spin channels of the active list: without unrestricted systems the channel
  // list is the system list itself.
  const bool have_uhf = m.nuhf > 0;
  int32_t* clist = have_uhf ? m.clist.as<int32_t>() : list;
  int32_t* dccount = have_uhf ? m.ccount.as<int32_t>() : dcount;
  int32_t* h_cl = have_uhf ? m.h_clist : m.h_list;
  a.clist = clist;
  auto channels = [&](cudaStream_t st) {
    if (!have_uhf) return;
    k_channels<<<1, 1024, 0, st>>>(list, dcount, m.beta_ch.as<int32_t>(), clist, dccount);
    m.prof.launches += 1;
    cudaMemcpyAsync(m.h_count + 2, dccount, 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(h_cl, clist, (size_t)m.nchan * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  };
  auto channel_count = [&]() { return have_uhf ? m.h_count[2] : m.h_count[0]; };
  // totals alpha + beta (and P_alpha - P_beta) of the unrestricted systems
  auto combine = [&](double* M, double* Pm, int cnt, cudaStream_t st) {
    if (!have_uhf || cnt == 0) return;
    const int per = std::max(1, std::min(64, (m.max_n * m.max_n + 255) / 256));
    k_combine_spin<<<dim3(per, cnt), 256, 0, st>>>(list, m.beta_ch.as<int32_t>(), m.nao.as<int32_t>(),
                                                    m.mat_off.as<int64_t>(), dch_mat, M, Pm);
    m.prof.launches += 1;
  };

  XTB_STAGE(kStCompact, 1,
            launch_compact(order, nsys, status, a.converged, a.iterations, req.max_iter, list,
                           dcount, s));
  cudaMemcpyAsync(m.h_count, dcount, 4, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(m.h_list, list, B * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  channels(s);
  cudaStreamSynchronize(s);
  int count = m.h_count[0];
  int ccount = channel_count();
  a.count = count;
  a.ccount = ccount;
  a.ck_qsh = m.ck_qsh.as<double>();
  a.ck_dip = m.ck_dip.as<double>();
  a.ck_qp = m.ck_qp.as<double>();
  a.ck_qmag = m.ck_qmag.as<double>();
  a.ck_mdip = m.ck_mdip.as<double>();
  a.ck_mqp = m.ck_mqp.as<double>();
  if (warm)
    XTB_STAGE(kStPotential, 1, launch_warm_init(a, s));
  else
    XTB_STAGE(kStPotential, 1, launch_sad_init(a, s));
  // ---- energy and force terms of converged systems ----
  const bool want_forces = (req.flags & XTBLOOM_COMPUTE_FORCES) != 0;
  const bool want_pcf = (req.flags & XTBLOOM_COMPUTE_POINT_CHARGE_FORCES) != 0;
  ForceArgs fbase{};
  fbase.t = t;
  fbase.cn = m.cn.as<double>();
  fbase.cn_d4 = m.cn_d4.as<double>();
  fbase.mrad = m.mrad.as<double>();
  fbase.dmrad = m.dmrad.as<double>();
  fbase.S = m.S.as<double>();
  fbase.P = m.P.as<double>();
  fbase.W = m.W.as<double>();
  fbase.vsh = m.vsh.as<double>();
  fbase.vd = m.vd.as<double>();
  fbase.vq = m.vq.as<double>();
  fbase.vmag = m.vmag.as<double>();
  fbase.Pm = m.Pm.as<double>();
  fbase.qsh = m.qsh.as<double>();
  fbase.dip = m.dip.as<double>();
  fbase.qp = m.qp.as<double>();
  fbase.gam = m.gam.as<double>();
  fbase.grad = m.grad.as<double>();
  fbase.acn = m.acn.as<double>();
  fbase.acn_d4 = m.acn_d4.as<double>();
  fbase.terms = m.terms.as<double>();
  fbase.want_grad = want_forces ? 1 : 0;
  fbase.atm_c6 = m.T.as<double>();      // free once the SCC has ended
  fbase.atm_dc6 = m.A.as<double>();
  fbase.work = m.scratch.as<double>();
  fbase.work_off = m.ch_scr.as<int64_t>();
  // Warm-started eigensolver state (k_refine.cu)
  const bool refine = m.refine_steps > 0;
  uint8_t* m_step = m.m_step.as<uint8_t>();
  uint8_t* m_apply = m.m_apply.as<uint8_t>();
  uint8_t* m_cold = m.m_cold.as<uint8_t>();
  uint8_t* m_warm = m.m_warm.as<uint8_t>();
  RefineArgs rbase{};
  rbase.nao = dch_nao;
  rbase.mat_off = dch_mat;
  rbase.ao_off = dch_ao;
  rbase.ch_sys = m.ch_sys.as<int32_t>();
  rbase.nel_a = m.ch_nel_a.as<double>();
  rbase.nel_b = m.ch_nel_b.as<double>();
  rbase.kt = req.kt;
  rbase.occ = m.occ.as<double>();
  rbase.occ_eps = m.occ_eps.as<double>();
  rbase.nvec = m.nvec.as<int32_t>();
  rbase.entropy = m.entropy.as<double>();
  rbase.bounds = m.w_bounds.as<double>();
  rbase.Sm = m.W.as<double>();
  rbase.G = m.C.as<double>();
  rbase.Ep = m.P.as<double>();
  rbase.V = m.Vw.as<double>();
  rbase.Vt = m.Vt.as<double>();
  rbase.Zrows = m.Zv.as<double>();
  rbase.eig = m.eig.as<double>();
  rbase.wstate = m.wstate.as<uint8_t>();
  rbase.phase = m.wphase.as<uint8_t>();
  rbase.m_step = m_step;
  rbase.m_apply = m_apply;
  rbase.m_cold = m_cold;
  rbase.m_warm = m_warm;
  rbase.emax = m.w_emax.as<unsigned long long>();
  rbase.fail = m.w_fail.as<int32_t>();
  rbase.arrive = m.w_arrive.as<int32_t>();
  rbase.stats = m.w_stats.as<int32_t>();
  rbase.iterations = m.iterations.as<int32_t>();
  rbase.prec = sprec;
  rbase.warm_from = m.refine_from;
  rbase.theta = m.refine_theta;
  rbase.theta_split = m.refine_theta_split;
  rbase.theta_final = m.refine_theta_final;
  rbase.final_rms = m.refine_final_factor * req.ctol;
  rbase.last_rms = m.last_rms.as<double>();
  // CTAs per channel of the correction kernel: one with many channels, up to
  // 16 when few are left (the non-converging tail), where it is on the
  // critical path
  auto refine_parts = [&](int cnt) {
    const int sms = sm_count();
    if (cnt >= sms) return 1;
    return std::max(1, std::min(16, (2 * sms) / std::max(cnt, 1)));
  };

  // Every kernel here reads and writes only the listed systems' slices.
  auto force_terms = [&](const int32_t* flist, int fcount, cudaStream_t st) {
    if (fcount <= 0) return;
    ForceArgs f = fbase;
    f.list = flist;
    f.count = fcount;
    SccArgs af = a;
    af.list = flist;
    af.count = fcount;
    if (want_forces) {
      // energy-weighted density per spin channel, then the alpha + beta totals
      int fcc = fcount;
      if (have_uhf) {
        channels(st);
        cudaStreamSynchronize(st);
        fcc = channel_count();
      } else if (refine) {
        cudaMemcpyAsync(m.h_list, flist, (size_t)fcount * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
      }
      if (refine) {
        // The energy-weighted density needs the eigenpairs of the last
        // iteration; a channel that ended refined has its occupied subspace
        // but not the individual levels, so its matrix A (kept) is solved
        // once more on the Householder path, and C formed from those vectors.
        eigensolve(clist, h_cl, fcc, 0, req.kt, 2e-7, kStTridiag, m_warm);
        XTB_STAGE_ON(st, kStDensity, 1,
                     gemm(clist, m.Zv.as<double>(), dch_mat, m.X.as<double>(), dch_xoff, m.C.as<double>(),
                          dnvec, dnao, dnao, false, nullptr, fcc, false, nullptr, st, m_warm));
      }
      XTB_STAGE_ON(st, kStForcePairs, 3,
                   launch_potential(af, af.qsh, af.dip, af.qp, m.max_atoms, m.max_shells, st);
                   gemm(clist, m.C.as<double>(), dch_mat, m.C.as<double>(), dch_mat, m.W.as<double>(),
                        dnao, dnao, dnvec, true, m.occ_eps.as<double>(), fcc, true, nullptr, st);
                   combine(m.W.as<double>(), nullptr, fcount, st);
                   launch_force_pairs(f, m.max_pairs, st));
    }
    XTB_STAGE_ON(st, kStClassical, 1, launch_classical(f, m.max_atoms, m.max_shells, st));
    if (want_forces) XTB_STAGE_ON(st, kStCnChain, 2, launch_cn_chain(f, m.max_atoms, st));
    if (m.have_pc && (want_forces || want_pcf))
      XTB_STAGE_ON(st, kStClassical, 1,
                   launch_pc_forces(t, flist, fcount, m.qsh.as<double>(), m.grad.as<double>(),
                                    m.pc_grad.as<double>(), m.pc_dq.as<double>(), st));
  };


  // One SCC iteration over the current active list (a.count systems): every
  // launch of it, ending with the compaction of the list and the copies of
  // the new count and list into pinned host memory.
  auto iteration = [&](int it) {
    XTB_STAGE(kStPotential, 1, launch_potential(a, a.qsh, a.dip, a.qp, m.max_atoms, m.max_shells, s));
    XTB_STAGE(kStFock, 1, launch_fock(a, m.max_n, s));
    XTB_STAGE(kStTransform, 2,
              gemm(clist, m.H.as<double>(), dch_mat, m.X.as<double>(), dch_xoff, m.T.as<double>(),
                   dnao, dnao, dnao, false, nullptr, a.ccount, false, sprec);
              gemm(clist, m.X.as<double>(), dch_xoff, m.T.as<double>(), dch_mat, m.A.as<double>(),
                   dnao, dnao, dnao, false, nullptr, a.ccount, true, sprec));
    if (refine) {
      // Warm-started refinement first (it reads A, which the Householder path
      // then overwrites for the channels it solves); U = A V goes to T, the
      // products V^T U and V^T V to W and C, the correction I + E to P and
      // V (I + E) to Vt: all free at this point of the iteration.
      RefineArgs ra = rbase;
      ra.list = clist;
      ra.count = a.ccount;
      XTB_STAGE(kStRefine, 1, launch_warm_begin(ra, s));
      for (int k = 0; k < m.refine_steps; ++k) {
        ra.step = k;
        XTB_STAGE(kStRefine, 6,
                  gemm(clist, m.A.as<double>(), dch_mat, m.Vw.as<double>(), dch_mat, m.T.as<double>(),
                       dnao, dnao, dnao, false, nullptr, a.ccount, false, sprec, s, m_step);
                  gemm(clist, m.Vw.as<double>(), dch_mat, m.T.as<double>(), dch_mat, m.W.as<double>(),
                       dnao, dnao, dnao, true, nullptr, a.ccount, true, sprec, s, m_step);
                  gemm(clist, m.Vw.as<double>(), dch_mat, m.Vw.as<double>(), dch_mat, m.C.as<double>(),
                       dnao, dnao, dnao, true, nullptr, a.ccount, true, sprec, s, m_step);
                  launch_refine_update(ra, m.max_n, refine_parts(a.ccount), s);
                  gemm(clist, m.Vw.as<double>(), dch_mat, m.P.as<double>(), dch_mat, m.Vt.as<double>(),
                       dnao, dnao, dnao, false, nullptr, a.ccount, false, sprec, s, m_apply);
                  launch_refine_apply(ra, m.max_n, k + 1 == m.refine_steps, s));
      }
      eigensolve(clist, h_cl, a.ccount, 2, req.kt, 2e-7, kStTridiag, m_cold);
      XTB_STAGE(kStRefine, 1, launch_vectors_from_rows(ra, m.max_n, s));
    } else {
      eigensolve(clist, h_cl, a.ccount, 0, req.kt, 2e-7, kStTridiag);
    }
    XTB_STAGE(kStDensity, 2,
              if (refine)
                gemm(clist, m.Vw.as<double>(), dch_mat, m.X.as<double>(), dch_xoff, m.C.as<double>(),
                     dnvec, dnao, dnao, true, nullptr, a.ccount, false, sprec);
              else
                gemm(clist, m.Zv.as<double>(), dch_mat, m.X.as<double>(), dch_xoff, m.C.as<double>(),
                     dnvec, dnao, dnao, false, nullptr, a.ccount, false, sprec);
              gemm(clist, m.C.as<double>(), dch_mat, m.C.as<double>(), dch_mat, m.P.as<double>(),
                   dnao, dnao, dnvec, true, m.occ.as<double>(), a.ccount, true, sprec);
              combine(m.P.as<double>(), m.Pm.as<double>(), a.count, s));
    XTB_STAGE(kStMulliken, 1, launch_mulliken(a, m.max_n, s));
    XTB_STAGE(kStEnergyMixer, 1, launch_energy_mixer(a, m.max_atoms, m.max_shells, m.max_dim, it == 0, s));
    XTB_STAGE(kStCompact, 1,
              launch_compact(order, nsys, status, a.converged, a.iterations, req.max_iter, list,
                             dcount, s));
    cudaMemcpyAsync(m.h_count, dcount, 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(m.h_list, list, B * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    channels(s);
  };
  // Graph replay: while the active set is unchanged (same count, hence the
  // same list), the iteration's launches are identical; the iteration is
  // captured once into a CUDA graph and replayed.  Not combined with the
  // per-stage timing events.
  cudaGraphExec_t gexec = nullptr;
  int graph_count = -1, prev_count = -1;
  int64_t graph_launches = 0;
  bool graphs_ok = m.graphs && !m.prof.on;
  for (int it = 0; it < req.max_iter && count > 0; ++it) {
    a.count = count;
    a.ccount = ccount;
    bool ran = false;
    if (graphs_ok && count == prev_count) {
      if (gexec == nullptr || graph_count != count) {
        if (gexec) cudaGraphExecDestroy(gexec);
        gexec = nullptr;
        const int64_t l0 = m.prof.launches;
        cudaGraph_t graph = nullptr;
        const cudaError_t le0 = launch_error;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
          iteration(it);
          const cudaError_t ce = cudaStreamEndCapture(s, &graph);
          if (ce == cudaSuccess && graph != nullptr &&
              cudaGraphInstantiate(&gexec, graph, 0) == cudaSuccess) {
            graph_count = count;
            graph_launches = m.prof.launches - l0;
          } else {
            gexec = nullptr;
            graphs_ok = false;   // capture failed: this call continues eagerly
          }
          if (graph) cudaGraphDestroy(graph);
        } else {
          graphs_ok = false;
        }
        m.prof.launches = l0;
        if (gexec == nullptr) launch_error = le0;   // nothing of the failed capture ran
        (void)cudaGetLastError();
      }
      if (gexec != nullptr && cudaGraphLaunch(gexec, s) == cudaSuccess) {
        m.prof.launches += graph_launches;
        ran = true;
      }
    }
    if (!ran) iteration(it);
    prev_count = count;
    cudaStreamSynchronize(s);
    if (m.trace) {
      std::fprintf(stderr, "[xtbloom_b200] iteration %d active %d -> %d  t=%.3f ms%s\n", it, a.count,
                   m.h_count[0],
                   std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count(),
                   ran ? " (graph)" : "");
    }
    count = m.h_count[0];
    ccount = channel_count();
    if (launch_error) break;
  }
  if (gexec) cudaGraphExecDestroy(gexec);
  k_finalize_status<<<(nsys + 255) / 256, 256, 0, s>>>(nsys, status, a.converged);
  m.prof.launches += 1;

  // ---- energy and force terms of the converged systems ----
  k_list_ready<<<1, 1024, 0, s>>>(order, nsys, status, a.converged, m.fdone.as<uint8_t>(), list,
                                  dcount);
  m.prof.launches += 1;
  cudaMemcpyAsync(m.h_count, dcount, 4, cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  count = m.h_count[0];
  force_terms(list, count, s);
  if (m.have_pc && want_pcf)
    XTB_STAGE(kStPublish, 1,
              launch_pc_publish(t, status, nsys, m.pc_grad.as<double>(), m.out_pcf.as<double>(), s));
  XTB_STAGE(kStPublish, 1,
            k_publish<<<nsys, 128, 0, s>>>(t, status, m.free_energy.as<double>(),
                                           m.terms.as<double>(), m.grad.as<double>(),
                                           m.qsh.as<double>(), m.dip.as<double>(),
                                           m.out_energy.as<double>(), m.out_forces.as<double>(),
                                           m.out_charges.as<double>(), m.out_dipoles.as<double>()));
#undef XTB_STAGE
#undef XTB_STAGE_ON
  if (launch_error == cudaSuccess) launch_error = cudaGetLastError();
  if (launch_error != cudaSuccess) {
    cudaStreamSynchronize(s);
    error = std::string("kernel launch failed: ") + cudaGetErrorString(launch_error);
    return XTBLOOM_STATUS_INTERNAL_ERROR;
  }
  if (m.mixed) {
    cudaMemcpyAsync(m.h_count + 3, m.umma_fault.p, 4, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    if (m.h_count[3] != 0) {
      error = "a tensor-core product of the split-precision form did not complete in time";
      return XTBLOOM_STATUS_INTERNAL_ERROR;
    }
  }
  // ---- copy into caller buffers ----
  const xtbloom_batch_result_t& r = *req.result;
  auto put = [&](const xtbloom_buffer_t& dst, const void* src, size_t bytes) {
    if (!dst.data || bytes == 0) return cudaSuccess;
    const cudaMemcpyKind kind =
        dst.memory_space == XTBLOOM_MEMORY_CUDA_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    return cudaMemcpyAsync(dst.data, src, bytes, kind, s);
  };
  if (req.flags & XTBLOOM_COMPUTE_ENERGY) put(r.energies, m.out_energy.p, B * 8);
  if (req.flags & XTBLOOM_COMPUTE_FORCES) put(r.forces, m.out_forces.p, 3 * N * 8);
  if (req.flags & XTBLOOM_COMPUTE_ATOMIC_CHARGES) put(r.atomic_charges, m.out_charges.p, N * 8);
  if (req.flags & XTBLOOM_COMPUTE_DIPOLE_MOMENTS) put(r.dipole_moments, m.out_dipoles.p, B * 24);
  if ((req.flags & XTBLOOM_COMPUTE_POINT_CHARGE_FORCES) && m.have_pc)
    put(r.point_charge_forces, m.out_pcf.p, (size_t)m.npc * 24);
  put(r.scc_iterations, m.iterations.p, B * 4);
  put(r.scc_converged, m.converged.p, B);
  put(r.per_system_status, status, B * 4);
  // a fully converged call leaves its converged state as the WARM checkpoint
  const bool fully_converged = count == nsys;
  if (fully_converged) {
    const size_t sh = (size_t)m.nshells * 8, at = (size_t)N * 8;
    const bool ok = m.ck_qsh.reserve(sh) && m.ck_dip.reserve(3 * at) && m.ck_qp.reserve(6 * at) &&
                    m.ck_qmag.reserve(sh) && m.ck_mdip.reserve(3 * at) && m.ck_mqp.reserve(6 * at) &&
                    cudaMemcpyAsync(m.ck_qsh.p, m.qsh.p, sh, cudaMemcpyDeviceToDevice, s) == cudaSuccess &&
                    cudaMemcpyAsync(m.ck_dip.p, m.dip.p, 3 * at, cudaMemcpyDeviceToDevice, s) == cudaSuccess &&
                    cudaMemcpyAsync(m.ck_qp.p, m.qp.p, 6 * at, cudaMemcpyDeviceToDevice, s) == cudaSuccess &&
                    (m.nuhf == 0 ||
                     (cudaMemcpyAsync(m.ck_qmag.p, m.qmag.p, sh, cudaMemcpyDeviceToDevice, s) == cudaSuccess &&
                      cudaMemcpyAsync(m.ck_mdip.p, m.pop_mdip.p, 3 * at, cudaMemcpyDeviceToDevice, s) == cudaSuccess &&
                      cudaMemcpyAsync(m.ck_mqp.p, m.pop_mqp.p, 6 * at, cudaMemcpyDeviceToDevice, s) == cudaSuccess));
    if (!ok) (void)cudaGetLastError();
    m.ck_valid = ok;
    if (ok) m.ck_id = ident;
  }
  const cudaError_t ce = cudaStreamSynchronize(s);
  if (ce != cudaSuccess) {
    m.ck_valid = false;
    error = std::string("CUDA failure: ") + cudaGetErrorString(ce);
    return XTBLOOM_STATUS_INTERNAL_ERROR;
  }
  const cudaError_t le = cudaGetLastError();
  if (le != cudaSuccess) {
    m.ck_valid = false;
    error = std::string("CUDA launch failure: ") + cudaGetErrorString(le);
    return XTBLOOM_STATUS_INTERNAL_ERROR;
  }
  if (m.prof.on) m.prof.collect();
  m.have_results = true;
  return XTBLOOM_STATUS_SUCCESS;
}

namespace {

// FP64 issue-rate probe for the roofline's FP64 bound: every thread runs
// eight independent FMA chains (2 flops each per step); the sum is written
// only when it is impossible, so the compiler keeps every FMA.
__global__ void __launch_bounds__(256) k_fp64_peak(int steps, double seed, double* sink) {
  double a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + 1e-3 * (threadIdx.x + k);
  const double b = 1.0 - 1e-9, c = 1e-9;
  for (int i = 0; i < steps; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
  }
  double t = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) t += a[k];
  if (t == -12345.678) sink[0] = t;
}

}  // namespace

xtbloom_status_t Engine::debug_fetch(const std::string& name, int64_t system, double* out,
                                     size_t capacity, size_t* count, std::string& error) {
  Impl& m = *impl_;
  if (name == "kernel_timing_on" || name == "kernel_timing_off") {
    // per-stage CUDA-event timing of later computes (graph replay is off while on)
    m.prof.on = name == "kernel_timing_on";
    *count = 0;
    return XTBLOOM_STATUS_SUCCESS;
  }
  if (name == "kernel_times" || name == "launch_count" || name == "reset_counters") {
    // Accumulated since the last reset: [ms, calls] per stage, or total launches.
    if (name == "reset_counters") {
      for (int i = 0; i < kStageCount; ++i) {
        m.prof.total_ms[i] = 0.0;
        m.prof.calls[i] = 0;
      }
      m.prof.launches = 0;
      *count = 0;
      return XTBLOOM_STATUS_SUCCESS;
    }
    const size_t len = name == "launch_count" ? 2 : 2 * (size_t)kStageCount;
    if (capacity < len) {
      error = "capacity too small";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    if (name == "launch_count") {
      out[0] = (double)m.prof.launches;
      out[1] = m.prof.on ? 1.0 : 0.0;
    } else {
      for (int i = 0; i < kStageCount; ++i) {
        out[2 * i] = m.prof.total_ms[i];
        out[2 * i + 1] = (double)m.prof.calls[i];
      }
    }
    *count = len;
    return XTBLOOM_STATUS_SUCCESS;
  }
  if (name == "split_iterations" && system == -1) {
    // the whole batch: SCC iterations each system ran with split-precision GEMMs
    if (!m.have_results) {
      error = "no retained results";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    if (capacity < (size_t)m.nsys) {
      error = "capacity too small";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    cudaSetDevice(device_);
    std::vector<int32_t> v(m.nsys);
    if (cudaMemcpy(v.data(), m.split_iters.p, (size_t)m.nsys * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
      error = "device read failed";
      return XTBLOOM_STATUS_INTERNAL_ERROR;
    }
    for (int64_t i = 0; i < m.nsys; ++i) out[i] = (double)v[i];
    *count = (size_t)m.nsys;
    return XTBLOOM_STATUS_SUCCESS;
  }
  if (name == "fp64_peak") {
    // measured FP64 FMA throughput of this device in TFLOP/s (best of 3 runs
    // of 2 x 8 x steps flops per thread on every SM)
    if (capacity < 1) {
      error = "capacity too small";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    cudaSetDevice(device_);
    Dbuf sink;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!sink.reserve(64) || cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
      error = "failed to set up the FP64 probe";
      return XTBLOOM_STATUS_ALLOCATION_FAILED;
    }
    const int blocks = sm_count() * 8, steps = 1 << 14;
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
      cudaEventRecord(e0, stream_);
      k_fp64_peak<<<blocks, 256, 0, stream_>>>(steps, 1.0 + rep, sink.as<double>());
      cudaEventRecord(e1, stream_);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      const double tf = 2.0 * 8.0 * steps * (double)blocks * 256.0 / (ms * 1e-3) / 1e12;
      if (rep > 0) best = std::max(best, tf);   // the first run warms the clocks up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    out[0] = best;
    *count = 1;
    return XTBLOOM_STATUS_SUCCESS;
  }
  if (name == "refine_stats" && system == -1) {
    // per SCC iteration (256 rows of 8): channels that refined, finished at
    // step 1, 2, 3 or later, failed, unfinished (went to the Householder path)
    if (capacity < 256 * 8) {
      error = "capacity too small";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    cudaSetDevice(device_);
    std::vector<int32_t> v(256 * 8, 0);
    if (m.w_stats.p != nullptr &&
        cudaMemcpy(v.data(), m.w_stats.p, v.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
      error = "device read failed";
      return XTBLOOM_STATUS_INTERNAL_ERROR;
    }
    for (size_t i = 0; i < v.size(); ++i) out[i] = (double)v[i];
    *count = v.size();
    return XTBLOOM_STATUS_SUCCESS;
  }
  if (name == "point_charge_dq" && system == -1) {
    // the whole batch: dE/dQ for every point charge of the most recent call
    if (!m.have_results || !m.have_pc) {
      error = "the most recent compute had no point charges";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    if (capacity < (size_t)m.npc) {
      error = "capacity too small";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    cudaSetDevice(device_);
    if (cudaMemcpy(out, m.pc_dq.p, (size_t)m.npc * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
      error = "device read failed";
      return XTBLOOM_STATUS_INTERNAL_ERROR;
    }
    *count = (size_t)m.npc;
    return XTBLOOM_STATUS_SUCCESS;
  }
  if (!m.have_results || system < 0 || system >= m.nsys) {
    error = "no retained results for that system";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  cudaSetDevice(device_);
  const int64_t a0 = m.topo.atom_off[system], na = m.topo.atom_off[system + 1] - a0;
  std::vector<int64_t> mat_off(m.nsys + 1), ao_off(m.nsys + 1), sh_off(m.nsys + 1);
  cudaMemcpy(mat_off.data(), m.mat_off.p, (m.nsys + 1) * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(ao_off.data(), m.ao_off.p, (m.nsys + 1) * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(sh_off.data(), m.shell_off.p, (m.nsys + 1) * 8, cudaMemcpyDeviceToHost);
  const int64_t n = m.h_nao[system];
  const double* src = nullptr;
  size_t len = 0;
  if (name == "cn") { src = m.cn.as<double>() + a0; len = na; }
  else if (name == "cn_d4") { src = m.cn_d4.as<double>() + a0; len = na; }
  else if (name == "overlap") { src = m.S.as<double>() + mat_off[system]; len = n * n; }
  else if (name == "h0") { src = m.H0.as<double>() + mat_off[system]; len = n * n; }
  else if (name == "x") { src = m.X.as<double>() + mat_off[system]; len = n * n; }
  else if (name == "density") { src = m.P.as<double>() + mat_off[system]; len = n * n; }
  else if (name == "hamiltonian") { src = m.H.as<double>() + mat_off[system]; len = n * n; }
  else if (name == "eigenvalues") { src = m.eig.as<double>() + ao_off[system]; len = n; }
  else if (name == "occupations") { src = m.occ.as<double>() + ao_off[system]; len = n; }
  else if (name == "qsh") { src = m.qsh.as<double>() + sh_off[system]; len = sh_off[system + 1] - sh_off[system]; }
  else if (name == "dipoles") { src = m.dip.as<double>() + 3 * a0; len = 3 * na; }
  else if (name == "quadrupoles") { src = m.qp.as<double>() + 6 * a0; len = 6 * na; }
  else if (name == "point_charge_dq" || name == "point_charge_potential") {
    if (!m.have_pc) {
      error = "the most recent compute had no point charges";
      return XTBLOOM_STATUS_INVALID_ARGUMENT;
    }
    if (name == "point_charge_dq") {
      src = m.pc_dq.as<double>() + m.h_pc_off[system];
      len = m.h_pc_off[system + 1] - m.h_pc_off[system];
    } else {
      src = m.vpc.as<double>() + sh_off[system];
      len = sh_off[system + 1] - sh_off[system];
    }
  }
  else if (name == "energy_terms") { src = m.terms.as<double>() + kTermCount * system; len = kTermCount; }
  else if (name == "gradient") {
    // fixed-point accumulator (2^-40 units) to values
    if (capacity < 3 * (size_t)na) { error = "capacity too small"; return XTBLOOM_STATUS_INVALID_ARGUMENT; }
    std::vector<long long> raw(3 * na);
    cudaMemcpy(raw.data(), m.grad.as<double>() + 3 * a0, 3 * na * 8, cudaMemcpyDeviceToHost);
    for (int64_t k = 0; k < 3 * na; ++k) out[k] = (double)raw[k] / 1099511627776.0;
    *count = 3 * na;
    return XTBLOOM_STATUS_SUCCESS;
  }
  else if (name == "dipole_integrals") {
    if (capacity < 3 * (size_t)(n * n)) { error = "capacity too small"; return XTBLOOM_STATUS_INVALID_ARGUMENT; }
    for (int c = 0; c < 3; ++c)
      cudaMemcpy(out + c * n * n, m.D.as<double>() + c * m.total_mat + mat_off[system], n * n * 8, cudaMemcpyDeviceToHost);
    *count = 3 * n * n;
    return XTBLOOM_STATUS_SUCCESS;
  } else if (name == "quadrupole_integrals") {
    if (capacity < 6 * (size_t)(n * n)) { error = "capacity too small"; return XTBLOOM_STATUS_INVALID_ARGUMENT; }
    for (int c = 0; c < 6; ++c)
      cudaMemcpy(out + c * n * n, m.Q.as<double>() + c * m.total_mat + mat_off[system], n * n * 8, cudaMemcpyDeviceToHost);
    *count = 6 * n * n;
    return XTBLOOM_STATUS_SUCCESS;
  } else {
    error = "unknown diagnostics name";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  if (capacity < len) {
    error = "capacity too small";
    return XTBLOOM_STATUS_INVALID_ARGUMENT;
  }
  cudaMemcpy(out, src, len * 8, cudaMemcpyDeviceToHost);
  *count = len;
  return XTBLOOM_STATUS_SUCCESS;
}

}  // namespace xtb
