// External point charges embedding GFN2 and GFN1 systems (xTB's softened
// shell monopole coupling, model/gfn2/external_point_charges.cpp:277-490 and
// model/gfn1/external_point_charges.cpp:317-323 of the reference): for shell
// s on atom A and charge p,
//   K_sp = (|R_A - R_p|^2 + a_sp^2)^-1/2,
//   a_sp = 2 / (eta_s + gamma_p) (GFN2: arithmetic mean of the hardnesses),
//   a_sp = 1 / (2 eta_s) + 1 / (2 gamma_p) (GFN1: harmonic mean),
//   V_s = sum_p Q_p K_sp (fixed by the geometry, added to the shell potential
//   every SCC iteration),  E_pc = sum_s q_s V_s,
//   dE/dR_A = -sum_{s in A, p} q_s Q_p d_Ap K_sp^3,  dE/dR_p = -sum over A of the same,
//   dE/dQ_p = sum_s q_s K_sp.
// There is no charge-charge term and no direct field on atomic multipoles.
#include "kernels.cuh"

namespace xtb {

__device__ __forceinline__ double pc_kernel(const DevTopo& t, int64_t at, double eta, int64_t p,
                                            double& dx, double& dy, double& dz) {
  dx = t.pos[3 * at] - t.pc_pos[3 * p];
  dy = t.pos[3 * at + 1] - t.pc_pos[3 * p + 1];
  dz = t.pos[3 * at + 2] - t.pc_pos[3 * p + 2];
  const double a = t.m.gfn1 ? 0.5 / eta + 0.5 / t.pc_gam[p] : 2.0 / (eta + t.pc_gam[p]);
  return 1.0 / sqrt(dx * dx + dy * dy + dz * dz + a * a);
}

// One CTA per system: V_s for every shell.
__global__ void __launch_bounds__(128) k_pc_potential(DevTopo t, const int32_t* list, double* vpc) {
  const int s = list[blockIdx.x];
  const int64_t s0 = t.shell_off[s], s1 = t.shell_off[s + 1];
  const int64_t p0 = t.pc_off[s], p1 = t.pc_off[s + 1];
  for (int64_t sh = s0 + threadIdx.x; sh < s1; sh += blockDim.x) {
    const int64_t at = t.sh_atom[sh];
    const double eta = t.sh_eta[sh];
    double v = 0.0;
    for (int64_t p = p0; p < p1; ++p) {
      double dx, dy, dz;
      v = fma(t.pc_q[p], pc_kernel(t, at, eta, p, dx, dy, dz), v);
    }
    vpc[sh] = v;
  }
}

// One CTA per converged system: atom gradients (threads over shells, one
// atomic add per shell and component) and, per charge, dE/dR_p and dE/dQ_p
// (threads over charges, no atomics).
__global__ void __launch_bounds__(128) k_pc_forces(DevTopo t, const int32_t* list, const double* qsh,
                                                   double* grad, double* pc_grad, double* pc_dq) {
  const int s = list[blockIdx.x];
  const int64_t s0 = t.shell_off[s], s1 = t.shell_off[s + 1];
  const int64_t p0 = t.pc_off[s], p1 = t.pc_off[s + 1];
  for (int64_t sh = s0 + threadIdx.x; sh < s1; sh += blockDim.x) {
    const int64_t at = t.sh_atom[sh];
    const double eta = t.sh_eta[sh], q = qsh[sh];
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int64_t p = p0; p < p1; ++p) {
      double dx, dy, dz;
      const double k = pc_kernel(t, at, eta, p, dx, dy, dz);
      const double w = q * t.pc_q[p] * k * k * k;
      gx -= w * dx;
      gy -= w * dy;
      gz -= w * dz;
    }
    fix_add(&grad[3 * at], gx);
    fix_add(&grad[3 * at + 1], gy);
    fix_add(&grad[3 * at + 2], gz);
  }
  for (int64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
    double fx = 0.0, fy = 0.0, fz = 0.0, dq = 0.0;
    for (int64_t sh = s0; sh < s1; ++sh) {
      double dx, dy, dz;
      const double k = pc_kernel(t, t.sh_atom[sh], t.sh_eta[sh], p, dx, dy, dz);
      const double q = qsh[sh];
      const double w = q * t.pc_q[p] * k * k * k;
      fx += w * dx;
      fy += w * dy;
      fz += w * dz;
      dq = fma(q, k, dq);
    }
    pc_grad[3 * p] = fx;
    pc_grad[3 * p + 1] = fy;
    pc_grad[3 * p + 2] = fz;
    pc_dq[p] = dq;
  }
}

// Point-charge forces for the caller (quiet NaN for the charges of failed systems).
__global__ void k_pc_publish(DevTopo t, const int32_t* status, const double* pc_grad, double* out) {
  const int s = blockIdx.x;
  const bool ok = status[s] == kOk;
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  for (int64_t i = 3 * t.pc_off[s] + threadIdx.x; i < 3 * t.pc_off[s + 1]; i += blockDim.x)
    out[i] = ok ? -pc_grad[i] : nan;
}

void launch_pc_potential(const DevTopo& t, const int32_t* list, int count, double* vpc,
                         cudaStream_t stream) {
  if (count == 0) return;
  k_pc_potential<<<count, 128, 0, stream>>>(t, list, vpc);
}

void launch_pc_forces(const DevTopo& t, const int32_t* list, int count, const double* qsh,
                      double* grad, double* pc_grad, double* pc_dq, cudaStream_t stream) {
  if (count == 0) return;
  k_pc_forces<<<count, 128, 0, stream>>>(t, list, qsh, grad, pc_grad, pc_dq);
}

void launch_pc_publish(const DevTopo& t, const int32_t* status, int nsys, const double* pc_grad,
                       double* out, cudaStream_t stream) {
  if (nsys == 0) return;
  k_pc_publish<<<nsys, 128, 0, stream>>>(t, status, pc_grad, out);
}

}  // namespace xtb
