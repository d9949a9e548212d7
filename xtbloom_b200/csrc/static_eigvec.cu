// Eigenvectors of one symmetric tridiagonal matrix by inverse iteration, with
// no device allocation: the work vectors live in a fixed array in the
// library's own device memory instead of a cudaMalloc'd workspace.
//
// Who needs this: callers that must not allocate between set-up and tear-down.
// cudaMalloc and cudaFree may synchronise the whole device (stalling every
// other stream of a serving process mid-step), may fail once a caller's memory
// budget is committed, and an allocator that is not stream-ordered cannot be
// used inside a latency-critical loop at all.  Such a caller passes device
// buffers it owns already and gets the vectors back with nothing allocated.
//
// Limits and rules of use:
//   * n <= kStaticMaxN (256): the scratch is 5 * 256 * 128 doubles (1.25 MiB),
//     one copy per device; larger matrices are rejected before any launch.
//   * Nothing in the scratch has to start at zero: the kernel writes every
//     element it reads, so the array is never cleared between calls.
//   * One call at a time per device: two calls in flight together (on two
//     streams, or from two host threads) share the one scratch array and
//     overwrite each other's work vectors.  Serialise them on one stream or
//     with events.
//   * The first call on each device resolves the scratch address
//     (cudaGetSymbolAddress, which can load the module), so it belongs in
//     the caller's set-up.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "inverse_iteration.cuh"
#include "static_eigvec.h"

namespace xtb {
namespace {

constexpr int kThreads = 128;
constexpr int64_t kScratchDoubles = 5LL * kStaticMaxN * kThreads;

static __device__ __align__(256) double g_static_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

__global__ void __launch_bounds__(kThreads)
    k_inverse_iteration_static(const double* d, const double* e, const double* ev, int n, int m,
                               double* Z, double* scratch, double ortol_rel) {
  inverse_iteration_block<kThreads>(d, e, ev, n, m, Z, scratch, ortol_rel, 0u, 0, kThreads);
}

}  // namespace

int static_eigvec_run(const double* d, const double* e, const double* ev, int n, int m, double* Z,
                      double ortol_rel, cudaStream_t stream, std::string& err) {
  if (n < 1 || n > kStaticMaxN) {
    err = "n = " + std::to_string(n) + " is outside 1.." + std::to_string(kStaticMaxN) +
          ", the size of the static scratch";
    return 1;
  }
  if (m < 0 || m > n) {
    err = "m = " + std::to_string(m) + " must lie in 0..n";
    return 1;
  }
  if (m == 0) return 0;
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) {
    err = std::string("no usable CUDA device: ") + cudaGetErrorString(ce);
    return 2;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    err = "device " + std::to_string(dev) + " is beyond the " + std::to_string(kMaxDevices) +
          " devices this routine keeps scratch addresses for";
    return 2;
  }
  // An error left by the caller's earlier asynchronous work would otherwise be
  // read (and cleared) after the launch as if the launch had failed; report it
  // as what it is and leave it pending for the caller.
  ce = cudaPeekAtLastError();
  if (ce != cudaSuccess) {
    err = std::string("an earlier CUDA error is pending on this thread (nothing was launched): ") +
          cudaGetErrorString(ce);
    return 3;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_scratch_ptr[dev] == nullptr) {
      void* p = nullptr;
      ce = cudaGetSymbolAddress(&p, g_static_scratch);
      if (ce != cudaSuccess || p == nullptr) {
        err = std::string("cudaGetSymbolAddress of the static scratch failed: ") + cudaGetErrorString(ce);
        return 2;
      }
      g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_ptr[dev];
  }
  k_inverse_iteration_static<<<1, kThreads, 0, stream>>>(d, e, ev, n, m, Z, scratch, ortol_rel);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    err = std::string("kernel launch failed: ") + cudaGetErrorString(ce);
    return 3;
  }
  return 0;
}

}  // namespace xtb
