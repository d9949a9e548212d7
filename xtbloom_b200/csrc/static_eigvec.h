// Host side of the static-scratch tridiagonal eigenvector routine.
#pragma once

#include <cuda_runtime.h>

#include <string>

namespace xtb {

constexpr int kStaticMaxN = 256;   // largest matrix the static scratch holds

// Enqueues inverse iteration for eigenvectors 0..m-1 of the n x n tridiagonal
// (d[n], e[n-1]) with ascending eigenvalues ev[m] on `stream`; vector j is
// written to Z[j*n .. j*n+n).  All pointers are device memory of the current
// device.  Returns 0 on success, 1 for an invalid size, 2 when the device or
// the scratch address is unavailable, 3 when the launch failed; err explains.
int static_eigvec_run(const double* d, const double* e, const double* ev, int n, int m, double* Z,
                      double ortol_rel, cudaStream_t stream, std::string& err);

}  // namespace xtb
