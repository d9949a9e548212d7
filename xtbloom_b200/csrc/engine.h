// Host orchestration of the batched GFN2-xTB single point on one GPU.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "xtbloom.h"

namespace xtb {

struct HostBatch {
  int64_t nsys = 0;
  std::vector<int64_t> atom_off;
  std::vector<int32_t> Z;
  std::vector<double> qmol;
  std::vector<int32_t> uhf;
  std::vector<int32_t> nch;   // spin channels per system (1 or 2)
  int32_t model = 2;          // XTBLOOM_MODEL_GFN2_XTB or XTBLOOM_MODEL_GFN1_XTB
};

struct ComputeRequest {
  const xtbloom_batch_t* batch = nullptr;
  const xtbloom_compute_options_t* options = nullptr;
  const xtbloom_batch_result_t* result = nullptr;
  // normalised options
  int32_t model = 2;   // XTBLOOM_MODEL_GFN2_XTB or XTBLOOM_MODEL_GFN1_XTB
  uint32_t flags = 0;
  int32_t max_iter = 250;
  double ctol = 1e-6, etol = 1e-8, kt = 0.0;
  int32_t memory = 8;
  double damping = 0.4;
  bool spin_channels = false;   // the batch carries a spin_channels field
  bool warm = false;            // strict WARM start from the retained checkpoint
  // uniform electric field per system (Hartree / (e bohr)), from the attachments
  std::vector<uint8_t> field_attached;
  std::vector<double> field;
  // charge response b + A q (per-atom shifts, per-system symmetric blocks)
  bool have_response = false;
  std::vector<double> resp_b, resp_A;
  std::vector<int64_t> resp_off;
};

class Engine {
 public:
  Engine(int device, cudaStream_t stream);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  // Runs one batch; returns an ABI status and fills error on failure.
  xtbloom_status_t compute(const ComputeRequest& req, std::string& error);
  xtbloom_status_t debug_fetch(const std::string& name, int64_t system, double* out,
                               size_t capacity, size_t* count, std::string& error);
  // Execution form of later computes: precision 0 = FP64 throughout, 1 =
  // split-precision GEMMs until a system's residual is below switch_residual
  // (then FP64 to convergence); graphs = replay captured SCC iterations.
  void set_execution(int precision, double switch_residual, bool graphs);
  // The WARM checkpoint is dropped (a plan's set-up compute must not leave one).
  void invalidate_checkpoint();
  // Bytes the engine holds: device buffers (grown by computes, kept for the
  // next) and pinned host staging.
  size_t device_bytes() const;
  size_t host_bytes() const;
  int device() const { return device_; }
  cudaStream_t stream() const { return stream_; }

  struct Impl;

 private:
  Impl* impl_;
  int device_;
  cudaStream_t stream_;
};

}  // namespace xtb
