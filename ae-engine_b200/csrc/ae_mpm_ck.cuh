// ae_mpm_ck.cuh -- CK-MPM (compact-kernel MPM) on the device: the reference's CkMpmSolver::step
// (ae_compute/src/ck_mpm.rs:187-480) over particles in its CkMpmParticle layout.
// All pointers here are device pointers; the C ABI in ae_mpm_api.cu stages host arrays.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ae_mpm.h"

namespace aemp {

class CkWork {
 public:
  CkWork() = default;
  CkWork(const CkWork&) = delete;
  CkWork& operator=(const CkWork&) = delete;
  ~CkWork();

  // `steps` solver steps over n particles (26 floats each, ae_mpm_ck_particle) in place.  With
  // kernel_ms (2 doubles, host), CUDA events around every launch give the summed durations of the
  // particle kernels and of the grid kernels (block compaction + update), and the call waits for
  // the stream.
  cudaError_t step(ae_mpm_ck_particle* particles, uint64_t n, const ae_mpm_ck_config& cfg, uint32_t steps,
                   cudaStream_t s, double* kernel_ms = nullptr);
  // kinetic_energy / average_velocity / average_volume_ratio (ck_mpm.rs:484-503); out on the host.
  cudaError_t stats(const ae_mpm_ck_particle* particles, uint64_t n, ae_mpm_ck_stats* out, cudaStream_t s);
  // CkMpmSolver::weight / weight_grad (ck_mpm.rs:163-185) at x[0..n).
  cudaError_t weights(const float* x, uint64_t n, float h, float* w, float* dw, cudaStream_t s);

  // kernels launched by the last step() call
  uint32_t last_launches() const { return launches_; }

 private:
  cudaError_t ensure(uint32_t grid_n);
  uint32_t gn_ = 0xffffffffu;  // grid the buffers are laid out for
  uint64_t blocks_ = 0;        // 4x4x4 node blocks
  float4* acc_ = nullptr;      // [blocks * 64][2]: (momentum, mass), (force, 0); zero between steps
  float4* vel_ = nullptr;      // [blocks * 64] grid velocity after the grid update
  uint32_t* flags_ = nullptr;  // [blocks] touched in the current step
  uint32_t* lists_ = nullptr;  // [blocks] touched blocks of the current step
  uint32_t* counts_ = nullptr; // [2] list lengths, alternating by step
  double* sums_ = nullptr;     // [5] stats accumulators
  bool clean_ = false;         // acc_ and flags_ are all zero
  uint32_t launches_ = 0;
};

}  // namespace aemp
