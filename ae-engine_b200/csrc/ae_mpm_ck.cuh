// ae_mpm_ck.cuh -- CK-MPM (compact-kernel MPM) on the device: the reference's CkMpmSolver::step
// (ae_compute/src/ck_mpm.rs:187-480) over particles in its CkMpmParticle layout.
// All pointers here are device pointers; the C ABI in ae_mpm_api.cu stages host arrays.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ae_mpm.h"
#include "radix_sort.cuh"

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
  // The same steps with node sums in particle order (a per-node gather over cell-sorted particles),
  // as the reference's serial loops add them: bitwise reproducible, and bit-exact against the
  // reference wherever ln(det F) agrees.  Slower than step().
  cudaError_t step_deterministic(ae_mpm_ck_particle* particles, uint64_t n, const ae_mpm_ck_config& cfg,
                                 uint32_t steps, cudaStream_t s);
  // kinetic_energy / average_velocity / average_volume_ratio (ck_mpm.rs:484-503); out on the host.
  cudaError_t stats(const ae_mpm_ck_particle* particles, uint64_t n, ae_mpm_ck_stats* out, cudaStream_t s);
  // CkMpmSolver::weight / weight_grad (ck_mpm.rs:163-185) at x[0..n).
  cudaError_t weights(const float* x, uint64_t n, float h, float* w, float* dw, cudaStream_t s);

  // kernels launched by the last step() call
  uint32_t last_launches() const { return launches_; }

 private:
  cudaError_t ensure(uint32_t grid_n);
  cudaError_t ensure_det(uint64_t n, uint32_t grid_n);
  cudaError_t begin_call(uint32_t grid_n, cudaStream_t s);
  uint32_t gn_ = 0xffffffffu;  // grid the buffers are laid out for
  uint64_t blocks_ = 0;        // 4x4x4 node blocks
  float4* acc_ = nullptr;      // [blocks * 64][2]: (momentum, mass), (force, 0); zero between steps
  float4* vel_ = nullptr;      // [blocks * 64] grid velocity after the grid update
  uint32_t* flags_ = nullptr;  // [blocks] touched in the current step
  uint32_t* lists_ = nullptr;  // [blocks] touched blocks of the current step
  uint32_t* counts_ = nullptr; // [2] list lengths, alternating by step
  double* sums_ = nullptr;     // [5] stats accumulators
  bool clean_ = false;         // acc_ and flags_ are all zero
  // deterministic mode: cell keys, stresses, per-cell [begin, end) of the sorted order (empty
  // between calls), sort scratch
  uint32_t* det_keys_ = nullptr;
  float* det_stress_ = nullptr;
  uint2* det_range_ = nullptr;
  uint64_t det_cap_ = 0, det_cells_ = 0;
  SortScratch det_sort_;
  uint32_t launches_ = 0;
};

}  // namespace aemp
