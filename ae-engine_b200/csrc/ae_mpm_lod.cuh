// ae_mpm_lod.cuh -- the engine tick's particle passes around the MPM substep, on the device:
// LOD classification (near / mid / far), the far-field ballistic update and the coarse
// temperature field (ae_engine/src/managers/simulation.rs:495-532, 612-679, 877-966).
// All pointers here are device pointers; the C ABI in ae_mpm_api.cu stages host arrays.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "radix_sort.cuh"

namespace aemp {

class LodWork {
 public:
  LodWork() = default;
  LodWork(const LodWork&) = delete;
  LodWork& operator=(const LodWork&) = delete;
  ~LodWork();

  // pos: count x 3 floats; active: count bytes (0/1) or null.  near_out / mid_out / far_out each
  // hold up to count indices.  Results: near = the max_near particles closest to the player among
  // those within near_dist (ascending index), mid = the rest within mid_dist (ascending index) then
  // the culled near ones (ascending index), far = the rest (ascending index).  counts[3] on the host.
  cudaError_t classify(const float* pos, const uint8_t* active, uint64_t count, const float player[3], float near_dist,
                       float mid_dist, uint64_t max_near, uint64_t* near_out, uint64_t* mid_out, uint64_t* far_out,
                       uint64_t counts[3], cudaStream_t s);

  // far particles far_idx[0..n) (null: 0..n): gravity on y, position, temperature blended toward
  // the nearest cell of the coarse field (coarse: cn^3 floats, x fastest).
  cudaError_t far_field(float* pos, float* vel, float* temp, const uint64_t* far_idx, uint64_t n, const float* coarse,
                        uint32_t cn, float cdx, const float origin[3], float far_dt, cudaStream_t s);

  // MpssBuffer housekeeping (ae_engine/src/lib.rs:347-358) over particles 0..n: passes 1 = world
  // bounds (reflect, halve the velocity), 2 = temperature clamp, 4 = phase transitions.
  // *transitions (host) = particles whose phase changed.
  cudaError_t housekeeping(float* pos, float* vel, float* temp, uint8_t* phase, const uint16_t* material,
                           const uint8_t* active, uint64_t n, const float bmin[3], const float bmax[3], float min_temp,
                           float max_temp, uint32_t passes, uint32_t* transitions, cudaStream_t s);

  // coarse field (cn^3 floats, updated in place): mass-weighted temperature of the near particles
  // near_idx[0..n) (null: 0..n; inactive ones skipped), relaxation, one FTCS diffusion step.
  cudaError_t coarse_field(const float* pos, const float* mass, const float* temp, const uint8_t* active,
                           const uint64_t* near_idx, uint64_t n, float* coarse, uint32_t cn, float cdx,
                           const float origin[3], float dt, cudaStream_t s);

 private:
  cudaError_t grow(uint64_t count, uint64_t cells);
  uint64_t cap_ = 0, cells_cap_ = 0;
  bool select_smem_set_ = false;
  uint32_t* tile_counts_ = nullptr;  // [3][tiles]
  uint32_t* tile_offs_ = nullptr;    // [3][tiles]
  uint32_t* totals_ = nullptr;       // [4]: class totals, housekeeping transition count
  uint64_t* near_tmp_ = nullptr;     // [cap] near candidates (ascending index)
  uint32_t* near_key_ = nullptr;     // [cap] their squared distance, as bits; later cell keys
  uint8_t* keep_ = nullptr;          // [cap]
  float* tm_ = nullptr;              // [cap] temperature x mass (coarse field), sorted by cell
  float* m_ = nullptr;               // [cap] mass, sorted by cell
  float* cell_a_ = nullptr;          // [cells] sums of temperature x mass
  float* cell_b_ = nullptr;          // [cells] sums of mass
  float* field_tmp_ = nullptr;       // [cells]
  uint32_t* run_start_ = nullptr;    // [cells] each cell's run in the cell-sorted near list
  uint32_t* run_end_ = nullptr;      // [cells]
  SortScratch sort_;
};

}  // namespace aemp
