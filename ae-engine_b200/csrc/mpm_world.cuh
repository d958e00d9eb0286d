// mpm_world.cuh -- device-resident MPM scenes ("worlds") and the substep pipeline.
//
// HBM layout of a world (all scenes share one set of arrays, so one launch of each kernel
// serves every scene):
//   particles   7 arrays of 4-wide vectors per slot (112 B/particle in f32), two copies
//               (G2P reads one and writes the other in sorted order):
//                 a0 = (x, y, z, m)          a1 = (F00, F01, F02, F10)   a2 = (F11, F12, F20, F21)
//                 a3 = (F22, J, material, original index)  [the last two as raw 32-bit patterns]
//                 a4 = (vx, vy, vz, C00)     a5 = (C01, C02, C10, C11)   a6 = (C12, C20, C21, C22)
//               G2P reads a0..a3 (64 B) and writes a0..a6; P2G reads a0..a6.
//   cell keys   u32 per slot: global block-major node index of the particle's stencil base, so a
//               key is also the index of that node in the grid arrays.
//   grid        per scene ceil(n/4)^3 blocks of 4x4x4 nodes plus one spare "dead" block; per node
//               an accumulator (m, px, py, pz) and a velocity (vx, vy, vz, m), both 16 B in f32.
//               Only blocks a particle stencil touched are updated; a touched-block list is built
//               by P2G and consumed (and cleared) by the grid update.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/ae_mpm.h"
#include "mpm_math.cuh"
#include "radix_sort.cuh"

namespace aemp {

template <class T>
struct V4T;
template <>
struct V4T<float> {
  using type = float4;
};
template <>
struct V4T<double> {
  using type = double4;
};

template <class T>
struct SceneDev {
  int32_t mode, wall_mode, wall_margin, wall_origin;
  int32_t n[3], nb[3];
  uint32_t blk_off;   // first global block of this scene
  uint32_t dead_key;  // key of slots past the live count (first node of the spare block)
  uint32_t mat_off;   // first entry of this scene in the material table
  uint32_t n_mat;     // scene materials; entry n_mat is the out-of-range fallback
  uint32_t p_off, p_cap, p_count;
  T dx, inv_dx, dt, restitution, damping;
  T origin[3], grav[3];
};

// Kernel argument block (passed by value).
template <class T>
struct WorldDev {
  using V4 = typename V4T<T>::type;
  const SceneDev<T>* scenes;
  const MatDev* mats;
  const int4* chunks;  // {scene, lo, hi_live, hi_cap}
  // a world of one scene: its chunks are consecutive ranges of blockDim.x slots, given here
  uint32_t one_scene, one_off, one_live_end, one_cap_end;
  const V4* in[7];
  V4* out[7];
  const uint32_t* perm;  // sorted position -> storage slot; nullptr = identity
  uint32_t* keys;        // keys for the next sort, written by G2P in the new slot order
  V4* acc;
  V4* vel;
  uint32_t* blk_flag;
  uint32_t* touched;
  uint32_t* touched_count;
  const uint32_t* blk_scene;
  uint32_t* err;  // per scene: [error bits, svd fallbacks, domain clamps, tile overflows]
  int32_t svd_fallback;
  int32_t max_tile_nodes;
  // snow particles whose F left the elastic region: {slot, scene}, filled by G2P
  uint2* clamp_queue;
  uint32_t* clamp_count;
  // deterministic mode
  const uint32_t* sorted_keys;
  uint32_t* cell_slot;  // per node: index of the occupied cell record, or 0xffffffff
  V4* cell_rec;         // 27 contributions per occupied cell
  uint32_t* cell_count;
  uint32_t* seg_start;  // sorted position where each occupied cell's run starts
};

enum : uint32_t { kErrNaN = 1u, kErrDomain = 2u };

// Device memory source for a world (the server reuses memory across batch rebuilds).
struct DevAlloc {
  virtual ~DevAlloc() {}
  virtual cudaError_t alloc(void** p, size_t bytes) = 0;
  virtual void release(void* p) = 0;
};

// Type-erased interface used by the C ABI.
struct WorldBase {
  virtual ~WorldBase() {}
  virtual int upload(uint32_t scene, const void* host, uint64_t n, bool f64) = 0;
  virtual int download(uint32_t scene, void* host, bool f64) = 0;
  // Many scenes per call (f32 worlds): every host<->device copy is queued back to back through one
  // staging area, so the copies run at link speed instead of one scene, one wait at a time.
  // upload_many is asynchronous like upload; download_many waits once, at the end.
  // With a copy stream, the host<->device copies go on that stream instead (ordered against the
  // world's own stream by events), so that they overlap another world's substeps; download_many
  // then returns without waiting and the results are in place once `copy` has drained.
  virtual int upload_many(uint32_t n, const uint32_t* scenes, const ae_mpm_particles* views, const uint64_t* counts,
                          cudaStream_t copy = nullptr) = 0;
  virtual int download_many(uint32_t n, const uint32_t* scenes, ae_mpm_particles* views,
                            cudaStream_t copy = nullptr) = 0;
  virtual int step(uint32_t n) = 0;
  virtual int sync() = 0;
  virtual int totals(uint32_t scene, double out[5]) = 0;
  virtual int errors(uint32_t scene, uint32_t* word, uint64_t counters[3]) = 0;
  virtual int set_scene_params(uint32_t scene, const ae_mpm_scene_desc& d) = 0;
  virtual int grid_download(uint32_t scene, float* mass, float* vel, uint64_t n_nodes) = 0;
  virtual int snapshot(bool restore) = 0;
  virtual uint64_t last_launches() const = 0;
  virtual uint64_t particles() const = 0;
  virtual cudaStream_t stream() const = 0;
  // replaces the world's stream by one of CUDA stream priority `priority` (lower = served first);
  // the world's queued work finishes first
  virtual int set_stream_priority(int priority) = 0;
  virtual ae_mpm_exec_opts& opts() = 0;
  virtual void invalidate_graph() = 0;
  virtual uint64_t device_bytes() const = 0;
  // copy scene `src_scene` of `src` (same precision, same grid size) into scene `dst_scene`
  // of this world on the device; the source world's queued work must have finished
  virtual int copy_scene_from(uint32_t dst_scene, WorldBase* src, uint32_t src_scene) = 0;
  // Continuous batching: scene slot `scene` takes a new scene `d` in place.  The slot keeps the
  // grid blocks, material entries and particle capacity it was created with, so d's grid must
  // need no more blocks, d no more materials and n no more particles.  `host` (a particle view as
  // for upload, or null: particles follow by copy_scene_from) supplies the n particles.
  virtual int assign_scene(uint32_t scene, const ae_mpm_scene_desc& d, const void* host, uint64_t n) = 0;
  // The slot holds no particles (and costs the substep nothing but its empty chunks).
  virtual int vacate_scene(uint32_t scene) = 0;
  virtual uint32_t scene_count(uint32_t scene) const = 0;
  virtual int precision() const = 0;
  // [sort, P2G, grid update, G2P (+ snow clamp), whole substep, the G2P or fused kernel alone]
  virtual int stage_times(uint32_t n, double out_us[6]) = 0;
  std::string err;
};

// Creates a world on the current device; returns nullptr and fills `why` on failure.
WorldBase* make_world(const ae_mpm_scene_desc* scenes, uint32_t n_scenes, const ae_mpm_exec_opts& opts,
                      std::string& why, int* status, DevAlloc* alloc = nullptr);

// Estimated device bytes for one scene (used by the server's HBM admission).
uint64_t scene_device_bytes(const ae_mpm_scene_desc& d, int precision);

// Device SM count (cached per device).
int device_sm_count();

// CUDA device of a context and its error text (defined with the C ABI).
int ctx_device(const ae_mpm_ctx* ctx);
void ctx_set_error(ae_mpm_ctx* ctx, const std::string& msg);

}  // namespace aemp
