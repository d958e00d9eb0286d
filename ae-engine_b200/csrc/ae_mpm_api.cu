// ae_mpm_api.cu -- C ABI of libae_mpm.so (declared in include/ae_mpm.h).
//
// The drop-in entry points keep the reference's call shape (caller-owned MpssBuffer arrays,
// particle_indices, MpmConfig, material/model tables) and move the selected particles through
// one device-resident world per context, re-created only when the grid size or particle count
// changes.  Nothing here falls back to CPU arithmetic: without a usable CUDA device every entry
// point that computes returns AE_MPM_ECUDA.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <omp.h>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ae_mpm.h"
#include "mpm_world.cuh"
#include "ae_mpm_ck.cuh"
#include "ae_mpm_lod.cuh"
#include "radix_sort.cuh"

using aemp::WorldBase;

struct ae_mpm_ctx {
  int device = 0;
  std::string err = "ok";
  // drop-in world cache
  WorldBase* dropin = nullptr;
  std::string dropin_sig;
  std::vector<ae_mpm_material> dropin_mats;
  // pinned staging for gathers through particle_indices
  float* pin = nullptr;
  size_t pin_bytes = 0;
  // radix sort API scratch
  aemp::SortScratch sort;
  uint32_t* sort_keys = nullptr;
  uint64_t sort_keys_cap = 0;
  // autotune cache: workload signature -> choice
  std::map<std::string, ae_mpm_tune_result> tuned;
  // engine tick passes (LOD, far field, coarse field) and their device staging for host arrays
  aemp::LodWork* lod = nullptr;
  // CK-MPM solver buffers
  aemp::CkWork* ck = nullptr;
  void* dstage = nullptr;
  size_t dstage_bytes = 0;
  // completion events of the drop-in's whole-array copies back to the host
  cudaEvent_t out_ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};

struct ae_mpm_world {
  ae_mpm_ctx* ctx;
  WorldBase* w;
  std::string sig;  // workload signature for the autotune cache
};

namespace aemp {
int ctx_device(const ae_mpm_ctx* ctx) { return ctx ? ctx->device : 0; }
void ctx_set_error(ae_mpm_ctx* ctx, const std::string& msg) {
  if (ctx) ctx->err = msg;
}
}  // namespace aemp

namespace {

int fail(ae_mpm_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int set_device(ae_mpm_ctx* ctx) {
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  return AE_MPM_OK;
}

std::string world_signature(const ae_mpm_scene_desc* s, uint32_t n, const ae_mpm_exec_opts& o) {
  // scene count, total particles, grid sizes and the material models of the batch
  uint64_t parts = 0;
  std::string g;
  for (uint32_t i = 0; i < n; ++i) {
    parts += s[i].max_particles;
    if (i < 8) g += std::to_string(s[i].n[0]) + "x" + std::to_string(s[i].n[1]) + "x" + std::to_string(s[i].n[2]) + ",";
  }
  uint32_t models = 0;
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t k = 0; k < s[i].n_materials; ++k) models |= 1u << (s[i].materials[k].model & 31);
  int bucket = 0;
  while ((1ull << bucket) < parts) ++bucket;
  return "m" + std::to_string(s[0].mode) + "p" + std::to_string(o.precision) + "d" + std::to_string(o.deterministic) +
         "s" + std::to_string(n) + "n" + std::to_string(bucket) + "g" + g + "k" + std::to_string(models);
}

int ensure_pinned(ae_mpm_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->pin_bytes) return AE_MPM_OK;
  if (ctx->pin) cudaFreeHost(ctx->pin);
  ctx->pin = nullptr;
  ctx->pin_bytes = 0;
  cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&ctx->pin), bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ENOMEM, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
  ctx->pin_bytes = bytes;
  return AE_MPM_OK;
}

int ensure_dstage(ae_mpm_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->dstage_bytes) return AE_MPM_OK;
  cudaFree(ctx->dstage);
  ctx->dstage = nullptr;
  ctx->dstage_bytes = 0;
  cudaError_t e = cudaMalloc(&ctx->dstage, bytes);
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  ctx->dstage_bytes = bytes;
  return AE_MPM_OK;
}

// device (or managed) memory, as opposed to ordinary or pinned host memory
bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

aemp::LodWork* lod_work(ae_mpm_ctx* ctx) {
  if (!ctx->lod) ctx->lod = new aemp::LodWork();
  return ctx->lod;
}

aemp::CkWork* ck_work(ae_mpm_ctx* ctx) {
  if (!ctx->ck) ctx->ck = new aemp::CkWork();
  return ctx->ck;
}

// reference-layout view over the pinned staging for n particles
ae_mpm_particles pinned_view(ae_mpm_ctx* ctx, uint64_t n) {
  ae_mpm_particles v;
  float* p = ctx->pin;
  v.pos = p;
  v.vel = p + 3 * n;
  v.strain = p + 6 * n;
  v.jacobian = p + 15 * n;
  v.c = p + 16 * n;
  v.mass = p + 25 * n;
  v.material_idx = reinterpret_cast<uint16_t*>(p + 26 * n);
  return v;
}

// Drop-in calls whose indices are ascending and select a quarter or more of the buffer copy the
// buffer's arrays whole and gather / scatter the selected particles on the device.  `full`: every
// field travels (reference mode); otherwise position, velocity and mass only, with F = I, C = 0,
// J = 1 (the velocity-only substep reads none of them and writes back position and velocity).
__global__ void dropin_gather_kernel(ae_mpm_particles src, const uint64_t* __restrict__ idx, uint64_t n,
                                     ae_mpm_particles dst, int full) {
  const uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint64_t i = idx[k];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    dst.pos[3 * k + a] = src.pos[3 * i + a];
    dst.vel[3 * k + a] = src.vel[3 * i + a];
  }
  dst.mass[k] = src.mass[i];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    dst.strain[9 * k + q] = full ? src.strain[9 * i + q] : ((q % 4 == 0) ? 1.0f : 0.0f);
    dst.c[9 * k + q] = full ? src.c[9 * i + q] : 0.0f;
  }
  dst.jacobian[k] = full ? src.jacobian[i] : 1.0f;
  dst.material_idx[k] = full ? src.material_idx[i] : uint16_t(0);
}

__global__ void dropin_scatter_kernel(ae_mpm_particles src, const uint64_t* __restrict__ idx, uint64_t n,
                                      ae_mpm_particles dst, int full) {
  const uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint64_t i = idx[k];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    dst.pos[3 * i + a] = src.pos[3 * k + a];
    dst.vel[3 * i + a] = src.vel[3 * k + a];
  }
  if (full) {
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      dst.strain[9 * i + q] = src.strain[9 * k + q];
      dst.c[9 * i + q] = src.c[9 * k + q];
    }
    dst.jacobian[i] = src.jacobian[k];
  }
}

// Host copy between the caller's (pageable) arrays and pinned staging, split over up to 8 threads
// for large arrays: the driver's own pageable copies run on one thread at a fraction of the link's
// bandwidth, while copies from pinned staging run at the link's speed.
void host_copy(void* dst, const void* src, size_t bytes) {
  const int t_max = bytes >= (size_t(8) << 20) ? std::min(8, omp_get_max_threads()) : 1;
  if (t_max <= 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t chunk = ((bytes + size_t(t_max) - 1) / size_t(t_max) + 63) & ~size_t(63);
#pragma omp parallel for num_threads(t_max) schedule(static)
  for (int t = 0; t < t_max; ++t) {
    const size_t lo = size_t(t) * chunk;
    if (lo < bytes)
      std::memcpy(static_cast<char*>(dst) + lo, static_cast<const char*>(src) + lo, std::min(chunk, bytes - lo));
  }
}

// Carves the device staging of a whole-array drop-in call: the buffer's arrays (capacity particles),
// the index list and the selected particles (n), each region on a 16-byte boundary.
struct DropinLayout {
  size_t off[16];
  size_t bytes;
};
DropinLayout dropin_layout(uint64_t capacity, uint64_t n, bool full) {
  const size_t sz[15] = {12 * capacity, 12 * capacity, 4 * capacity, full ? 36 * capacity : 0, full ? 36 * capacity : 0,
                         full ? 4 * capacity : 0, full ? 2 * capacity : 0, 8 * n, 12 * n, 12 * n, 36 * n, 4 * n, 36 * n,
                         4 * n, 2 * n};
  DropinLayout l{};
  size_t o = 0;
  for (int r = 0; r < 15; ++r) {
    l.off[r] = o;
    o += (sz[r] + 15) & ~size_t(15);
  }
  l.off[15] = o;
  l.bytes = o;
  return l;
}

int dropin_run(ae_mpm_ctx* ctx, int mode, const ae_mpm_particles* buffer, uint64_t capacity, const ae_mpm_grid* grid,
               const ae_mpm_config* config, const std::vector<ae_mpm_material>& mats, float total_dt,
               const uint64_t* idx, uint64_t n) {
  if (config->substeps == 0) return AE_MPM_OK;  // `for _ in 0..0` runs no substep
  if (grid->nx == 0 || grid->ny == 0 || grid->nz == 0 || grid->nx > (1u << 20) || grid->ny > (1u << 20) ||
      grid->nz > (1u << 20))
    return fail(ctx, AE_MPM_EINVAL, "grid needs 1..2^20 nodes per axis");
  if (!(grid->dx > 0.0f)) return fail(ctx, AE_MPM_EINVAL, "grid dx must be positive");
  if (!buffer->pos || !buffer->vel || !buffer->mass ||
      (mode == AE_MPM_MODE_REFERENCE && (!buffer->strain || !buffer->jacobian || !buffer->c || !buffer->material_idx)))
    return fail(ctx, AE_MPM_EINVAL, "particle buffer has a null array");
  // bounds and order of the index list (split over threads for long lists; the message names the
  // first index out of range)
  uint64_t max_idx = 0;
  uint64_t descents = 0;
  const int t_idx = n >= (uint64_t(1) << 16) ? std::min(8, omp_get_max_threads()) : 1;
#pragma omp parallel for num_threads(t_idx) schedule(static) reduction(max : max_idx) reduction(+ : descents)
  for (int64_t k = 0; k < int64_t(n); ++k) {
    max_idx = std::max(max_idx, idx[k]);
    if (k > 0 && idx[k] <= idx[k - 1]) ++descents;
  }
  if (max_idx >= capacity)
    for (uint64_t k = 0; k < n; ++k)
      if (idx[k] >= capacity)
        return fail(ctx, AE_MPM_EINVAL, "particle index " + std::to_string(idx[k]) + " >= capacity");
  const bool ascending = descents == 0;
  int rc = set_device(ctx);
  if (rc) return rc;
  ae_mpm_scene_desc d{};
  d.mode = mode;
  d.n[0] = uint32_t(grid->nx);
  d.n[1] = uint32_t(grid->ny);
  d.n[2] = uint32_t(grid->nz);
  d.dx = grid->dx;
  for (int a = 0; a < 3; ++a) {
    d.origin[a] = grid->origin[a];
    d.gravity[a] = config->gravity[a];
  }
  d.dt = total_dt / float(config->substeps);
  d.damping = config->damping;
  d.wall_origin = n >= 50000 ? 1 : 0;  // mpm_solver.rs:1077 switches to the parallel path
  d.wall_margin = 0;
  d.n_materials = uint32_t(mats.size());
  d.materials = mats.data();
  // capacity: the power of two at or above n, the particle bucket the cached world is keyed by, so a
  // later call with a different count in the same bucket (the near set changes from tick to tick)
  // reuses the world
  uint64_t cap = 1;
  while (cap < n) cap <<= 1;
  d.max_particles = cap;
  ae_mpm_exec_opts o;
  ae_mpm_exec_opts_default(&o);
  std::string sig = world_signature(&d, 1, o) + "|" + std::to_string(mats.size());
  if (!ctx->dropin || ctx->dropin_sig != sig) {
    delete ctx->dropin;
    ctx->dropin = nullptr;
    auto it = ctx->tuned.find(world_signature(&d, 1, o));
    if (it != ctx->tuned.end()) {
      o.p2g_variant = it->second.p2g_variant;
      o.block_threads = it->second.block_threads;
      o.sort_interval = it->second.sort_interval;
    }
    std::string why;
    int st = 0;
    ctx->dropin = aemp::make_world(&d, 1, o, why, &st);
    if (!ctx->dropin) return fail(ctx, st ? st : AE_MPM_ECUDA, why);
    ctx->dropin_sig = sig;
  } else {
    rc = ctx->dropin->set_scene_params(0, d);
    if (rc) return fail(ctx, rc, ctx->dropin->err);
  }
  WorldBase* w = ctx->dropin;
  const bool full = mode == AE_MPM_MODE_REFERENCE;
  if (ascending && 4 * n >= capacity) {
    // whole arrays in, gather and scatter on the device, whole arrays out: the unselected particles
    // travel both ways unchanged (the caller holds the buffer exclusively for the call)
    const DropinLayout l = dropin_layout(capacity, n, full);
    rc = ensure_dstage(ctx, l.bytes);
    if (rc) return rc;
    char* dst = static_cast<char*>(ctx->dstage);
    ae_mpm_particles dfull{}, dsel{};
    dfull.pos = reinterpret_cast<float*>(dst + l.off[0]);
    dfull.vel = reinterpret_cast<float*>(dst + l.off[1]);
    dfull.mass = reinterpret_cast<float*>(dst + l.off[2]);
    if (full) {
      dfull.strain = reinterpret_cast<float*>(dst + l.off[3]);
      dfull.c = reinterpret_cast<float*>(dst + l.off[4]);
      dfull.jacobian = reinterpret_cast<float*>(dst + l.off[5]);
      dfull.material_idx = reinterpret_cast<uint16_t*>(dst + l.off[6]);
    }
    uint64_t* didx = reinterpret_cast<uint64_t*>(dst + l.off[7]);
    dsel.pos = reinterpret_cast<float*>(dst + l.off[8]);
    dsel.vel = reinterpret_cast<float*>(dst + l.off[9]);
    dsel.strain = reinterpret_cast<float*>(dst + l.off[10]);
    dsel.jacobian = reinterpret_cast<float*>(dst + l.off[11]);
    dsel.c = reinterpret_cast<float*>(dst + l.off[12]);
    dsel.mass = reinterpret_cast<float*>(dst + l.off[13]);
    dsel.material_idx = reinterpret_cast<uint16_t*>(dst + l.off[14]);
    // pinned staging mirrors the device layout of the whole arrays and the index list
    rc = ensure_pinned(ctx, l.off[8]);
    if (rc) return rc;
    char* hp = reinterpret_cast<char*>(ctx->pin);
    cudaStream_t st = w->stream();
    cudaError_t e = cudaSuccess;
    // each array: host copy into pinned staging, then its DMA, which overlaps the next host copy
    auto in = [&](int r, const void* src, size_t b) {
      if (e != cudaSuccess) return;
      host_copy(hp + l.off[r], src, b);
      e = cudaMemcpyAsync(dst + l.off[r], hp + l.off[r], b, cudaMemcpyHostToDevice, st);
    };
    in(0, buffer->pos, 12 * capacity);
    in(1, buffer->vel, 12 * capacity);
    in(2, buffer->mass, 4 * capacity);
    if (full) {
      in(3, buffer->strain, 36 * capacity);
      in(4, buffer->c, 36 * capacity);
      in(5, buffer->jacobian, 4 * capacity);
      in(6, buffer->material_idx, 2 * capacity);
    }
    in(7, idx, 8 * n);
    const unsigned blocks = unsigned((n + 255) / 256);
    if (e == cudaSuccess) {
      dropin_gather_kernel<<<blocks, 256, 0, st>>>(dfull, didx, n, dsel, full ? 1 : 0);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, std::string("drop-in gather: ") + cudaGetErrorString(e));
    if ((rc = w->upload(0, &dsel, n, false)) || (rc = w->step(uint32_t(config->substeps))) ||
        (rc = w->download(0, &dsel, false)))
      return fail(ctx, rc, w->err);
    dropin_scatter_kernel<<<blocks, 256, 0, st>>>(dsel, didx, n, dfull, full ? 1 : 0);
    e = cudaGetLastError();
    // the written arrays back: DMA into pinned staging, then host copies into the caller's arrays
    const int outs[5] = {0, 1, 3, 4, 5};
    const size_t out_b[5] = {12 * capacity, 12 * capacity, 36 * capacity, 36 * capacity, 4 * capacity};
    void* const out_dst[5] = {buffer->pos, buffer->vel, buffer->strain, buffer->c, buffer->jacobian};
    const int n_out = full ? 5 : 2;
    // each array's host copy starts when its own DMA has landed, while the next one transfers
    for (int k = 0; k < n_out && e == cudaSuccess; ++k) {
      if (!ctx->out_ev[k]) e = cudaEventCreateWithFlags(&ctx->out_ev[k], cudaEventDisableTiming);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(hp + l.off[outs[k]], dst + l.off[outs[k]], out_b[k], cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaEventRecord(ctx->out_ev[k], st);
    }
    for (int k = 0; k < n_out && e == cudaSuccess; ++k) {
      e = cudaEventSynchronize(ctx->out_ev[k]);
      if (e == cudaSuccess) host_copy(out_dst[k], hp + l.off[outs[k]], out_b[k]);
    }
    if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, std::string("drop-in scatter: ") + cudaGetErrorString(e));
    return AE_MPM_OK;
  }
  // gather the selected particles into pinned staging
  rc = ensure_pinned(ctx, sizeof(float) * 26 * n + sizeof(uint16_t) * n + 64);
  if (rc) return rc;
  ae_mpm_particles v = pinned_view(ctx, n);
  // long lists gather on the OpenMP team (reads only); the scatter back is parallel only for
  // ascending (hence distinct) indices, so a repeated index keeps the reference's last-write-wins
  const int t_host = n >= 4096 ? std::min(8, omp_get_max_threads()) : 1;
#pragma omp parallel for num_threads(t_host) schedule(static)
  for (int64_t kk = 0; kk < int64_t(n); ++kk) {
    const uint64_t k = uint64_t(kk);
    const uint64_t i = idx[k];
    std::memcpy(v.pos + 3 * k, buffer->pos + 3 * i, 3 * sizeof(float));
    std::memcpy(v.vel + 3 * k, buffer->vel + 3 * i, 3 * sizeof(float));
    v.mass[k] = buffer->mass[i];
    if (buffer->strain) {
      std::memcpy(v.strain + 9 * k, buffer->strain + 9 * i, 9 * sizeof(float));
    } else {
      for (int q = 0; q < 9; ++q) v.strain[9 * k + q] = (q % 4 == 0) ? 1.0f : 0.0f;
    }
    if (buffer->c) {
      std::memcpy(v.c + 9 * k, buffer->c + 9 * i, 9 * sizeof(float));
    } else {
      std::memset(v.c + 9 * k, 0, 9 * sizeof(float));
    }
    v.jacobian[k] = buffer->jacobian ? buffer->jacobian[i] : 1.0f;
    v.material_idx[k] = buffer->material_idx ? buffer->material_idx[i] : 0;
  }
  if ((rc = w->upload(0, &v, n, false)) || (rc = w->step(uint32_t(config->substeps))) || (rc = w->download(0, &v, false)))
    return fail(ctx, rc, w->err);
#pragma omp parallel for num_threads(ascending ? t_host : 1) schedule(static)
  for (int64_t kk = 0; kk < int64_t(n); ++kk) {
    const uint64_t k = uint64_t(kk);
    const uint64_t i = idx[k];
    std::memcpy(buffer->pos + 3 * i, v.pos + 3 * k, 3 * sizeof(float));
    std::memcpy(buffer->vel + 3 * i, v.vel + 3 * k, 3 * sizeof(float));
    if (mode == AE_MPM_MODE_REFERENCE) {
      std::memcpy(buffer->strain + 9 * i, v.strain + 9 * k, 9 * sizeof(float));
      std::memcpy(buffer->c + 9 * i, v.c + 9 * k, 9 * sizeof(float));
      buffer->jacobian[i] = v.jacobian[k];
    }
  }
  return AE_MPM_OK;
}

}  // namespace

extern "C" {

int ae_mpm_abi_version(void) { return AE_MPM_ABI_VERSION; }

void ae_mpm_exec_opts_default(ae_mpm_exec_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = 32;
  o->deterministic = 0;
  o->sort_interval = 1;
  o->p2g_variant = AE_MPM_P2G_AUTO;
  o->block_threads = 0;
  o->use_graph = 1;
  o->track_totals = 0;
  o->svd_fp64_fallback = 1;
}

int ae_mpm_ctx_create(int device, ae_mpm_ctx** out) {
  if (!out) return AE_MPM_EINVAL;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return AE_MPM_ECUDA;
  if (device < 0 || device >= count) return AE_MPM_EINVAL;
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return AE_MPM_ECUDA;
  auto* c = new ae_mpm_ctx();
  c->device = device;
  *out = c;
  return AE_MPM_OK;
}

void ae_mpm_ctx_destroy(ae_mpm_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  delete ctx->dropin;
  delete ctx->lod;
  delete ctx->ck;
  cudaFree(ctx->dstage);
  for (cudaEvent_t ev : ctx->out_ev)
    if (ev) cudaEventDestroy(ev);
  if (ctx->pin) cudaFreeHost(ctx->pin);
  aemp::sort_scratch_free(ctx->sort);
  cudaFree(ctx->sort_keys);
  delete ctx;
}

const char* ae_mpm_last_error(const ae_mpm_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int ae_mpm_step_parallel_with_grid(ae_mpm_ctx* ctx, const ae_mpm_particles* buffer, uint64_t capacity,
                                   const ae_mpm_grid* grid, const ae_mpm_config* config,
                                   const ae_mpm_material* material_table, uint32_t n_materials,
                                   const int32_t* model_table, uint32_t n_models, float total_dt,
                                   const uint64_t* particle_indices, uint64_t n_indices) {
  if (!ctx) return AE_MPM_EINVAL;
  if (n_indices == 0) return AE_MPM_OK;  // mpm_solver.rs:1072-1074
  if (!buffer || !grid || !config || !particle_indices) return fail(ctx, AE_MPM_EINVAL, "null argument");
  if (n_materials == 0 || !material_table)
    return fail(ctx, AE_MPM_EINVAL, "material_table is empty (the reference indexes material_table[0])");
  if (n_models > 0 && !model_table) return fail(ctx, AE_MPM_EINVAL, "model_table is null");
  // effective (params, model) per material index, with the reference's fallbacks
  // (mpm_solver.rs:840-841: params default to material_table[0], model to NeoHookean)
  const uint32_t ne = std::max(n_materials, n_models);
  std::vector<ae_mpm_material> mats(ne);
  for (uint32_t k = 0; k < ne; ++k) {
    mats[k] = material_table[k < n_materials ? k : 0];
    mats[k].model = k < n_models ? model_table[k] : AE_MPM_NEO_HOOKEAN;
    if (mats[k].model < AE_MPM_NEO_HOOKEAN || mats[k].model > AE_MPM_RIGID)
      return fail(ctx, AE_MPM_EINVAL, "model_table holds a value that is not a ConstitutiveModel");
  }
  return dropin_run(ctx, AE_MPM_MODE_REFERENCE, buffer, capacity, grid, config, mats, total_dt, particle_indices,
                    n_indices);
}

int ae_mpm_step_velocity_only_parallel(ae_mpm_ctx* ctx, const ae_mpm_particles* buffer, uint64_t capacity,
                                       const ae_mpm_grid* grid, const ae_mpm_config* config, float total_dt,
                                       const uint64_t* particle_indices, uint64_t n_indices) {
  if (!ctx) return AE_MPM_EINVAL;
  if (n_indices == 0) return AE_MPM_OK;  // mpm_solver.rs:1344-1346
  if (!buffer || !grid || !config || !particle_indices) return fail(ctx, AE_MPM_EINVAL, "null argument");
  std::vector<ae_mpm_material> mats(1);
  std::memset(&mats[0], 0, sizeof(mats[0]));
  mats[0].density = 1.0f;
  mats[0].young_modulus = 1.0f;
  mats[0].model = AE_MPM_NEO_HOOKEAN;  // unused: the velocity-only substep has no stress
  return dropin_run(ctx, AE_MPM_MODE_VELOCITY_ONLY, buffer, capacity, grid, config, mats, total_dt, particle_indices,
                    n_indices);
}

int ae_mpm_grid_download(ae_mpm_ctx* ctx, float* mass, float* vel, uint64_t n_nodes) {
  if (!ctx) return AE_MPM_EINVAL;
  if (!ctx->dropin) return fail(ctx, AE_MPM_EINVAL, "no drop-in step has run on this context");
  int rc = set_device(ctx);
  if (rc) return rc;
  rc = ctx->dropin->grid_download(0, mass, vel, n_nodes);
  return rc ? fail(ctx, rc, ctx->dropin->err) : AE_MPM_OK;
}

// the caller's options (or the defaults) with the autotuner's choice for this workload, if any
static ae_mpm_exec_opts resolve_opts(ae_mpm_ctx* ctx, const ae_mpm_scene_desc* scenes, uint32_t n_scenes,
                                     const ae_mpm_exec_opts* opts) {
  ae_mpm_exec_opts o;
  if (opts)
    o = *opts;
  else
    ae_mpm_exec_opts_default(&o);
  if (o.precision != 64) o.precision = 32;
  auto it = ctx->tuned.find(world_signature(scenes, n_scenes, o));
  if (it != ctx->tuned.end()) {
    if (o.p2g_variant == AE_MPM_P2G_AUTO) o.p2g_variant = it->second.p2g_variant;
    if (o.block_threads == 0) o.block_threads = it->second.block_threads;
    if (opts == nullptr || opts->p2g_variant == AE_MPM_P2G_AUTO) o.sort_interval = it->second.sort_interval;
  }
  if (o.p2g_variant == AE_MPM_P2G_AUTO) o.p2g_variant = AE_MPM_P2G_LANES;
  if (o.block_threads == 0) o.block_threads = 256;
  return o;
}

int ae_mpm_world_create(ae_mpm_ctx* ctx, const ae_mpm_scene_desc* scenes, uint32_t n_scenes,
                        const ae_mpm_exec_opts* opts, ae_mpm_world** out) {
  if (!ctx || !out) return AE_MPM_EINVAL;
  *out = nullptr;
  if (!scenes || n_scenes == 0) return fail(ctx, AE_MPM_EINVAL, "no scenes");
  int rc = set_device(ctx);
  if (rc) return rc;
  const ae_mpm_exec_opts o = resolve_opts(ctx, scenes, n_scenes, opts);
  std::string why;
  int st = 0;
  WorldBase* w = aemp::make_world(scenes, n_scenes, o, why, &st);
  if (!w) return fail(ctx, st ? st : AE_MPM_ECUDA, why);
  *out = new ae_mpm_world{ctx, w, world_signature(scenes, n_scenes, o)};
  return AE_MPM_OK;
}

int ae_mpm_world_destroy(ae_mpm_world* world) {
  if (!world) return AE_MPM_EINVAL;
  cudaSetDevice(world->ctx->device);
  delete world->w;
  delete world;
  return AE_MPM_OK;
}

#define AE_WORLD_CALL(expr)                                 \
  do {                                                      \
    if (!world) return AE_MPM_EINVAL;                       \
    int rc_ = set_device(world->ctx);                       \
    if (rc_) return rc_;                                    \
    rc_ = (expr);                                           \
    if (rc_) return fail(world->ctx, rc_, world->w->err);   \
    return AE_MPM_OK;                                       \
  } while (0)

int ae_mpm_world_upload(ae_mpm_world* world, uint32_t scene, const ae_mpm_particles* host, uint64_t n) {
  if (world && !host) return fail(world->ctx, AE_MPM_EINVAL, "null particle view");
  AE_WORLD_CALL(world->w->upload(scene, host, n, false));
}
int ae_mpm_world_upload_f64(ae_mpm_world* world, uint32_t scene, const ae_mpm_particles_f64* host, uint64_t n) {
  if (world && !host) return fail(world->ctx, AE_MPM_EINVAL, "null particle view");
  AE_WORLD_CALL(world->w->upload(scene, host, n, true));
}
int ae_mpm_world_set_scene(ae_mpm_world* world, uint32_t scene, const ae_mpm_scene_desc* desc) {
  if (world && !desc) return fail(world->ctx, AE_MPM_EINVAL, "null scene description");
  AE_WORLD_CALL(world->w->set_scene_params(scene, *desc));
}
int ae_mpm_world_step(ae_mpm_world* world, uint32_t n_substeps) { AE_WORLD_CALL(world->w->step(n_substeps)); }
int ae_mpm_world_sync(ae_mpm_world* world) { AE_WORLD_CALL(world->w->sync()); }
int ae_mpm_world_download(ae_mpm_world* world, uint32_t scene, ae_mpm_particles* host) {
  if (world && !host) return fail(world->ctx, AE_MPM_EINVAL, "null particle view");
  AE_WORLD_CALL(world->w->download(scene, host, false));
}
int ae_mpm_world_download_f64(ae_mpm_world* world, uint32_t scene, ae_mpm_particles_f64* host) {
  if (world && !host) return fail(world->ctx, AE_MPM_EINVAL, "null particle view");
  AE_WORLD_CALL(world->w->download(scene, host, true));
}
int ae_mpm_world_upload_many(ae_mpm_world* world, uint32_t n, const uint32_t* scenes, const ae_mpm_particles* views,
                             const uint64_t* counts) {
  AE_WORLD_CALL(world->w->upload_many(n, scenes, views, counts));
}
int ae_mpm_world_download_many(ae_mpm_world* world, uint32_t n, const uint32_t* scenes, ae_mpm_particles* views) {
  AE_WORLD_CALL(world->w->download_many(n, scenes, views));
}
// ---------------------------------------------------------------------------------------------
// pipelined batch: the scenes of one call in consecutive groups, one world per group
// ---------------------------------------------------------------------------------------------
struct ae_mpm_batch {
  ae_mpm_ctx* ctx = nullptr;
  std::vector<WorldBase*> worlds;
  std::vector<uint32_t> first;  // group g holds scenes [first[g], first[g + 1])
  cudaStream_t up = nullptr, down = nullptr;
  ~ae_mpm_batch() {
    if (down) cudaStreamSynchronize(down);
    for (WorldBase* w : worlds) delete w;
    if (up) cudaStreamDestroy(up);
    if (down) cudaStreamDestroy(down);
  }
};

uint32_t ae_mpm_batch_partition(const uint64_t* capacities, uint32_t n_scenes, uint32_t n_groups,
                                uint32_t* first_scene) {
  if (!capacities || !first_scene || n_scenes == 0) return 0;
  const uint32_t g_n = n_groups == 0 ? 1u : (n_groups > n_scenes ? n_scenes : n_groups);
  // consecutive groups of about equal capacity, none empty: boundary g goes after the first scene
  // at which the running capacity reaches g / g_n of the total, as long as every later group can
  // still have a scene of its own
  uint64_t total = 0;
  for (uint32_t i = 0; i < n_scenes; ++i) total += capacities[i];
  uint32_t nb = 0;  // boundaries written
  first_scene[nb++] = 0;
  uint64_t acc = 0;
  for (uint32_t i = 0; i < n_scenes && nb < g_n; ++i) {
    acc += capacities[i];
    const uint32_t g = nb;
    const bool left_enough = n_scenes - (i + 1) >= g_n - g;
    if (left_enough && (unsigned __int128)acc * g_n >= (unsigned __int128)total * g) first_scene[nb++] = i + 1;
  }
  while (nb < g_n) {  // capacity-free tail scenes: one scene per remaining group
    first_scene[nb] = first_scene[nb - 1] + 1;
    ++nb;
  }
  first_scene[g_n] = n_scenes;
  return g_n;
}

int ae_mpm_batch_create(ae_mpm_ctx* ctx, const ae_mpm_scene_desc* scenes, uint32_t n_scenes,
                        const ae_mpm_exec_opts* opts, uint32_t n_groups, ae_mpm_batch** out) {
  if (!ctx || !out) return AE_MPM_EINVAL;
  *out = nullptr;
  if (!scenes || n_scenes == 0) return fail(ctx, AE_MPM_EINVAL, "no scenes");
  if (opts && opts->precision == 64) return fail(ctx, AE_MPM_EINVAL, "a batch runs f32 worlds");
  int rc = set_device(ctx);
  if (rc) return rc;
  std::vector<uint64_t> caps(n_scenes);
  for (uint32_t i = 0; i < n_scenes; ++i) caps[i] = scenes[i].max_particles;
  std::vector<uint32_t> first(n_scenes + 1);
  const uint32_t g_n = ae_mpm_batch_partition(caps.data(), n_scenes, n_groups, first.data());
  first.resize(g_n + 1);
  auto* b = new ae_mpm_batch;
  b->ctx = ctx;
  b->first = first;
  cudaError_t e = cudaStreamCreateWithFlags(&b->up, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->down, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete b;
    return fail(ctx, AE_MPM_ECUDA, cudaGetErrorString(e));
  }
  int least = 0, greatest = 0;  // numerically: greatest <= least
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  for (uint32_t g = 0; g < g_n; ++g) {
    const uint32_t k = first[g + 1] - first[g];
    const ae_mpm_exec_opts o = resolve_opts(ctx, scenes + first[g], k, opts);
    std::string why;
    int st = 0;
    WorldBase* w = aemp::make_world(scenes + first[g], k, o, why, &st);
    if (!w) {
      delete b;
      return fail(ctx, st ? st : AE_MPM_ECUDA, "batch group " + std::to_string(g) + ": " + why);
    }
    b->worlds.push_back(w);
    // earlier groups on higher stream priorities: the GPU serves group g first and fills its
    // kernels' launch gaps and tails with later groups' work, so group g finishes (and its
    // results start across PCIe) while later groups still compute
    const int prio = greatest + int(g) < least ? greatest + int(g) : least;
    if ((rc = w->set_stream_priority(prio))) {
      const std::string why2 = w->err;
      delete b;
      return fail(ctx, rc, "batch group " + std::to_string(g) + ": " + why2);
    }
  }
  *out = b;
  return AE_MPM_OK;
}

int ae_mpm_batch_destroy(ae_mpm_batch* batch) {
  if (!batch) return AE_MPM_EINVAL;
  cudaSetDevice(batch->ctx->device);
  delete batch;
  return AE_MPM_OK;
}

uint32_t ae_mpm_batch_groups(const ae_mpm_batch* batch, uint32_t* first_scene) {
  if (!batch) return 0;
  const uint32_t g_n = uint32_t(batch->worlds.size());
  if (first_scene)
    for (uint32_t g = 0; g <= g_n; ++g) first_scene[g] = batch->first[g];
  return g_n;
}

int ae_mpm_batch_run(ae_mpm_batch* batch, const ae_mpm_particles* in, const uint64_t* counts, ae_mpm_particles* out,
                     uint32_t n_substeps) {
  if (!batch) return AE_MPM_EINVAL;
  ae_mpm_ctx* ctx = batch->ctx;
  if (!in || !counts || !out) return fail(ctx, AE_MPM_EINVAL, "null view or count array");
  int rc = set_device(ctx);
  if (rc) return rc;
  const uint32_t g_n = uint32_t(batch->worlds.size());
  std::vector<uint32_t> ids;
  for (uint32_t i = 0; i < batch->first.back(); ++i) ids.push_back(i);
  // AE_MPM_BATCH_PROFILE: a timeline of the call on stderr (device events per group and stream,
  // host time after each queueing call), in ms from the start of the call
  const bool prof = std::getenv("AE_MPM_BATCH_PROFILE") != nullptr;
  std::vector<cudaEvent_t> pev;
  std::vector<double> host_ms;
  const auto h0 = std::chrono::steady_clock::now();
  auto host_mark = [&]() {
    if (prof) host_ms.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count());
  };
  auto mark = [&](cudaStream_t st) {
    if (!prof) return;
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) == cudaSuccess) cudaEventRecord(e, st);
    pev.push_back(e);
  };
  mark(batch->up);
  // every group's inputs queue on the upload stream in group order; group g's substeps start
  // when its inputs are in (served before later groups' by stream priority), and its results
  // leave on the download stream while later groups compute
  auto group_fail = [&](uint32_t g, int code) {  // nothing may still read or write the caller's buffers
    cudaStreamSynchronize(batch->up);
    cudaStreamSynchronize(batch->down);
    for (WorldBase* w : batch->worlds) cudaStreamSynchronize(w->stream());
    return fail(ctx, code, "batch group " + std::to_string(g) + ": " + batch->worlds[g]->err);
  };
  for (uint32_t g = 0; g < g_n; ++g) {
    const uint32_t f = batch->first[g], k = batch->first[g + 1] - f;
    if ((rc = batch->worlds[g]->upload_many(k, ids.data(), in + f, counts + f, batch->up))) return group_fail(g, rc);
    mark(batch->up);
    host_mark();
  }
  for (uint32_t g = 0; g < g_n; ++g) {
    WorldBase* w = batch->worlds[g];
    mark(w->stream());
    if ((rc = w->step(n_substeps))) return group_fail(g, rc);
    mark(w->stream());
    host_mark();
  }
  for (uint32_t g = 0; g < g_n; ++g) {
    const uint32_t f = batch->first[g], k = batch->first[g + 1] - f;
    if ((rc = batch->worlds[g]->download_many(k, ids.data(), out + f, batch->down))) return group_fail(g, rc);
    mark(batch->down);
    host_mark();
  }
  cudaError_t e = cudaStreamSynchronize(batch->down);
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, cudaGetErrorString(e));
  if (prof) {
    host_mark();
    for (cudaEvent_t ev : pev)
      if (ev) cudaEventSynchronize(ev);
    auto at = [&](size_t i) {
      float ms = 0.f;
      if (pev[0] && pev[i]) cudaEventElapsedTime(&ms, pev[0], pev[i]);
      return double(ms);
    };
    std::fprintf(stderr, "ae_mpm_batch: %u groups, %u substeps\n", g_n, n_substeps);
    for (uint32_t g = 0; g < g_n; ++g)
      std::fprintf(stderr, "  group %u: inputs in %.2f, substeps %.2f-%.2f, results out %.2f ms\n", g, at(1 + g),
                   at(1 + g_n + 2 * g), at(2 + g_n + 2 * g), at(1 + 3 * g_n + g));
    std::fprintf(stderr, "  host after each call:");
    for (double h : host_ms) std::fprintf(stderr, " %.2f", h);
    std::fprintf(stderr, " ms\n");
    for (cudaEvent_t ev : pev)
      if (ev) cudaEventDestroy(ev);
  }
  // error words of every group (the first reported wins; every group's results are in place)
  int first_rc = AE_MPM_OK;
  for (uint32_t g = 0; g < g_n; ++g) {
    rc = batch->worlds[g]->sync();
    if (rc && !first_rc) first_rc = fail(ctx, rc, "batch group " + std::to_string(g) + ": " + batch->worlds[g]->err);
  }
  return first_rc;
}

int ae_mpm_world_totals(ae_mpm_world* world, uint32_t scene, double out[5]) {
  if (world && !out) return fail(world->ctx, AE_MPM_EINVAL, "null output");
  AE_WORLD_CALL(world->w->totals(scene, out));
}
int ae_mpm_world_errors(ae_mpm_world* world, uint32_t scene, uint32_t* error_word, uint64_t counters[3]) {
  AE_WORLD_CALL(world->w->errors(scene, error_word, counters));
}

int ae_mpm_world_stage_times(ae_mpm_world* world, uint32_t n_substeps, double out_us[5]) {
  if (world && !out_us) return fail(world->ctx, AE_MPM_EINVAL, "null output");
  double six[6];
  if (!world) return AE_MPM_EINVAL;
  int rc = set_device(world->ctx);
  if (rc) return rc;
  rc = world->w->stage_times(n_substeps, six);
  if (rc) return fail(world->ctx, rc, world->w->err);
  for (int k = 0; k < 5; ++k) out_us[k] = six[k];
  return AE_MPM_OK;
}

int ae_mpm_world_stage_times_split(ae_mpm_world* world, uint32_t n_substeps, double out_us[6]) {
  if (world && !out_us) return fail(world->ctx, AE_MPM_EINVAL, "null output");
  AE_WORLD_CALL(world->w->stage_times(n_substeps, out_us));
}

int ae_mpm_world_launch_count(const ae_mpm_world* world, uint64_t* launches) {
  if (!world || !launches) return AE_MPM_EINVAL;
  *launches = world->w->last_launches();
  return AE_MPM_OK;
}

void* ae_mpm_world_stream(ae_mpm_world* world) { return world ? static_cast<void*>(world->w->stream()) : nullptr; }

uint64_t ae_mpm_world_particles(const ae_mpm_world* world) { return world ? world->w->particles() : 0; }
uint64_t ae_mpm_world_scene_particles(const ae_mpm_world* world, uint32_t scene) {
  return world ? world->w->scene_count(scene) : 0;
}

static int host_sort(ae_mpm_ctx* ctx, const uint32_t* keys, uint64_t n, uint32_t key_bits, uint32_t* sorted_keys_out,
                     uint32_t* perm_out, bool counting) {
  if (!ctx) return AE_MPM_EINVAL;
  if (n == 0) return AE_MPM_OK;
  if (!keys || !sorted_keys_out || !perm_out || key_bits == 0 || key_bits > (counting ? 16u : 32u) ||
      n >= (1ull << 32))
    return fail(ctx, AE_MPM_EINVAL, counting ? "bad counting sort arguments" : "bad radix sort arguments");
  int rc = set_device(ctx);
  if (rc) return rc;
  if (ctx->sort.n_cap < n) {
    cudaError_t e = aemp::sort_scratch_alloc(ctx->sort, n);
    if (e != cudaSuccess) return fail(ctx, AE_MPM_ENOMEM, cudaGetErrorString(e));
  }
  if (ctx->sort_keys_cap < n) {
    cudaFree(ctx->sort_keys);
    ctx->sort_keys = nullptr;
    ctx->sort_keys_cap = 0;
    cudaError_t e = cudaMalloc(&ctx->sort_keys, sizeof(uint32_t) * n);
    if (e != cudaSuccess) return fail(ctx, AE_MPM_ENOMEM, cudaGetErrorString(e));
    ctx->sort_keys_cap = n;
  }
  cudaError_t e = cudaMemcpy(ctx->sort_keys, keys, sizeof(uint32_t) * n, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, cudaGetErrorString(e));
  const uint32_t *sk = nullptr, *pm = nullptr;
  if (counting)
    aemp::counting_sort_pairs(ctx->sort_keys, n, int(key_bits), ctx->sort, 0, &sk, &pm);
  else
    aemp::radix_sort_pairs(ctx->sort_keys, n, int(key_bits), ctx->sort, 0, &sk, &pm);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(sorted_keys_out, sk, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(perm_out, pm, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, cudaGetErrorString(e));
  return AE_MPM_OK;
}

int ae_mpm_radix_sort_keys(ae_mpm_ctx* ctx, const uint32_t* keys, uint64_t n, uint32_t key_bits,
                           uint32_t* sorted_keys_out, uint32_t* perm_out) {
  return host_sort(ctx, keys, n, key_bits, sorted_keys_out, perm_out, false);
}

int ae_mpm_counting_sort_keys(ae_mpm_ctx* ctx, const uint32_t* keys, uint64_t n, uint32_t key_bits,
                              uint32_t* sorted_keys_out, uint32_t* perm_out) {
  return host_sort(ctx, keys, n, key_bits, sorted_keys_out, perm_out, true);
}

// ---------------------------------------------------------------------------------------------
// engine tick passes around the substep (simulation.rs:495-532, 612-679, 877-966)
// ---------------------------------------------------------------------------------------------
int ae_mpm_lod_classify(ae_mpm_ctx* ctx, const float* pos, const uint8_t* active, uint64_t count,
                        const float player[3], float near_dist, float mid_dist, uint64_t max_near, uint64_t* near_out,
                        uint64_t* n_near, uint64_t* mid_out, uint64_t* n_mid, uint64_t* far_out, uint64_t* n_far) {
  if (!ctx) return AE_MPM_EINVAL;
  if (!player || !n_near || !n_mid || !n_far || (count && (!pos || !near_out || !mid_out || !far_out)) ||
      count >= (1ull << 32))
    return fail(ctx, AE_MPM_EINVAL, "lod_classify: null array or more than 2^32 - 1 particles");
  *n_near = *n_mid = *n_far = 0;
  if (count == 0) return AE_MPM_OK;
  int rc = set_device(ctx);
  if (rc) return rc;
  aemp::LodWork* lw = lod_work(ctx);
  uint64_t counts[3] = {0, 0, 0};
  cudaError_t e;
  if (is_device_ptr(pos)) {
    e = lw->classify(pos, active, count, player, near_dist, mid_dist, max_near, near_out, mid_out, far_out, counts, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  } else {
    // device copies of pos and active, three output lists; each region starts on a 16-byte boundary
    const size_t b_pos = (sizeof(float) * 3 * count + 15) & ~size_t(15), b_act = active ? ((count + 15) & ~size_t(15)) : 0;
    rc = ensure_dstage(ctx, b_pos + b_act + 3 * sizeof(uint64_t) * count);
    if (rc) return rc;
    char* d = static_cast<char*>(ctx->dstage);
    float* dpos = reinterpret_cast<float*>(d);
    uint8_t* dact = active ? reinterpret_cast<uint8_t*>(d + b_pos) : nullptr;
    uint64_t* dl = reinterpret_cast<uint64_t*>(d + b_pos + b_act);
    e = cudaMemcpyAsync(dpos, pos, sizeof(float) * 3 * count, cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess && active) e = cudaMemcpyAsync(dact, active, count, cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess)
      e = lw->classify(dpos, dact, count, player, near_dist, mid_dist, max_near, dl, dl + count, dl + 2 * count, counts, 0);
    if (e == cudaSuccess && counts[0]) e = cudaMemcpyAsync(near_out, dl, sizeof(uint64_t) * counts[0], cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess && counts[1])
      e = cudaMemcpyAsync(mid_out, dl + count, sizeof(uint64_t) * counts[1], cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess && counts[2])
      e = cudaMemcpyAsync(far_out, dl + 2 * count, sizeof(uint64_t) * counts[2], cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  }
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, std::string("lod_classify: ") + cudaGetErrorString(e));
  *n_near = counts[0];
  *n_mid = counts[1];
  *n_far = counts[2];
  return AE_MPM_OK;
}

int ae_mpm_far_field_update(ae_mpm_ctx* ctx, float* pos, float* vel, float* temperature, uint64_t count,
                            const uint64_t* far_idx, uint64_t n_far, const float* coarse_temperature, uint32_t coarse_n,
                            float coarse_dx, const float coarse_origin[3], float far_dt) {
  if (!ctx) return AE_MPM_EINVAL;
  if (!coarse_origin || (n_far && (!pos || !vel || !temperature || !far_idx || !coarse_temperature)) || coarse_n == 0 ||
      uint64_t(coarse_n) * coarse_n * coarse_n >= (1ull << 31))
    return fail(ctx, AE_MPM_EINVAL, "far_field_update: null array or coarse_n out of range");
  if (n_far == 0) return AE_MPM_OK;
  int rc = set_device(ctx);
  if (rc) return rc;
  aemp::LodWork* lw = lod_work(ctx);
  const uint64_t cells = uint64_t(coarse_n) * coarse_n * coarse_n;
  cudaError_t e;
  if (is_device_ptr(pos)) {
    e = lw->far_field(pos, vel, temperature, far_idx, n_far, coarse_temperature, coarse_n, coarse_dx, coarse_origin,
                      far_dt, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  } else {
    for (uint64_t k = 0; k < n_far; ++k)
      if (far_idx[k] >= count) return fail(ctx, AE_MPM_EINVAL, "far_field_update: index out of range");
    if (4 * n_far >= count) {
      // most particles are far: copy the whole arrays and the index list, let the device gather
      // and scatter, and copy the arrays back (no host-side loop over the particles)
      auto up16 = [](size_t b) { return (b + 15) & ~size_t(15); };
      const size_t b3 = up16(12 * count), b1 = up16(4 * count), bi = up16(8 * n_far), bc = up16(4 * cells);
      rc = ensure_dstage(ctx, 2 * b3 + b1 + bi + bc);
      if (rc) return rc;
      char* d = static_cast<char*>(ctx->dstage);
      float* dpos = reinterpret_cast<float*>(d);
      float* dvel = reinterpret_cast<float*>(d + b3);
      float* dtemp = reinterpret_cast<float*>(d + 2 * b3);
      uint64_t* didx = reinterpret_cast<uint64_t*>(d + 2 * b3 + b1);
      float* dcoarse = reinterpret_cast<float*>(d + 2 * b3 + b1 + bi);
      e = cudaMemcpyAsync(dpos, pos, 12 * count, cudaMemcpyHostToDevice, 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(dvel, vel, 12 * count, cudaMemcpyHostToDevice, 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(dtemp, temperature, 4 * count, cudaMemcpyHostToDevice, 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(didx, far_idx, 8 * n_far, cudaMemcpyHostToDevice, 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(dcoarse, coarse_temperature, 4 * cells, cudaMemcpyHostToDevice, 0);
      if (e == cudaSuccess)
        e = lw->far_field(dpos, dvel, dtemp, didx, n_far, dcoarse, coarse_n, coarse_dx, coarse_origin, far_dt, 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(pos, dpos, 12 * count, cudaMemcpyDeviceToHost, 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(vel, dvel, 12 * count, cudaMemcpyDeviceToHost, 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(temperature, dtemp, 4 * count, cudaMemcpyDeviceToHost, 0);
      if (e == cudaSuccess) e = cudaStreamSynchronize(0);
      if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, std::string("far_field_update: ") + cudaGetErrorString(e));
      return AE_MPM_OK;
    }
    // few far particles: gather them (pos, vel, temperature: 7 floats each) and the field, one
    // copy each way
    const size_t bytes = sizeof(float) * (7 * n_far + cells);
    rc = ensure_pinned(ctx, bytes);
    if (rc) return rc;
    rc = ensure_dstage(ctx, bytes);
    if (rc) return rc;
    float* h = ctx->pin;
    for (uint64_t k = 0; k < n_far; ++k) {
      const uint64_t i = far_idx[k];
      std::memcpy(h + 3 * k, pos + 3 * i, sizeof(float) * 3);
      std::memcpy(h + 3 * (n_far + k), vel + 3 * i, sizeof(float) * 3);
      h[6 * n_far + k] = temperature[i];
    }
    std::memcpy(h + 7 * n_far, coarse_temperature, sizeof(float) * cells);
    float* d = static_cast<float*>(ctx->dstage);
    e = cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess)
      e = lw->far_field(d, d + 3 * n_far, d + 6 * n_far, nullptr, n_far, d + 7 * n_far, coarse_n, coarse_dx,
                        coarse_origin, far_dt, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(float) * 7 * n_far, cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e == cudaSuccess)
      for (uint64_t k = 0; k < n_far; ++k) {
        const uint64_t i = far_idx[k];
        pos[3 * i + 1] = h[3 * k + 1];
        vel[3 * i + 1] = h[3 * (n_far + k) + 1];
        temperature[i] = h[6 * n_far + k];
      }
  }
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, std::string("far_field_update: ") + cudaGetErrorString(e));
  return AE_MPM_OK;
}

int ae_mpm_coarse_field_update(ae_mpm_ctx* ctx, const float* pos, const float* mass, const float* temperature,
                               const uint8_t* active, uint64_t count, const uint64_t* near_idx, uint64_t n_near,
                               float* coarse_temperature, uint32_t coarse_n, float coarse_dx,
                               const float coarse_origin[3], float dt) {
  if (!ctx) return AE_MPM_EINVAL;
  if (!coarse_origin || !coarse_temperature || (n_near && (!pos || !mass || !temperature || !near_idx)) ||
      coarse_n == 0 || uint64_t(coarse_n) * coarse_n * coarse_n >= (1ull << 31) || n_near >= (1ull << 32))
    return fail(ctx, AE_MPM_EINVAL, "coarse_field_update: null array or size out of range");
  int rc = set_device(ctx);
  if (rc) return rc;
  aemp::LodWork* lw = lod_work(ctx);
  const uint64_t cells = uint64_t(coarse_n) * coarse_n * coarse_n;
  cudaError_t e;
  if (is_device_ptr(coarse_temperature)) {
    e = lw->coarse_field(pos, mass, temperature, active, near_idx, n_near, coarse_temperature, coarse_n, coarse_dx,
                         coarse_origin, dt, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  } else {
    for (uint64_t k = 0; k < n_near; ++k)
      if (near_idx[k] >= count) return fail(ctx, AE_MPM_EINVAL, "coarse_field_update: index out of range");
    // gather the near particles (pos, mass, temperature: 5 floats; active: 1 byte) and the field
    const size_t b_f = sizeof(float) * (5 * n_near + cells), b_a = (n_near + 15) & ~uint64_t(15);
    rc = ensure_pinned(ctx, b_f + b_a);
    if (rc) return rc;
    rc = ensure_dstage(ctx, b_f + b_a);
    if (rc) return rc;
    float* h = ctx->pin;
    uint8_t* ha = reinterpret_cast<uint8_t*>(h + 5 * n_near + cells);
    for (uint64_t k = 0; k < n_near; ++k) {
      const uint64_t i = near_idx[k];
      std::memcpy(h + 3 * k, pos + 3 * i, sizeof(float) * 3);
      h[3 * n_near + k] = mass[i];
      h[4 * n_near + k] = temperature[i];
      ha[k] = active ? active[i] : uint8_t(1);
    }
    std::memcpy(h + 5 * n_near, coarse_temperature, sizeof(float) * cells);
    float* d = static_cast<float*>(ctx->dstage);
    uint8_t* da = reinterpret_cast<uint8_t*>(d + 5 * n_near + cells);
    e = cudaMemcpyAsync(d, h, b_f + n_near, cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess)
      e = lw->coarse_field(d, d + 3 * n_near, d + 4 * n_near, da, nullptr, n_near, d + 5 * n_near, coarse_n, coarse_dx,
                           coarse_origin, dt, 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(coarse_temperature, d + 5 * n_near, sizeof(float) * cells, cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  }
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, std::string("coarse_field_update: ") + cudaGetErrorString(e));
  return AE_MPM_OK;
}

int ae_mpm_mpss_housekeeping(ae_mpm_ctx* ctx, float* pos, float* vel, float* temperature, uint8_t* phase,
                             const uint16_t* material_idx, const uint8_t* active, uint64_t count,
                             const float bounds_min[3], const float bounds_max[3], float min_temp, float max_temp,
                             uint32_t passes, uint32_t* transitions) {
  if (!ctx) return AE_MPM_EINVAL;
  if (!transitions || !bounds_min || !bounds_max || (passes & ~7u) ||
      (count && (((passes & 1u) && (!pos || !vel)) || ((passes & 6u) && !temperature) ||
                 ((passes & 4u) && (!phase || !material_idx)))))
    return fail(ctx, AE_MPM_EINVAL, "mpss_housekeeping: null array for a selected pass, or unknown pass bits");
  *transitions = 0;
  if (count == 0 || passes == 0) return AE_MPM_OK;
  int rc = set_device(ctx);
  if (rc) return rc;
  aemp::LodWork* lw = lod_work(ctx);
  const bool b1 = passes & 1u, b2 = (passes & 6u) != 0, b4 = passes & 4u;
  const void* probe = b1 ? static_cast<const void*>(pos) : static_cast<const void*>(temperature);
  cudaError_t e;
  if (is_device_ptr(probe)) {
    e = lw->housekeeping(pos, vel, temperature, phase, material_idx, active, count, bounds_min, bounds_max, min_temp,
                         max_temp, passes, transitions, 0);
  } else {
    // device copies of the arrays the selected passes use, 16-byte aligned regions
    auto up16 = [](size_t b) { return (b + 15) & ~size_t(15); };
    const size_t bp = b1 ? up16(12 * count) : 0, bt = b2 ? up16(4 * count) : 0, bph = b4 ? up16(count) : 0,
                 bm = b4 ? up16(2 * count) : 0, ba = active ? up16(count) : 0;
    rc = ensure_dstage(ctx, 2 * bp + bt + bph + bm + ba);
    if (rc) return rc;
    char* d = static_cast<char*>(ctx->dstage);
    float* dpos = b1 ? reinterpret_cast<float*>(d) : nullptr;
    float* dvel = b1 ? reinterpret_cast<float*>(d + bp) : nullptr;
    float* dt = b2 ? reinterpret_cast<float*>(d + 2 * bp) : nullptr;
    uint8_t* dph = b4 ? reinterpret_cast<uint8_t*>(d + 2 * bp + bt) : nullptr;
    uint16_t* dm = b4 ? reinterpret_cast<uint16_t*>(d + 2 * bp + bt + bph) : nullptr;
    uint8_t* da = active ? reinterpret_cast<uint8_t*>(d + 2 * bp + bt + bph + bm) : nullptr;
    e = cudaSuccess;
    if (b1) e = cudaMemcpyAsync(dpos, pos, 12 * count, cudaMemcpyHostToDevice, 0);
    if (b1 && e == cudaSuccess) e = cudaMemcpyAsync(dvel, vel, 12 * count, cudaMemcpyHostToDevice, 0);
    if (b2 && e == cudaSuccess) e = cudaMemcpyAsync(dt, temperature, 4 * count, cudaMemcpyHostToDevice, 0);
    if (b4 && e == cudaSuccess) e = cudaMemcpyAsync(dph, phase, count, cudaMemcpyHostToDevice, 0);
    if (b4 && e == cudaSuccess) e = cudaMemcpyAsync(dm, material_idx, 2 * count, cudaMemcpyHostToDevice, 0);
    if (active && e == cudaSuccess) e = cudaMemcpyAsync(da, active, count, cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess)
      e = lw->housekeeping(dpos, dvel, dt, dph, dm, da, count, bounds_min, bounds_max, min_temp, max_temp, passes,
                           transitions, 0);
    if (b1 && e == cudaSuccess) e = cudaMemcpyAsync(pos, dpos, 12 * count, cudaMemcpyDeviceToHost, 0);
    if (b1 && e == cudaSuccess) e = cudaMemcpyAsync(vel, dvel, 12 * count, cudaMemcpyDeviceToHost, 0);
    if ((passes & 2u) && e == cudaSuccess) e = cudaMemcpyAsync(temperature, dt, 4 * count, cudaMemcpyDeviceToHost, 0);
    if (b4 && e == cudaSuccess) e = cudaMemcpyAsync(phase, dph, count, cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  }
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, std::string("mpss_housekeeping: ") + cudaGetErrorString(e));
  return AE_MPM_OK;
}

void ae_mpm_ck_config_default(ae_mpm_ck_config* out) {
  if (!out) return;
  // CkMpmConfig::default(), ck_mpm.rs:61-77
  *out = ae_mpm_ck_config{};
  out->dt = 1.0f / 240.0f;
  out->grid_h = 0.05f;
  out->grid_n = 32;
  out->gravity[1] = -9.81f;
  out->youngs_modulus = 1e5f;
  out->poissons_ratio = 0.3f;
  out->density = 1000.0f;
  for (int k = 0; k < 3; ++k) out->bounds_min[k] = -1.0f, out->bounds_max[k] = 1.0f;
  out->restitution = 0.3f;
  out->dual_grid = 1;
}

namespace {
// ae_mpm_ck_step / _timed / _deterministic: host records are staged through the context
int ck_run(ae_mpm_ctx* ctx, ae_mpm_ck_particle* particles, uint64_t n, const ae_mpm_ck_config* config, uint32_t steps,
           double* kernel_ms, bool deterministic) {
  if (!ctx) return AE_MPM_EINVAL;
  if (kernel_ms) kernel_ms[0] = kernel_ms[1] = 0.0;
  if (deterministic && n >= (1ull << 32))
    return fail(ctx, AE_MPM_EINVAL, "ck_step_deterministic: more than 2^32 - 1 particles");
  if (!config || (n && !particles)) return fail(ctx, AE_MPM_EINVAL, "ck_step: null config or particles");
  if (config->grid_n > 1024) return fail(ctx, AE_MPM_EINVAL, "ck_step: grid_n above 1024");
  if (n == 0 || steps == 0) return AE_MPM_OK;
  int rc = set_device(ctx);
  if (rc) return rc;
  aemp::CkWork* ck = ck_work(ctx);
  cudaError_t e;
  auto run = [&](ae_mpm_ck_particle* p) {
    return deterministic ? ck->step_deterministic(p, n, *config, steps, 0) : ck->step(p, n, *config, steps, 0, kernel_ms);
  };
  if (is_device_ptr(particles)) {
    e = run(particles);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  } else {
    const size_t bytes = n * sizeof(ae_mpm_ck_particle);
    rc = ensure_dstage(ctx, bytes);
    if (rc) return rc;
    auto* d = static_cast<ae_mpm_ck_particle*>(ctx->dstage);
    e = cudaMemcpyAsync(d, particles, bytes, cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess) e = run(d);
    if (e == cudaSuccess) e = cudaMemcpyAsync(particles, d, bytes, cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  }
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, std::string("ck_step: ") + cudaGetErrorString(e));
  return AE_MPM_OK;
}
}  // namespace

int ae_mpm_ck_step(ae_mpm_ctx* ctx, ae_mpm_ck_particle* particles, uint64_t n, const ae_mpm_ck_config* config,
                   uint32_t steps) {
  return ck_run(ctx, particles, n, config, steps, nullptr, false);
}

int ae_mpm_ck_step_timed(ae_mpm_ctx* ctx, ae_mpm_ck_particle* particles, uint64_t n, const ae_mpm_ck_config* config,
                         uint32_t steps, double kernel_ms[2]) {
  return ck_run(ctx, particles, n, config, steps, kernel_ms, false);
}

int ae_mpm_ck_step_deterministic(ae_mpm_ctx* ctx, ae_mpm_ck_particle* particles, uint64_t n,
                                 const ae_mpm_ck_config* config, uint32_t steps) {
  return ck_run(ctx, particles, n, config, steps, nullptr, true);
}

int ae_mpm_ck_stats_compute(ae_mpm_ctx* ctx, const ae_mpm_ck_particle* particles, uint64_t n, ae_mpm_ck_stats* out) {
  if (!ctx) return AE_MPM_EINVAL;
  if (!out || (n && !particles)) return fail(ctx, AE_MPM_EINVAL, "ck_stats: null particles or output");
  int rc = set_device(ctx);
  if (rc) return rc;
  aemp::CkWork* ck = ck_work(ctx);
  cudaError_t e;
  if (n == 0 || is_device_ptr(particles)) {
    e = ck->stats(particles, n, out, 0);
  } else {
    const size_t bytes = n * sizeof(ae_mpm_ck_particle);
    rc = ensure_dstage(ctx, bytes);
    if (rc) return rc;
    auto* d = static_cast<ae_mpm_ck_particle*>(ctx->dstage);
    e = cudaMemcpyAsync(d, particles, bytes, cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess) e = ck->stats(d, n, out, 0);
  }
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, std::string("ck_stats: ") + cudaGetErrorString(e));
  return AE_MPM_OK;
}

int ae_mpm_ck_weights(ae_mpm_ctx* ctx, const float* x, uint64_t n, float h, float* w, float* dw) {
  if (!ctx) return AE_MPM_EINVAL;
  if (n && (!x || !w || !dw)) return fail(ctx, AE_MPM_EINVAL, "ck_weights: null array");
  if (n == 0) return AE_MPM_OK;
  int rc = set_device(ctx);
  if (rc) return rc;
  aemp::CkWork* ck = ck_work(ctx);
  cudaError_t e;
  if (is_device_ptr(x)) {
    e = ck->weights(x, n, h, w, dw, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  } else {
    const size_t b = (4 * n + 15) & ~size_t(15);
    rc = ensure_dstage(ctx, 3 * b);
    if (rc) return rc;
    char* d = static_cast<char*>(ctx->dstage);
    float* dx = reinterpret_cast<float*>(d);
    float* dwt = reinterpret_cast<float*>(d + b);
    float* dg = reinterpret_cast<float*>(d + 2 * b);
    e = cudaMemcpyAsync(dx, x, 4 * n, cudaMemcpyHostToDevice, 0);
    if (e == cudaSuccess) e = ck->weights(dx, n, h, dwt, dg, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(w, dwt, 4 * n, cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dw, dg, 4 * n, cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  }
  if (e != cudaSuccess) return fail(ctx, AE_MPM_ECUDA, std::string("ck_weights: ") + cudaGetErrorString(e));
  return AE_MPM_OK;
}

// Autotuner: P2G variant x particles per block x sort interval, timed with CUDA events on the
// world's stream from the same starting state (snapshot restored between trials).
int ae_mpm_world_autotune(ae_mpm_world* world, uint32_t substeps_per_trial, ae_mpm_tune_result* out) {
  if (!world) return AE_MPM_EINVAL;
  ae_mpm_ctx* ctx = world->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  WorldBase* w = world->w;
  if (substeps_per_trial == 0) substeps_per_trial = 8;
  const ae_mpm_exec_opts saved = w->opts();
  if ((rc = w->snapshot(false))) return fail(ctx, rc, w->err);
  std::vector<int> variants = {AE_MPM_P2G_LANES, AE_MPM_P2G_TILE, AE_MPM_P2G_WARP_AGG, AE_MPM_P2G_GLOBAL};
  std::vector<int> threads = {128, 256};
  std::vector<int> intervals = {1, 2, 4, 8, 16, 32};
  if (saved.deterministic) {
    variants = {saved.p2g_variant};
    intervals = {1};
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  ae_mpm_tune_result best{saved.p2g_variant, saved.block_threads, saved.sort_interval, 1e30f};
  for (int v : variants)
    for (int t : threads)
      for (int si : intervals) {
        w->opts().p2g_variant = v;
        w->opts().block_threads = t;
        w->opts().sort_interval = si;
        w->invalidate_graph();
        if ((rc = w->snapshot(true))) break;
        // warm-up reaches the graph path too; each trial then times whole graph periods
        uint32_t trial = std::max<uint32_t>(substeps_per_trial, uint32_t(2 * si));
        if ((rc = w->step(trial))) break;
        cudaStream_t s = w->stream();
        cudaEventRecord(e0, s);
        if ((rc = w->step(trial))) break;
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        float us = 1000.0f * ms / float(trial);
        if (us < best.us_per_substep) best = ae_mpm_tune_result{v, t, si, us};
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    w->opts() = saved;
    w->invalidate_graph();
    w->snapshot(true);
    return fail(ctx, rc, w->err);
  }
  w->opts().p2g_variant = best.p2g_variant;
  w->opts().block_threads = best.block_threads;
  w->opts().sort_interval = best.sort_interval;
  w->invalidate_graph();
  if ((rc = w->snapshot(true))) return fail(ctx, rc, w->err);
  ctx->tuned[world->sig] = best;
  if (out) *out = best;
  return AE_MPM_OK;
}

}  // extern "C"
