// ae_mpm_lod.cu -- the engine tick's particle passes around the MPM substep, on the device
// (ae_engine/src/managers/simulation.rs).  Every pass restates the reference's f32 arithmetic
// operation by operation with explicitly rounded intrinsics (__fmul_rn / __fadd_rn / __fdiv_rn are
// never fused into FMAs), so results match the CPU path bit for bit:
//
//   classify      stable 3-way partition of the particles by squared distance to the player
//                 (count per 2048-particle tile, scan of the tile counts, scatter in index order).
//                 When more than max_near fall within near_dist, a one-block radix select over
//                 the near candidates' squared distances (non-negative floats, so their bit patterns
//                 order like the values) flags the max_near closest, and a second partition splits
//                 the candidates into the kept near list and the tail appended to the mid list.
//   far_field     one thread per far particle: gravity on y, position, nearest-cell sample.
//   coarse_field  the near particles' cells are radix-sorted (stable, so each cell keeps the
//                 reference's index order), each cell's run is located, and one thread per cell
//                 sums its run sequentially, which
//                 reproduces the reference's serial accumulation exactly; then relaxation and one
//                 FTCS step, one thread per cell.
#include "ae_mpm_lod.cuh"

#include <algorithm>
#include <cmath>

namespace aemp {

namespace {

constexpr int kPT = 256, kPItems = 8, kPTile = kPT * kPItems;  // partition: 2048 items per tile
constexpr int kPWarps = kPT / 32;

__device__ __forceinline__ int64_t as_isize(float v) {  // Rust `f32 as isize`
  if (v != v) return 0;
  if (v >= 9.2233720368547758e18f) return INT64_MAX;
  if (v <= -9.2233720368547758e18f) return INT64_MIN;
  return static_cast<int64_t>(v);
}

__device__ __forceinline__ uint32_t warp_scan_incl(uint32_t x, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// class of particle idx: 0 near, 1 mid, 2 far, 3 skipped (inactive); simulation.rs:499-513
struct PosClass {
  const float* pos;
  const uint8_t* active;
  float px, py, pz, near2, mid2;
  __device__ __forceinline__ int operator()(uint64_t idx, uint64_t& item, float& d2) const {
    item = idx;
    d2 = 0.0f;
    if (active && !active[idx]) return 3;
    const float dx = __fsub_rn(pos[3 * idx], px), dy = __fsub_rn(pos[3 * idx + 1], py), dz = __fsub_rn(pos[3 * idx + 2], pz);
    d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    return d2 < near2 ? 0 : (d2 < mid2 ? 1 : 2);  // NaN compares false: far
  }
};

// near candidate k: 0 kept, 1 culled to mid
struct KeepClass {
  const uint64_t* near;
  const uint8_t* keep;
  __device__ __forceinline__ int operator()(uint64_t k, uint64_t& item, float& d2) const {
    item = near[k];
    d2 = 0.0f;
    return keep[k] ? 0 : 1;
  }
};

template <class Cls>
__global__ void __launch_bounds__(kPT) part_count(Cls cls, uint64_t n, uint32_t* tile_counts, uint32_t tiles) {
  __shared__ uint32_t wc[kPWarps][3];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t base = uint64_t(blockIdx.x) * kPTile + uint64_t(w) * (32 * kPItems);
  uint32_t c0 = 0, c1 = 0, c2 = 0;
#pragma unroll
  for (int r = 0; r < kPItems; ++r) {
    const uint64_t idx = base + uint64_t(r) * 32 + lane;
    uint64_t item;
    float d2;
    const int k = idx < n ? cls(idx, item, d2) : 3;
    c0 += __popc(__ballot_sync(0xffffffffu, k == 0));
    c1 += __popc(__ballot_sync(0xffffffffu, k == 1));
    c2 += __popc(__ballot_sync(0xffffffffu, k == 2));
  }
  if (lane == 0) {
    wc[w][0] = c0;
    wc[w][1] = c1;
    wc[w][2] = c2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    uint32_t s = 0;
    for (int ww = 0; ww < kPWarps; ++ww) s += wc[ww][threadIdx.x];
    tile_counts[uint64_t(threadIdx.x) * tiles + blockIdx.x] = s;
  }
}

// one block: exclusive scan of each class's tile counts, and the class totals
__global__ void __launch_bounds__(1024) part_scan(const uint32_t* tile_counts, uint32_t* tile_offs, uint32_t tiles,
                                                  uint32_t* totals) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t carry;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int c = 0; c < 3; ++c) {
    if (tid == 0) carry = 0;
    __syncthreads();
    for (uint32_t start = 0; start < tiles; start += 1024) {
      const uint32_t i = start + tid;
      const uint32_t x = i < tiles ? tile_counts[uint64_t(c) * tiles + i] : 0u;
      const uint32_t incl = warp_scan_incl(x, lane);
      if (lane == 31) ws[w] = incl;
      __syncthreads();
      if (w == 0) {
        const uint32_t v = ws[lane];
        ws[lane] = warp_scan_incl(v, lane) - v;
      }
      __syncthreads();
      const uint32_t cc = carry;
      if (i < tiles) tile_offs[uint64_t(c) * tiles + i] = cc + ws[w] + incl - x;
      __syncthreads();
      if (tid == 1023) carry = cc + ws[w] + incl;
      __syncthreads();
    }
    if (tid == 0) totals[c] = carry;
    __syncthreads();
  }
}

// writes each item at its class's tile offset + rank in index order; class 1 lands at out1_base +
// position, class 0 optionally also writes its squared distance
template <class Cls>
__global__ void __launch_bounds__(kPT) part_scatter(Cls cls, uint64_t n, const uint32_t* tile_offs, uint32_t tiles,
                                                    uint64_t* out0, float* d2_0, uint64_t* out1, uint64_t out1_base,
                                                    uint64_t* out2) {
  __shared__ uint32_t wc[kPWarps][3];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t base = uint64_t(blockIdx.x) * kPTile + uint64_t(w) * (32 * kPItems);
  int k[kPItems];
  uint64_t item[kPItems];
  float d2[kPItems];
  uint32_t c0 = 0, c1 = 0, c2 = 0;
#pragma unroll
  for (int r = 0; r < kPItems; ++r) {
    const uint64_t idx = base + uint64_t(r) * 32 + lane;
    k[r] = idx < n ? cls(idx, item[r], d2[r]) : 3;
    c0 += __popc(__ballot_sync(0xffffffffu, k[r] == 0));
    c1 += __popc(__ballot_sync(0xffffffffu, k[r] == 1));
    c2 += __popc(__ballot_sync(0xffffffffu, k[r] == 2));
  }
  if (lane == 0) {
    wc[w][0] = c0;
    wc[w][1] = c1;
    wc[w][2] = c2;
  }
  __syncthreads();
  uint32_t wb[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    uint32_t s = tile_offs[uint64_t(q) * tiles + blockIdx.x];
    for (int ww = 0; ww < w; ++ww) s += wc[ww][q];
    wb[q] = s;
  }
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < kPItems; ++r) {
    const uint32_t m0 = __ballot_sync(0xffffffffu, k[r] == 0);
    const uint32_t m1 = __ballot_sync(0xffffffffu, k[r] == 1);
    const uint32_t m2 = __ballot_sync(0xffffffffu, k[r] == 2);
    if (k[r] == 0) {
      const uint32_t p = wb[0] + __popc(m0 & lt);
      out0[p] = item[r];
      if (d2_0) d2_0[p] = d2[r];
    } else if (k[r] == 1) {
      out1[out1_base + wb[1] + __popc(m1 & lt)] = item[r];
    } else if (k[r] == 2) {
      out2[wb[2] + __popc(m2 & lt)] = item[r];
    }
    wb[0] += __popc(m0);
    wb[1] += __popc(m1);
    wb[2] += __popc(m2);
  }
}

// One block: flags the k smallest of n keys (k >= 1, k < n), equal keys by position.  Four 8-bit
// radix-select passes find the k-th smallest key T and how many of the keys equal to T are kept;
// the keys below T and the first of those equal to T (a block-wide scan of per-thread counts over
// contiguous chunks gives their positional ranks) are flagged.
constexpr uint32_t kSelectSmemKeys = 40960;  // 160 KB: candidates up to this count are read once
__global__ void __launch_bounds__(1024) select_keep(const uint32_t* gkeys, uint32_t n, uint32_t k, uint8_t* keep) {
  extern __shared__ uint32_t skeys[];  // n keys when n <= kSelectSmemKeys (dynamic size 0 otherwise)
  __shared__ uint32_t hist[256];
  __shared__ uint32_t s_prefix, s_mask, s_rem;
  __shared__ uint32_t wsum[32];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const bool cached = n <= kSelectSmemKeys;
  if (cached)
    for (uint32_t i = tid; i < n; i += 1024) skeys[i] = gkeys[i];
  const uint32_t* keys = cached ? skeys : gkeys;
  if (tid == 0) {
    s_prefix = 0;
    s_mask = 0;
    s_rem = k;
  }
  __syncthreads();
  for (int shift = 24; shift >= 0; shift -= 8) {
    if (tid < 256) hist[tid] = 0;
    __syncthreads();
    const uint32_t prefix = s_prefix, mask = s_mask;
    for (uint32_t i = tid; i < n; i += 1024) {
      const uint32_t key = keys[i];
      if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (w == 0) {  // the digit whose bucket holds the s_rem-th smallest remaining key
      uint32_t c = 0;
#pragma unroll
      for (int b = 0; b < 8; ++b) c += hist[8 * lane + b];
      const uint32_t incl = warp_scan_incl(c, lane), rem = s_rem;
      const uint32_t hit = __ballot_sync(0xffffffffu, incl >= rem);
      if (lane == __ffs(hit) - 1) {
        uint32_t cum = incl - c;
        int d = 8 * lane;
        for (int b = 0; b < 8; ++b, ++d) {
          if (cum + hist[d] >= rem) break;
          cum += hist[d];
        }
        s_prefix = prefix | (uint32_t(d) << shift);
        s_mask = mask | (255u << shift);
        s_rem = rem - cum;
      }
    }
    __syncthreads();
  }
  const uint32_t T = s_prefix, rem = s_rem;
  const uint32_t chunk = (n + 1023) / 1024, c0 = min(n, tid * chunk), c1 = min(n, c0 + chunk);
  uint32_t eq = 0;
  for (uint32_t i = c0; i < c1; ++i) eq += keys[i] == T;
  const uint32_t incl = warp_scan_incl(eq, lane);
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    const uint32_t v = wsum[lane];
    wsum[lane] = warp_scan_incl(v, lane) - v;
  }
  __syncthreads();
  uint32_t before = wsum[w] + incl - eq;
  for (uint32_t i = c0; i < c1; ++i) {
    const uint32_t key = keys[i];
    bool kp = key < T;
    if (key == T) kp = before++ < rem;
    keep[i] = kp ? 1 : 0;
  }
}

// simulation.rs:626-650 per far particle
__global__ void far_field_kernel(float* pos, float* vel, float* temp, const uint64_t* idx, uint64_t n,
                                 const float* coarse, uint32_t cn, float cdx, float ox, float oy, float oz, float far_dt) {
  for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < n; k += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t i = idx ? idx[k] : k;
    const float vy = __fsub_rn(vel[3 * i + 1], __fmul_rn(9.81f, far_dt));
    vel[3 * i + 1] = vy;
    const float py = __fadd_rn(pos[3 * i + 1], __fmul_rn(vy, far_dt));
    pos[3 * i + 1] = py;
    const int64_t gx = as_isize(__fdiv_rn(__fsub_rn(pos[3 * i], ox), cdx));
    const int64_t gy = as_isize(__fdiv_rn(__fsub_rn(py, oy), cdx));
    const int64_t gz = as_isize(__fdiv_rn(__fsub_rn(pos[3 * i + 2], oz), cdx));
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx < int64_t(cn) && gy < int64_t(cn) && gz < int64_t(cn)) {
      const float field = coarse[gx + gy * int64_t(cn) + gz * int64_t(cn) * int64_t(cn)];
      const float t = temp[i];
      temp[i] = __fadd_rn(t, __fmul_rn(__fmul_rn(__fsub_rn(field, t), 0.02f), far_dt));
    }
  }
}

// cell key of near particle k (simulation.rs:889-905), or `dead` when skipped
__global__ void coarse_keys(const float* pos, const uint8_t* active, const uint64_t* idx, uint64_t n, uint32_t cn,
                            float inv_dx, float ox, float oy, float oz, uint32_t dead, uint32_t* keys) {
  for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < n; k += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t i = idx ? idx[k] : k;
    uint32_t key = dead;
    if (!active || active[i]) {
      const int64_t gx = as_isize(__fmul_rn(__fsub_rn(pos[3 * i], ox), inv_dx));
      const int64_t gy = as_isize(__fmul_rn(__fsub_rn(pos[3 * i + 1], oy), inv_dx));
      const int64_t gz = as_isize(__fmul_rn(__fsub_rn(pos[3 * i + 2], oz), inv_dx));
      if (gx >= 0 && gy >= 0 && gz >= 0 && gx < int64_t(cn) && gy < int64_t(cn) && gz < int64_t(cn))
        key = uint32_t(gx + gy * int64_t(cn) + gz * int64_t(cn) * int64_t(cn));
    }
    keys[k] = key;
  }
}

// the near particles' (temperature x mass, mass) in cell order (simulation.rs:906-908)
__global__ void coarse_gather(const float* mass, const float* temp, const uint64_t* idx, const uint32_t* perm,
                              uint64_t n, float* tm, float* m) {
  for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < n; k += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t kk = perm[k];
    const uint64_t i = idx ? idx[kk] : kk;
    const float mi = fmaxf(mass[i], 1e-6f);
    tm[k] = __fmul_rn(temp[i], mi);
    m[k] = mi;
  }
}

// each cell's run [start, end) in the sorted order (cells without particles keep start == end == 0)
__global__ void coarse_runs(const uint32_t* skeys, uint64_t n, uint32_t dead, uint32_t* run_start, uint32_t* run_end) {
  for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < n; k += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t key = skeys[k];
    if (key == dead) continue;
    if (k == 0 || skeys[k - 1] != key) run_start[key] = uint32_t(k);
    if (k + 1 == n || skeys[k + 1] != key) run_end[key] = uint32_t(k + 1);
  }
}

// One warp per cell: the warp stages its cell's run in shared memory 256 entries at a time
// (coalesced loads) and lane 0 adds them in order, as the reference's serial loop does.
constexpr int kSumBatch = 256;
__global__ void __launch_bounds__(256) coarse_sums(const uint32_t* run_start, const uint32_t* run_end, const float* tm,
                                                   const float* m, uint64_t cells, float* cell_tm, float* cell_m) {
  __shared__ float st[8][2][kSumBatch];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint64_t c = blockIdx.x * 8ull + w; c < cells; c += uint64_t(gridDim.x) * 8) {
    const uint32_t s0 = run_start[c], e0 = run_end[c];
    float a = 0.0f, b = 0.0f;
    for (uint32_t base = s0; base < e0; base += kSumBatch) {
      const uint32_t cnt = min(uint32_t(kSumBatch), e0 - base);
      for (uint32_t t = lane; t < cnt; t += 32) {
        st[w][0][t] = tm[base + t];
        st[w][1][t] = m[base + t];
      }
      __syncwarp();
      if (lane == 0)
        for (uint32_t t = 0; t < cnt; ++t) {
          a = __fadd_rn(a, st[w][0][t]);
          b = __fadd_rn(b, st[w][1][t]);
        }
      __syncwarp();
    }
    if (lane == 0) {
      cell_tm[c] = a;
      cell_m[c] = b;
    }
  }
}

// relaxation toward the injected temperature (simulation.rs:914-923)
__global__ void coarse_blend(const float* coarse, const float* cell_tm, const float* cell_m, uint64_t cells, float blend,
                             float* blended) {
  for (uint64_t c = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; c < cells; c += uint64_t(gridDim.x) * blockDim.x) {
    float t = coarse[c];
    if (cell_m[c] > 1e-6f) t = __fadd_rn(t, __fmul_rn(__fsub_rn(__fdiv_rn(cell_tm[c], cell_m[c]), t), blend));
    blended[c] = t;
  }
}

// one FTCS step over the 6 neighbours, neighbours summed in the reference's order (:929-964)
__global__ void coarse_diffuse(const float* f, uint32_t cn, float coef, float* out) {
  const uint64_t n = cn, nn = n * n, cells = nn * n;
  for (uint64_t g = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; g < cells; g += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t i = g % n, j = (g / n) % n, k = g / nn;
    float lap = 0.0f;
    int count = 0;
    if (i > 0) lap = __fadd_rn(lap, f[g - 1]), ++count;
    if (i + 1 < n) lap = __fadd_rn(lap, f[g + 1]), ++count;
    if (j > 0) lap = __fadd_rn(lap, f[g - n]), ++count;
    if (j + 1 < n) lap = __fadd_rn(lap, f[g + n]), ++count;
    if (k > 0) lap = __fadd_rn(lap, f[g - nn]), ++count;
    if (k + 1 < n) lap = __fadd_rn(lap, f[g + nn]), ++count;
    float t = f[g];
    if (count > 0) {
      const float avg = __fdiv_rn(lap, float(count));
      t = __fadd_rn(t, __fmul_rn(__fmul_rn(coef, __fsub_rn(avg, t)), float(count)));
    }
    out[g] = t;
  }
}

// MpssPhase (mpss.rs:67-75): Solid 0, Liquid 1, Gas 2, Plasma 3, Granular 4, Crystal 5, Amorphous 6.
// One hop of apply_phase_transitions' table (mpss.rs:512-524): the arms in order, a failing guard
// falling through to the next arm.
__device__ __forceinline__ uint8_t phase_hop(uint16_t m, uint8_t cur, float t) {
  if (m == 1 && cur == 0 && t >= 273.0f) return 1;
  if (m == 1 && cur == 1 && t >= 373.0f) return 2;
  if (m == 1 && cur == 2 && t < 373.0f) return 1;
  if (m == 1 && cur == 1 && t < 273.0f) return 0;
  if (m == 3 && cur == 0 && t >= 1811.0f) return 1;
  if (m == 3 && cur == 1 && t >= 3134.0f) return 2;
  if (m == 3 && cur == 2 && t < 3134.0f) return 1;
  if (m == 3 && cur == 1 && t < 1811.0f) return 0;
  if (m == 0 && cur == 0 && t >= 500.0f) return 2;
  if (m == 2 && cur == 0 && t >= 1923.0f) return 2;
  return cur;
}

// MpssBuffer housekeeping after the substep (ae_engine/src/lib.rs:347-358): per active particle,
// reflecting world bounds (mpss.rs:449-476), temperature clamp (:479-497), phase transitions with
// up to 3 hops (:500-548), in that order; passes selects them (1, 2, 4).  The loop bounds are
// warp-uniform so the transition count is a warp ballot.
__global__ void housekeeping_kernel(float* pos, float* vel, float* temp, uint8_t* phase, const uint16_t* mat,
                                    const uint8_t* active, uint64_t n, float x0, float y0, float z0, float x1, float y1,
                                    float z1, float tmin, float tmax, uint32_t passes, uint32_t* transitions) {
  const float lo[3] = {x0, y0, z0}, hi[3] = {x1, y1, z1};
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t base = uint64_t(blockIdx.x) * blockDim.x; base < n; base += stride) {
    const uint64_t i = base + threadIdx.x;
    bool changed = false;
    if (i < n && (!active || active[i])) {
      if (passes & 1u) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float p = pos[3 * i + d];
          if (p < lo[d]) {
            pos[3 * i + d] = lo[d];
            const float v = vel[3 * i + d];
            if (v < 0.0f) vel[3 * i + d] = __fmul_rn(-v, 0.5f);
          } else if (p > hi[d]) {
            pos[3 * i + d] = hi[d];
            const float v = vel[3 * i + d];
            if (v > 0.0f) vel[3 * i + d] = __fmul_rn(-v, 0.5f);
          }
        }
      }
      if (passes & 2u) {
        const float t = temp[i];
        if (t > tmax)
          temp[i] = tmax;
        else if (t < tmin)
          temp[i] = tmin;
      }
      if (passes & 4u) {
        const float t = temp[i];
        const uint16_t m = mat[i];
        const uint8_t cur = phase[i];
        uint8_t next = cur;
        for (int hop = 0; hop < 3; ++hop) {
          const uint8_t h = phase_hop(m, next, t);
          if (h == next) break;
          next = h;
        }
        if (next != cur) {
          phase[i] = next;
          changed = true;
        }
      }
    }
    const uint32_t c = __popc(__ballot_sync(0xffffffffu, changed));
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(transitions, c);
  }
}

inline unsigned grid_for(uint64_t n, int threads) {
  const uint64_t b = (n + threads - 1) / threads;
  return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(b, 148ull * 16)));
}

int bits_for(uint64_t v) {  // bits needed to hold values 0..v
  int b = 1;
  while (b < 32 && (uint64_t(1) << b) <= v) ++b;
  return b;
}

}  // namespace

#define LOD_TRY(x)                          \
  do {                                      \
    cudaError_t e_ = (x);                   \
    if (e_ != cudaSuccess) return e_;       \
  } while (0)

LodWork::~LodWork() {
  void* ps[] = {tile_counts_, tile_offs_, totals_, near_tmp_, near_key_, keep_, tm_, m_, cell_a_, cell_b_, field_tmp_,
                run_start_, run_end_};
  for (void* p : ps)
    if (p) cudaFree(p);
  sort_scratch_free(sort_);
}

cudaError_t LodWork::grow(uint64_t count, uint64_t cells) {
  if (count > cap_ || !totals_) {
    const uint64_t cap = std::max<uint64_t>(count, std::max<uint64_t>(cap_ * 2, 4096));
    void* ps[] = {tile_counts_, tile_offs_, near_tmp_, near_key_, keep_, tm_, m_};
    for (void* p : ps)
      if (p) cudaFree(p);
    tile_counts_ = tile_offs_ = near_key_ = nullptr;
    near_tmp_ = nullptr;
    keep_ = nullptr;
    tm_ = m_ = nullptr;
    cap_ = 0;
    const uint64_t tiles = (cap + kPTile - 1) / kPTile;
    LOD_TRY(cudaMalloc(&tile_counts_, sizeof(uint32_t) * 3 * tiles));
    LOD_TRY(cudaMalloc(&tile_offs_, sizeof(uint32_t) * 3 * tiles));
    if (!totals_) LOD_TRY(cudaMalloc(&totals_, sizeof(uint32_t) * 4));
    LOD_TRY(cudaMalloc(&near_tmp_, sizeof(uint64_t) * cap));
    LOD_TRY(cudaMalloc(&near_key_, sizeof(uint32_t) * cap));
    LOD_TRY(cudaMalloc(&keep_, cap));
    LOD_TRY(cudaMalloc(&tm_, sizeof(float) * cap));
    LOD_TRY(cudaMalloc(&m_, sizeof(float) * cap));
    LOD_TRY(sort_scratch_alloc(sort_, cap));
    cap_ = cap;
  }
  if (cells > cells_cap_) {
    void* ps[] = {cell_a_, cell_b_, field_tmp_, run_start_, run_end_};
    for (void* p : ps)
      if (p) cudaFree(p);
    cell_a_ = cell_b_ = field_tmp_ = nullptr;
    run_start_ = run_end_ = nullptr;
    cells_cap_ = 0;
    LOD_TRY(cudaMalloc(&cell_a_, sizeof(float) * cells));
    LOD_TRY(cudaMalloc(&cell_b_, sizeof(float) * cells));
    LOD_TRY(cudaMalloc(&field_tmp_, sizeof(float) * cells));
    LOD_TRY(cudaMalloc(&run_start_, sizeof(uint32_t) * cells));
    LOD_TRY(cudaMalloc(&run_end_, sizeof(uint32_t) * cells));
    cells_cap_ = cells;
  }
  return cudaSuccess;
}

cudaError_t LodWork::classify(const float* pos, const uint8_t* active, uint64_t count, const float player[3],
                              float near_dist, float mid_dist, uint64_t max_near, uint64_t* near_out, uint64_t* mid_out,
                              uint64_t* far_out, uint64_t counts[3], cudaStream_t s) {
  counts[0] = counts[1] = counts[2] = 0;
  if (count == 0) return cudaSuccess;
  LOD_TRY(grow(count, 0));
  const uint32_t tiles = uint32_t((count + kPTile - 1) / kPTile);
  // squared distances as the reference computes them (simulation.rs:484-485)
  const PosClass pc{pos, active, player[0], player[1], player[2], near_dist * near_dist, mid_dist * mid_dist};
  part_count<PosClass><<<tiles, kPT, 0, s>>>(pc, count, tile_counts_, tiles);
  part_scan<<<1, 1024, 0, s>>>(tile_counts_, tile_offs_, tiles, totals_);
  part_scatter<PosClass><<<tiles, kPT, 0, s>>>(pc, count, tile_offs_, tiles, near_tmp_,
                                               reinterpret_cast<float*>(near_key_), mid_out, uint64_t(0), far_out);
  LOD_TRY(cudaGetLastError());
  uint32_t tot[4] = {0, 0, 0, 0};
  LOD_TRY(cudaMemcpyAsync(tot, totals_, sizeof(tot), cudaMemcpyDeviceToHost, s));
  LOD_TRY(cudaStreamSynchronize(s));
  const uint64_t n_near = tot[0], n_mid = tot[1], n_far = tot[2];
  if (n_near <= max_near) {
    if (n_near) LOD_TRY(cudaMemcpyAsync(near_out, near_tmp_, sizeof(uint64_t) * n_near, cudaMemcpyDeviceToDevice, s));
    counts[0] = n_near;
    counts[1] = n_mid;
    counts[2] = n_far;
    return cudaSuccess;
  }
  // cap (simulation.rs:519-530): the max_near smallest squared distances stay near, ties by index
  if (max_near) {
    const size_t sm = n_near <= kSelectSmemKeys ? sizeof(uint32_t) * n_near : 0;
    if (!select_smem_set_) {
      LOD_TRY(cudaFuncSetAttribute(select_keep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(sizeof(uint32_t) * kSelectSmemKeys)));
      select_smem_set_ = true;
    }
    select_keep<<<1, 1024, sm, s>>>(near_key_, uint32_t(n_near), uint32_t(max_near), keep_);
  }
  else
    LOD_TRY(cudaMemsetAsync(keep_, 0, n_near, s));
  const uint32_t tiles2 = uint32_t((n_near + kPTile - 1) / kPTile);
  const KeepClass kc{near_tmp_, keep_};
  part_count<KeepClass><<<tiles2, kPT, 0, s>>>(kc, n_near, tile_counts_, tiles2);
  part_scan<<<1, 1024, 0, s>>>(tile_counts_, tile_offs_, tiles2, totals_);
  part_scatter<KeepClass><<<tiles2, kPT, 0, s>>>(kc, n_near, tile_offs_, tiles2, near_out, static_cast<float*>(nullptr),
                                                 mid_out, n_mid, static_cast<uint64_t*>(nullptr));
  LOD_TRY(cudaGetLastError());
  counts[0] = max_near;
  counts[1] = n_mid + (n_near - max_near);
  counts[2] = n_far;
  return cudaSuccess;
}

cudaError_t LodWork::housekeeping(float* pos, float* vel, float* temp, uint8_t* phase, const uint16_t* material,
                                  const uint8_t* active, uint64_t n, const float bmin[3], const float bmax[3],
                                  float min_temp, float max_temp, uint32_t passes, uint32_t* transitions,
                                  cudaStream_t s) {
  *transitions = 0;
  if (n == 0) return cudaSuccess;
  LOD_TRY(grow(1, 0));
  LOD_TRY(cudaMemsetAsync(totals_ + 3, 0, sizeof(uint32_t), s));
  housekeeping_kernel<<<grid_for(n, 256), 256, 0, s>>>(pos, vel, temp, phase, material, active, n, bmin[0], bmin[1],
                                                      bmin[2], bmax[0], bmax[1], bmax[2], min_temp, max_temp, passes,
                                                      totals_ + 3);
  LOD_TRY(cudaGetLastError());
  LOD_TRY(cudaMemcpyAsync(transitions, totals_ + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  return cudaStreamSynchronize(s);
}

cudaError_t LodWork::far_field(float* pos, float* vel, float* temp, const uint64_t* far_idx, uint64_t n,
                               const float* coarse, uint32_t cn, float cdx, const float origin[3], float far_dt,
                               cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  far_field_kernel<<<grid_for(n, 256), 256, 0, s>>>(pos, vel, temp, far_idx, n, coarse, cn, cdx, origin[0], origin[1],
                                                   origin[2], far_dt);
  return cudaGetLastError();
}

cudaError_t LodWork::coarse_field(const float* pos, const float* mass, const float* temp, const uint8_t* active,
                                  const uint64_t* near_idx, uint64_t n, float* coarse, uint32_t cn, float cdx,
                                  const float origin[3], float dt, cudaStream_t s) {
  const uint64_t cells = uint64_t(cn) * cn * cn;
  if (cells == 0) return cudaSuccess;
  LOD_TRY(grow(std::max<uint64_t>(n, 1), cells));
  if (n == 0) {  // no particles: the injection adds nothing
    LOD_TRY(cudaMemsetAsync(cell_a_, 0, sizeof(float) * cells, s));
    LOD_TRY(cudaMemsetAsync(cell_b_, 0, sizeof(float) * cells, s));
  }
  if (n > 0) {
    const uint32_t dead = uint32_t(cells);
    const float inv_dx = 1.0f / cdx;
    coarse_keys<<<grid_for(n, 256), 256, 0, s>>>(pos, active, near_idx, n, cn, inv_dx, origin[0], origin[1], origin[2],
                                                dead, near_key_);
    const uint32_t *sorted = nullptr, *perm = nullptr;
    radix_sort_pairs(near_key_, n, bits_for(cells), sort_, s, &sorted, &perm);
    coarse_gather<<<grid_for(n, 256), 256, 0, s>>>(mass, temp, near_idx, perm, n, tm_, m_);
    LOD_TRY(cudaMemsetAsync(run_start_, 0, sizeof(uint32_t) * cells, s));
    LOD_TRY(cudaMemsetAsync(run_end_, 0, sizeof(uint32_t) * cells, s));
    coarse_runs<<<grid_for(n, 256), 256, 0, s>>>(sorted, n, dead, run_start_, run_end_);
    coarse_sums<<<unsigned(std::min<uint64_t>((cells + 7) / 8, 148 * 16)), 256, 0, s>>>(run_start_, run_end_, tm_, m_,
                                                                                      cells, cell_a_, cell_b_);
  }
  const float inject_rate = 0.1f;
  const float blend = std::fmin(inject_rate * dt, 1.0f);
  const float alpha = 10.0f;
  const float coef = std::fmin(alpha * dt / (cdx * cdx), 0.16f);
  coarse_blend<<<grid_for(cells, 256), 256, 0, s>>>(coarse, cell_a_, cell_b_, cells, blend, field_tmp_);
  coarse_diffuse<<<grid_for(cells, 256), 256, 0, s>>>(field_tmp_, cn, coef, coarse);
  return cudaGetLastError();
}

}  // namespace aemp
