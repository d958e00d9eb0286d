// radix_sort.cu -- stable LSD radix sort of cell keys (see radix_sort.cuh for the design).
#include "radix_sort.cuh"

namespace aemp {

namespace {

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

__global__ void __launch_bounds__(kSortThreads) sort_hist(const uint32_t* __restrict__ keys, uint64_t n, int shift,
                                                          uint32_t mask, uint32_t* __restrict__ hist,
                                                          uint32_t* __restrict__ totals, uint32_t tiles) {
  __shared__ uint32_t cnt[kMaxRadix];
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < kMaxRadix; i += kSortThreads) cnt[i] = 0;
  __syncthreads();
  const uint64_t base = uint64_t(blockIdx.x) * kSortTile;
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    uint64_t idx = base + uint64_t(k) * kSortThreads + tid;
    bool valid = idx < n;
    uint32_t d = valid ? (__ldg(keys + idx) >> shift) & mask : 0xffffffffu;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    if (valid && lane == __ffs(peers) - 1) atomicAdd(&cnt[d], uint32_t(__popc(peers)));
  }
  __syncthreads();
  for (uint32_t d = tid; d <= mask; d += kSortThreads) {
    uint32_t c = cnt[d];
    hist[uint64_t(d) * tiles + blockIdx.x] = c;
    if (c) atomicAdd(&totals[d], c);
  }
}

constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads) sort_scan(const uint32_t* __restrict__ hist,
                                                          const uint32_t* __restrict__ totals,
                                                          uint32_t* __restrict__ offsets, uint32_t tiles) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t d = blockIdx.x;
  if (w == 0) {
    uint32_t s = 0;
    for (uint32_t i = lane; i < d; i += 32) s += totals[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) carry = s;
  }
  __syncthreads();
  const uint32_t* row = hist + uint64_t(d) * tiles;
  uint32_t* orow = offsets + uint64_t(d) * tiles;
  for (uint32_t start = 0; start < tiles; start += kScanThreads) {
    uint32_t i = start + tid;
    uint32_t x = (i < tiles) ? row[i] : 0u;
    uint32_t incl = warp_incl_scan(x, lane);
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    if (w == 0) {
      uint32_t ws = warp_sums[lane];
      uint32_t wi = warp_incl_scan(ws, lane);
      warp_sums[lane] = wi - ws;
    }
    __syncthreads();
    uint32_t c = carry;
    if (i < tiles) orow[i] = c + warp_sums[w] + incl - x;
    __syncthreads();
    if (tid == kScanThreads - 1) carry = c + warp_sums[w] + incl;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kSortThreads) sort_scatter(const uint32_t* __restrict__ keys_in,
                                                             const uint32_t* __restrict__ vals_in,
                                                             uint32_t* __restrict__ keys_out,
                                                             uint32_t* __restrict__ vals_out, uint64_t n, int shift,
                                                             uint32_t mask, const uint32_t* __restrict__ offsets,
                                                             uint32_t tiles) {
  __shared__ uint32_t wcnt[kSortWarps][kMaxRadix];
  __shared__ uint32_t tstart[kMaxRadix];
  __shared__ uint32_t goff[kMaxRadix];
  __shared__ uint32_t wsum[kSortWarps];
  __shared__ uint32_t skeys[kSortTile];
  __shared__ uint32_t svals[kSortTile];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int i = tid; i < kSortWarps * kMaxRadix; i += kSortThreads) (&wcnt[0][0])[i] = 0;
  __syncthreads();
  const uint64_t base = uint64_t(blockIdx.x) * kSortTile;
  uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    uint64_t idx = base + uint64_t(w) * (32 * kSortItems) + uint64_t(r) * 32 + lane;
    bool valid = idx < n;
    key[r] = valid ? __ldg(keys_in + idx) : 0xffffffffu;
    val[r] = valid ? (vals_in ? __ldg(vals_in + idx) : uint32_t(idx)) : 0u;
    uint32_t d = valid ? (key[r] >> shift) & mask : 0xffffffffu;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t cur = valid ? wcnt[w][d] : 0u;
    rank[r] = cur + __popc(peers & lt);
    __syncwarp();
    if (valid && lane == __ffs(peers) - 1) wcnt[w][d] = cur + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // per digit: exclusive prefix over warps and the tile total
  uint32_t total = 0;
  if (uint32_t(tid) <= mask) {
#pragma unroll
    for (int ww = 0; ww < kSortWarps; ++ww) {
      uint32_t c = wcnt[ww][tid];
      wcnt[ww][tid] = total;
      total += c;
    }
    goff[tid] = offsets[uint64_t(tid) * tiles + blockIdx.x];
  }
  // exclusive scan of the tile totals over digits (one digit per thread, kMaxRadix == threads)
  uint32_t incl = warp_incl_scan(total, lane);
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    uint32_t ws = (lane < kSortWarps) ? wsum[lane] : 0u;
    uint32_t wi = warp_incl_scan(ws, lane);
    if (lane < kSortWarps) wsum[lane] = wi - ws;
  }
  __syncthreads();
  tstart[tid] = wsum[w] + incl - total;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    uint64_t idx = base + uint64_t(w) * (32 * kSortItems) + uint64_t(r) * 32 + lane;
    if (idx < n) {
      uint32_t d = (key[r] >> shift) & mask;
      uint32_t pos = tstart[d] + wcnt[w][d] + rank[r];
      skeys[pos] = key[r];
      svals[pos] = val[r];
    }
  }
  __syncthreads();
  const uint32_t tile_n = uint32_t((n - base) < uint64_t(kSortTile) ? (n - base) : uint64_t(kSortTile));
  for (uint32_t i = tid; i < tile_n; i += kSortThreads) {
    uint32_t k = skeys[i];
    uint32_t d = (k >> shift) & mask;
    uint32_t o = goff[d] + (i - tstart[d]);
    keys_out[o] = k;
    vals_out[o] = svals[i];
  }
}

// ---- short lists: the whole sort in one CTA ----------------------------------------------------
// For up to kSmallSortMax keys the three kernels per pass are launch-bound (the engine's near-field
// call sorts 16 384 keys).  One CTA of 1024 threads keeps keys and 16-bit indices in shared memory
// and runs every pass there: each warp ranks its contiguous run of keys row by row (match on the
// digit, as sort_scatter does), a per-digit prefix over warps and a scan over digits give each
// key its place, and the keys move between two shared buffers.  Stable, as the multi-kernel path.
constexpr int kSmallThreads = 1024;
constexpr int kSmallWarps = kSmallThreads / 32;
constexpr int kSmallRows = kSmallSortMax / kSmallThreads;  // rows of 32 keys per warp at most

size_t small_sort_smem() {
  return sizeof(uint32_t) * 2 * kSmallSortMax + sizeof(uint16_t) * 2 * kSmallSortMax +
         sizeof(uint16_t) * kSmallWarps * kMaxRadix + sizeof(uint32_t) * (kMaxRadix + kSmallWarps);
}

__global__ void __launch_bounds__(kSmallThreads, 1) sort_small(const uint32_t* __restrict__ keys_in, uint32_t n,
                                                              SortPlan plan, uint32_t* __restrict__ keys_out,
                                                              uint32_t* __restrict__ perm_out) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* kbuf = reinterpret_cast<uint32_t*>(smem);                // [2][kSmallSortMax]
  uint16_t* vbuf = reinterpret_cast<uint16_t*>(kbuf + 2 * kSmallSortMax);  // [2][kSmallSortMax]
  uint16_t* wcnt = vbuf + 2 * kSmallSortMax;                         // [kSmallWarps][kMaxRadix]
  uint32_t* dstart = reinterpret_cast<uint32_t*>(wcnt + kSmallWarps * kMaxRadix);  // [kMaxRadix]
  uint32_t* wsum = dstart + kMaxRadix;                               // [kSmallWarps]
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t lt = lanemask_lt();
  // each warp owns `seg` consecutive keys, `rows` rows of 32
  const uint32_t rows = (n + 32u * kSmallWarps - 1) / (32u * kSmallWarps);
  const uint32_t seg = rows * 32u;
  for (uint32_t i = tid; i < n; i += kSmallThreads) {
    kbuf[i] = __ldg(keys_in + i);
    vbuf[i] = uint16_t(i);
  }
  int cur = 0;
  for (int ps = 0; ps < plan.passes; ++ps) {
    const int shift = plan.shift[ps];
    const uint32_t mask = (1u << plan.bits[ps]) - 1u;
    const uint32_t* kin = kbuf + cur * kSmallSortMax;
    const uint16_t* vin = vbuf + cur * kSmallSortMax;
    uint32_t* kout = kbuf + (cur ^ 1) * kSmallSortMax;
    uint16_t* vout = vbuf + (cur ^ 1) * kSmallSortMax;
    for (int i = tid; i < kSmallWarps * kMaxRadix; i += kSmallThreads) wcnt[i] = 0;
    __syncthreads();
    uint32_t rank[kSmallRows];
#pragma unroll
    for (int r = 0; r < kSmallRows; ++r) {
      rank[r] = 0;
      if (uint32_t(r) >= rows) continue;  // warp-uniform
      const uint32_t idx = uint32_t(w) * seg + uint32_t(r) * 32u + uint32_t(lane);
      const bool valid = idx < n;
      const uint32_t d = valid ? (kin[idx] >> shift) & mask : 0xffffffffu;
      const uint32_t peers = __match_any_sync(0xffffffffu, d);
      const uint32_t c = valid ? wcnt[w * kMaxRadix + d] : 0u;
      rank[r] = c + __popc(peers & lt);
      __syncwarp();
      if (valid && lane == __ffs(peers) - 1) wcnt[w * kMaxRadix + d] = uint16_t(c + __popc(peers));
      __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix over warps, and the digit's total
    uint32_t total = 0;
    if (uint32_t(tid) < uint32_t(kMaxRadix)) {
      for (int ww = 0; ww < kSmallWarps; ++ww) {
        const uint32_t c = wcnt[ww * kMaxRadix + tid];
        wcnt[ww * kMaxRadix + tid] = uint16_t(total);
        total += c;
      }
    }
    // exclusive scan of the digit totals (digits 0..255 live in warps 0..7)
    const uint32_t incl = warp_incl_scan(total, lane);
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      const uint32_t ws = lane < kSmallWarps ? wsum[lane] : 0u;
      const uint32_t wi = warp_incl_scan(ws, lane);
      if (lane < kSmallWarps) wsum[lane] = wi - ws;
    }
    __syncthreads();
    if (uint32_t(tid) < uint32_t(kMaxRadix)) dstart[tid] = wsum[w] + incl - total;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSmallRows; ++r) {
      if (uint32_t(r) >= rows) continue;
      const uint32_t idx = uint32_t(w) * seg + uint32_t(r) * 32u + uint32_t(lane);
      if (idx < n) {
        const uint32_t k = kin[idx];
        const uint32_t d = (k >> shift) & mask;
        const uint32_t pos = dstart[d] + wcnt[w * kMaxRadix + d] + rank[r];
        kout[pos] = k;
        vout[pos] = vin[idx];
      }
    }
    __syncthreads();
    cur ^= 1;
  }
  const uint32_t* kf = kbuf + cur * kSmallSortMax;
  const uint16_t* vf = vbuf + cur * kSmallSortMax;
  for (uint32_t i = tid; i < n; i += kSmallThreads) {
    keys_out[i] = kf[i];
    perm_out[i] = vf[i];
  }
}

// ---- one-pass counting sort (keys of at most kCountingSortBits bits) ------------------------------
constexpr int kCountThreads = 256;

__global__ void __launch_bounds__(kCountThreads) count_hist(const uint32_t* __restrict__ keys, uint64_t n, uint32_t mask,
                                                            uint32_t* __restrict__ bins) {
  const int lane = threadIdx.x & 31;
  for (uint64_t base = uint64_t(blockIdx.x) * kCountThreads; base < n; base += uint64_t(gridDim.x) * kCountThreads) {
    const uint64_t i = base + threadIdx.x;
    const bool valid = i < n;
    const uint32_t k = valid ? (__ldg(keys + i) & mask) : 0xffffffffu;
    const uint32_t peers = __match_any_sync(0xffffffffu, k);  // one atomic per key per warp
    if (valid && lane == __ffs(peers) - 1) atomicAdd(bins + k, uint32_t(__popc(peers)));
  }
}

// exclusive scan of the bins within each segment of 1024 (one CTA per segment, one bin per
// thread, coalesced), in place; seg_total[b] = the sum of segment b.  The scatter adds the
// segment's offset, the exclusive scan of seg_total, which each of its CTAs forms itself.
constexpr int kSegBins = 1024;
constexpr int kMaxSegs = (1 << kCountingSortBits) / kSegBins;

__global__ void __launch_bounds__(kSegBins) count_scan(uint32_t* __restrict__ bins, uint32_t nb,
                                                       uint32_t* __restrict__ seg_total) {
  __shared__ uint32_t wsum[32];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const uint32_t i = blockIdx.x * kSegBins + tid;
  const uint32_t x = i < nb ? bins[i] : 0u;
  const uint32_t incl = warp_incl_scan(x, lane);
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    const uint32_t ws = wsum[lane];
    wsum[lane] = warp_incl_scan(ws, lane) - ws;
  }
  __syncthreads();
  if (i < nb) bins[i] = wsum[w] + incl - x;
  if (tid == kSegBins - 1) seg_total[blockIdx.x] = wsum[w] + incl;
}

__global__ void __launch_bounds__(kCountThreads) count_scatter(const uint32_t* __restrict__ keys, uint64_t n,
                                                               uint32_t mask, uint32_t* __restrict__ bins,
                                                               const uint32_t* __restrict__ seg_total,
                                                               uint32_t n_segs, uint32_t* __restrict__ keys_out,
                                                               uint32_t* __restrict__ perm_out) {
  __shared__ uint32_t seg_off[kMaxSegs];
  const int lane = threadIdx.x & 31;
  const uint32_t lt = lanemask_lt();
  if (threadIdx.x < 32) {  // exclusive scan of the segment totals, two per lane
    const uint32_t a = 2u * lane < n_segs ? seg_total[2 * lane] : 0u;
    const uint32_t b = 2u * lane + 1u < n_segs ? seg_total[2 * lane + 1] : 0u;
    const uint32_t incl = warp_incl_scan(a + b, lane);
    seg_off[2 * lane] = incl - a - b;
    seg_off[2 * lane + 1] = incl - b;
  }
  __syncthreads();
  for (uint64_t base = uint64_t(blockIdx.x) * kCountThreads; base < n; base += uint64_t(gridDim.x) * kCountThreads) {
    const uint64_t i = base + threadIdx.x;
    const bool valid = i < n;
    const uint32_t k = valid ? __ldg(keys + i) : 0xffffffffu;
    const uint32_t d = valid ? (k & mask) : 0xffffffffu;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    uint32_t pos = 0;
    if (valid && lane == leader) pos = atomicAdd(bins + d, uint32_t(__popc(peers))) + seg_off[d / kSegBins];
    pos = __shfl_sync(0xffffffffu, pos, leader) + __popc(peers & lt);
    if (valid) {
      keys_out[pos] = k;
      perm_out[pos] = uint32_t(i);
    }
  }
}

}  // namespace

cudaError_t sort_scratch_alloc(SortScratch& s, uint64_t n, SortAllocFn alloc, void* user) {
  sort_scratch_free(s);
  auto A = [&](uint32_t** p, size_t bytes) -> cudaError_t {
    void* q = nullptr;
    cudaError_t e = alloc ? alloc(user, &q, bytes) : cudaMalloc(&q, bytes);
    *p = static_cast<uint32_t*>(q);
    return e;
  };
  const uint64_t tiles = sort_tiles(n > 0 ? n : 1), m = n > 0 ? n : 1;
  cudaError_t e;
  if ((e = A(&s.hist, sizeof(uint32_t) * kMaxRadix * tiles)) != cudaSuccess) return e;
  if ((e = A(&s.offsets, sizeof(uint32_t) * kMaxRadix * tiles)) != cudaSuccess) return e;
  if ((e = A(&s.totals, sizeof(uint32_t) * 4 * kMaxRadix)) != cudaSuccess) return e;
  if ((e = A(&s.keys_alt, sizeof(uint32_t) * m)) != cudaSuccess) return e;
  if ((e = A(&s.vals_a, sizeof(uint32_t) * m)) != cudaSuccess) return e;
  if ((e = A(&s.vals_b, sizeof(uint32_t) * m)) != cudaSuccess) return e;
  if (n > uint64_t(kSmallSortMax) && (e = A(&s.bins, sizeof(uint32_t) << kCountingSortBits)) != cudaSuccess) return e;
  s.n_cap = n;
  return cudaSuccess;
}

void sort_scratch_free(SortScratch& s, SortFreeFn release, void* user) {
  uint32_t* ps[7] = {s.hist, s.offsets, s.totals, s.keys_alt, s.vals_a, s.vals_b, s.bins};
  for (uint32_t* p : ps)
    if (p) {
      if (release)
        release(user, p);
      else
        cudaFree(p);
    }
  s = SortScratch{};
}

int radix_sort_pairs(uint32_t* keys, uint64_t n, int key_bits, SortScratch& s, cudaStream_t stream,
                     const uint32_t** sorted_keys_out, const uint32_t** perm_out) {
  if (n == 0) {
    *sorted_keys_out = keys;
    *perm_out = s.vals_a;
    return 0;
  }
  const SortPlan p = make_sort_plan(key_bits);
  if (n <= uint64_t(kSmallSortMax)) {
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
      cudaFuncSetAttribute(sort_small, cudaFuncAttributeMaxDynamicSharedMemorySize, int(small_sort_smem()));
      attr_set[dev] = true;
    }
    sort_small<<<1, kSmallThreads, small_sort_smem(), stream>>>(keys, uint32_t(n), p, s.keys_alt, s.vals_a);
    *sorted_keys_out = s.keys_alt;
    *perm_out = s.vals_a;
    return 1;
  }
  const uint32_t tiles = uint32_t(sort_tiles(n));
  cudaMemsetAsync(s.totals, 0, sizeof(uint32_t) * 4 * kMaxRadix, stream);
  uint32_t* kin = keys;
  uint32_t* kout = s.keys_alt;
  const uint32_t* vin = nullptr;
  uint32_t* vout = s.vals_a;
  int launches = 0;
  for (int ps = 0; ps < p.passes; ++ps) {
    const uint32_t mask = (p.bits[ps] >= 32) ? 0xffffffffu : ((1u << p.bits[ps]) - 1u);
    uint32_t* tot = s.totals + ps * kMaxRadix;
    sort_hist<<<tiles, kSortThreads, 0, stream>>>(kin, n, p.shift[ps], mask, s.hist, tot, tiles);
    sort_scan<<<mask + 1, kScanThreads, 0, stream>>>(s.hist, tot, s.offsets, tiles);
    sort_scatter<<<tiles, kSortThreads, 0, stream>>>(kin, vin, kout, vout, n, p.shift[ps], mask, s.offsets, tiles);
    launches += 3;
    uint32_t* nk = (kout == s.keys_alt) ? keys : s.keys_alt;
    kin = kout;
    kout = nk;
    vin = vout;
    vout = (vout == s.vals_a) ? s.vals_b : s.vals_a;
  }
  *sorted_keys_out = kin;
  *perm_out = vin;
  return launches;
}

}  // namespace aemp

namespace aemp {

int radix_sort_pairs_into(const uint32_t* keys_in, uint64_t n, int key_bits, uint32_t* keys_out, uint32_t* vals_out,
                          uint32_t* keys_alt, uint32_t* vals_alt, uint32_t* hist, uint32_t* offsets, uint32_t* totals,
                          cudaStream_t stream) {
  if (n == 0) return 0;
  const SortPlan p = make_sort_plan(key_bits);
  const uint32_t tiles = uint32_t(sort_tiles(n));
  cudaMemsetAsync(totals, 0, sizeof(uint32_t) * 4 * kMaxRadix, stream);
  const uint32_t* kin = keys_in;
  const uint32_t* vin = nullptr;
  int launches = 0;
  for (int ps = 0; ps < p.passes; ++ps) {
    // the last pass writes the caller's output; earlier passes alternate so that holds
    const bool to_out = ((p.passes - 1 - ps) % 2) == 0;
    uint32_t* kout = to_out ? keys_out : keys_alt;
    uint32_t* vout = to_out ? vals_out : vals_alt;
    const uint32_t mask = (1u << p.bits[ps]) - 1u;
    uint32_t* tot = totals + ps * kMaxRadix;
    sort_hist<<<tiles, kSortThreads, 0, stream>>>(kin, n, p.shift[ps], mask, hist, tot, tiles);
    sort_scan<<<mask + 1, kScanThreads, 0, stream>>>(hist, tot, offsets, tiles);
    sort_scatter<<<tiles, kSortThreads, 0, stream>>>(kin, vin, kout, vout, n, p.shift[ps], mask, offsets, tiles);
    launches += 3;
    kin = kout;
    vin = vout;
  }
  return launches;
}

}  // namespace aemp

namespace aemp {

int counting_sort_pairs(uint32_t* keys, uint64_t n, int key_bits, SortScratch& s, cudaStream_t stream,
                        const uint32_t** sorted_keys_out, const uint32_t** perm_out) {
  *sorted_keys_out = s.keys_alt;
  *perm_out = s.vals_a;
  if (n == 0) return 0;
  // short lists sort in one CTA (stable and cheaper); wide keys need the radix passes
  if (n <= uint64_t(kSmallSortMax) || key_bits > kCountingSortBits || !s.bins)
    return radix_sort_pairs(keys, n, key_bits, s, stream, sorted_keys_out, perm_out);
  if (key_bits < 1) key_bits = 1;
  const uint32_t nb = 1u << key_bits, mask = nb - 1u;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t want = (n + kCountThreads - 1) / kCountThreads;
  const unsigned grid = unsigned(want < uint64_t(sms) * 8 ? want : uint64_t(sms) * 8);
  const uint32_t n_segs = (nb + kSegBins - 1) / kSegBins;  // <= kMaxSegs; totals has 4 * kMaxRadix entries
  cudaMemsetAsync(s.bins, 0, sizeof(uint32_t) * nb, stream);
  count_hist<<<grid, kCountThreads, 0, stream>>>(keys, n, mask, s.bins);
  count_scan<<<n_segs, kSegBins, 0, stream>>>(s.bins, nb, s.totals);
  count_scatter<<<grid, kCountThreads, 0, stream>>>(keys, n, mask, s.bins, s.totals, n_segs, s.keys_alt, s.vals_a);
  return 3;
}

}  // namespace aemp
