// radix_sort.cuh -- stable LSD radix sort of 32-bit cell keys with a 32-bit payload, sm_100a.
//
// The reference has no sort on its MPM path (its P2G walks particle_indices in buffer order,
// ae_particle/src/mpm_solver.rs:831, 1108); the sort is what lets P2G aggregate same-cell
// contributions.  It must be bit-exact against a stable CPU sort of the same keys: equal keys
// keep their input order.
//
// One pass per digit (<= 8 bits), three kernels per pass:
//   1. sort_hist:    per-tile digit counts (warp-aggregated with __match_any_sync), written
//                    digit-major, plus the global digit totals (one atomic per tile and digit).
//   2. sort_scan:    one block per digit: exclusive scan of that digit's per-tile counts,
//                    offset by the totals of all smaller digits.
//   3. sort_scatter: each warp ranks its 256 keys in input order (match + popc), the block
//                    turns warp counts into tile-local positions, stages keys in shared memory
//                    in sorted order and writes runs of equal digits contiguously to HBM.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace aemp {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per block
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kMaxRadix = 256;
constexpr int kSmallSortMax = 16384;  // radix_sort_pairs sorts up to this many keys in one CTA
constexpr int kCountingSortBits = 16;  // counting_sort_pairs takes keys of at most this many bits

struct SortPlan {
  int passes;
  int shift[4];
  int bits[4];
};

inline SortPlan make_sort_plan(int key_bits) {
  SortPlan p{};
  if (key_bits < 1) key_bits = 1;
  if (key_bits > 32) key_bits = 32;
  p.passes = (key_bits + 7) / 8;
  int per = (key_bits + p.passes - 1) / p.passes;
  int s = 0;
  for (int i = 0; i < p.passes; ++i) {
    int b = (key_bits - s < per) ? key_bits - s : per;
    p.shift[i] = s;
    p.bits[i] = b;
    s += b;
  }
  return p;
}

// Scratch for one sort of up to n keys (device pointers owned by the caller).
struct SortScratch {
  uint32_t* hist = nullptr;     // [kMaxRadix * tiles]
  uint32_t* offsets = nullptr;  // [kMaxRadix * tiles]
  uint32_t* totals = nullptr;   // [4 * kMaxRadix]
  uint32_t* keys_alt = nullptr; // [n]
  uint32_t* vals_a = nullptr;   // [n]
  uint32_t* vals_b = nullptr;   // [n]
  uint32_t* bins = nullptr;     // [1 << kCountingSortBits] (counting sort; allocated for n > kSmallSortMax)
  uint64_t n_cap = 0;
};

inline uint64_t sort_tiles(uint64_t n) { return (n + kSortTile - 1) / kSortTile; }

// Allocates scratch for n keys; returns cudaSuccess or the failing call's status.
// `alloc(p, bytes)` / `release(p)` default to cudaMalloc / cudaFree.
typedef cudaError_t (*SortAllocFn)(void* user, void** p, size_t bytes);
typedef void (*SortFreeFn)(void* user, void* p);
cudaError_t sort_scratch_alloc(SortScratch& s, uint64_t n, SortAllocFn alloc = nullptr, void* user = nullptr);
void sort_scratch_free(SortScratch& s, SortFreeFn release = nullptr, void* user = nullptr);

// Sorts keys[0..n) (only bits [0, key_bits) compared).  On return *perm_out points to the
// permutation (perm[i] = input index of the i-th smallest key) and *sorted_keys_out to the sorted
// keys; both live in `keys` / scratch buffers and are valid until the next sort.  `keys` is
// clobbered.  Queues 3 kernels per pass plus one memset on `stream` (one kernel when n <=
// kSmallSortMax); returns the launch count.
int radix_sort_pairs(uint32_t* keys, uint64_t n, int key_bits, SortScratch& s, cudaStream_t stream,
                     const uint32_t** sorted_keys_out, const uint32_t** perm_out);

// Groups keys[0..n) by key in one pass (key_bits <= kCountingSortBits): a histogram, one scan
// over the 2^key_bits bins and a scatter that claims places with atomics.  The keys come out
// sorted, but equal keys in no defined order (the order atomics give them), so only callers whose
// results do not depend on that order may use it.  Same outputs and lifetime rules as
// radix_sort_pairs.  n <= kSmallSortMax, wider keys or scratch without bins go to
// radix_sort_pairs (which clobbers `keys`); the counting pass itself only reads them.  Returns the
// launch count.
int counting_sort_pairs(uint32_t* keys, uint64_t n, int key_bits, SortScratch& s, cudaStream_t stream,
                        const uint32_t** sorted_keys_out, const uint32_t** perm_out);

// Same sort with every buffer supplied by the caller: keys_in is only read; the result lands in
// keys_out / vals_out; keys_alt / vals_alt (n entries each), hist and offsets (kMaxRadix *
// sort_tiles(n) entries each) and totals (4 * kMaxRadix entries) are scratch.  Clears the
// totals itself; allocates nothing.  Returns the kernel launch count.
int radix_sort_pairs_into(const uint32_t* keys_in, uint64_t n, int key_bits, uint32_t* keys_out, uint32_t* vals_out,
                          uint32_t* keys_alt, uint32_t* vals_alt, uint32_t* hist, uint32_t* offsets, uint32_t* totals,
                          cudaStream_t stream);

}  // namespace aemp
