// ae_mpm_noalloc.cu -- the radix sort by cell key for callers that cannot allocate GPU memory.
//
// Some callers must not call cudaMalloc: an engine whose frame loop runs on device memory it
// reserved up front (an allocation there can block on the driver and stall the frame), code that
// queues work while a CUDA stream is being captured into a graph (where cudaMalloc is not
// permitted), or a host that hands every byte of HBM to its own pool.  ae_mpm_radix_sort_keys
// allocates its scratch on first use, so this file offers the same sort with its scratch in a
// fixed file-scope device array instead.  The caller still provides the input keys and the output
// buffers (device memory it owns); nothing here allocates, frees, or calls an allocating library.
//
// The array below is created by the CUDA runtime when the library's module is loaded on a device,
// and every device that loads the library keeps its copy (kNoallocScratchBytes, about 9 MB) until
// the process exits.  All calls on one device share it and it keeps the last call's contents:
// what must start at zero (the per-digit totals) is cleared by each call, and two calls whose
// work overlaps on the GPU race on the array, so a caller queues them on one stream or otherwise
// orders them.
//
// The device address of the array is looked up once per device and kept for the life of the
// process.  A cudaDeviceReset after the first call unloads the module and leaves that address
// stale, so a process that resets a device must not call this entry point on it again.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/ae_mpm.h"
#include "mpm_world.cuh"
#include "radix_sort.cuh"

namespace {

constexpr uint64_t kMaxKeys = AE_MPM_NOALLOC_MAX_KEYS;
constexpr uint64_t kTiles = (kMaxKeys + aemp::kSortTile - 1) / aemp::kSortTile;
// carve-up of the scratch (32-bit words): hist | offsets | totals | keys_alt | vals_alt
constexpr uint64_t kHistWords = uint64_t(aemp::kMaxRadix) * kTiles;
constexpr uint64_t kTotalsWords = 4 * uint64_t(aemp::kMaxRadix);
constexpr uint64_t kScratchWords = 2 * kHistWords + kTotalsWords + 2 * kMaxKeys;
constexpr uint64_t kNoallocScratchBytes = kScratchWords * sizeof(uint32_t);
static_assert(kNoallocScratchBytes <= (16ull << 20), "the no-allocation scratch array stays under 16 MB per device");

static __device__ __align__(256) uint32_t g_sort_scratch[kScratchWords];

// Device address of g_sort_scratch for each device, looked up once per device with that device
// current.  In host code the symbol itself only names the array; only this address may be given
// to a kernel.
std::mutex g_mu;
uint32_t* g_scratch_addr[64] = {};

int scratch_for_current_device(uint32_t** out, std::string& why) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    why = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
    return AE_MPM_ECUDA;
  }
  if (dev < 0 || dev >= 64) {
    why = "device ordinal out of range for the scratch table";
    return AE_MPM_EINVAL;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess || !p) {
      why = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
      return AE_MPM_ECUDA;
    }
    g_scratch_addr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_scratch_addr[dev];
  return AE_MPM_OK;
}

}  // namespace

extern "C" int ae_mpm_radix_sort_keys_noalloc(ae_mpm_ctx* ctx, const uint32_t* keys_dev, uint64_t n, uint32_t key_bits,
                                              uint32_t* sorted_keys_dev, uint32_t* perm_dev, void* stream) {
  auto fail = [&](int code, const std::string& msg) {
    aemp::ctx_set_error(ctx, msg);
    return code;
  };
  if (n == 0) return AE_MPM_OK;
  if (n > kMaxKeys)
    return fail(AE_MPM_EINVAL, "ae_mpm_radix_sort_keys_noalloc: " + std::to_string(n) +
                                   " keys exceed the fixed scratch limit of " + std::to_string(kMaxKeys));
  if (!keys_dev || !sorted_keys_dev || !perm_dev || key_bits == 0 || key_bits > 32)
    return fail(AE_MPM_EINVAL, "ae_mpm_radix_sort_keys_noalloc: null buffer or key_bits outside 1..32");
  // The passes read one buffer while other blocks write the next, and with an odd pass count the
  // first pass writes straight into sorted_keys_dev: the three buffers must not overlap.
  auto overlap = [n](const void* a, const void* b) {
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    const uintptr_t len = uintptr_t(n) * sizeof(uint32_t);
    return x < y + len && y < x + len;
  };
  if (overlap(keys_dev, sorted_keys_dev) || overlap(keys_dev, perm_dev) || overlap(sorted_keys_dev, perm_dev))
    return fail(AE_MPM_EINVAL, "ae_mpm_radix_sort_keys_noalloc: keys_dev, sorted_keys_dev and perm_dev must not overlap");
  if (ctx) {
    cudaError_t e = cudaSetDevice(aemp::ctx_device(ctx));
    if (e != cudaSuccess) return fail(AE_MPM_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  }
  uint32_t* s = nullptr;
  std::string why;
  int rc = scratch_for_current_device(&s, why);
  if (rc) return fail(rc, why);
  uint32_t* hist = s;
  uint32_t* offsets = hist + kHistWords;
  uint32_t* totals = offsets + kHistWords;
  uint32_t* keys_alt = totals + kTotalsWords;
  uint32_t* vals_alt = keys_alt + kMaxKeys;
  aemp::radix_sort_pairs_into(keys_dev, n, int(key_bits), sorted_keys_dev, perm_dev, keys_alt, vals_alt, hist, offsets,
                              totals, static_cast<cudaStream_t>(stream));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(AE_MPM_ECUDA, std::string("radix sort launch: ") + cudaGetErrorString(e));
  return AE_MPM_OK;
}
