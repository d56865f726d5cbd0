// bb_sort_static.cu -- bb_radix_sort_pairs_static: the same onesweep radix sort as
// bb_radix_sort_pairs, with its scratch in a fixed file-scope device array instead of a
// cudaMalloc'd block, so that a call allocates nothing (for callers that must not allocate
// device memory on their path, e.g. a real-time loop with a fixed memory budget).
//
// Scratch: BB_SORT_STATIC_MAX_KEYS keys at most.  Its address is looked up once per device
// with cudaGetSymbolAddress while that device is current; that first call loads the module's
// globals and so belongs before any stream capture.  All calls on one device share the array,
// so calls must not overlap in time (issue them on one stream, or order them with events).
#include <mutex>

#include "bb_common.cuh"
#include "bb_kernels.cuh"

namespace {
constexpr uint32_t kTile = BB_SORT_TILE;  // keys per onesweep tile
constexpr uint32_t kMaxKeys = BB_SORT_STATIC_MAX_KEYS;
constexpr int kMaxPasses = 4;
constexpr size_t kCounterBytes = (sizeof(DevCounters) + 255) / 256 * 256;
// same layout as bb_sort_carve for n = kMaxKeys, 4 passes: counters | 2x8x256 histogram |
// 16 tile counters | per-pass tile status | temporary keys | temporary values
constexpr size_t kStaticBytes =
    kCounterBytes + 2 * 8 * 256 * 4 + 16 * 4 + size_t(kMaxPasses) * (kMaxKeys / kTile + 1) * 256 * 4 + 8ull * kMaxKeys;

__device__ __align__(256) unsigned char g_sort_static[kStaticBytes];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
char* g_static_base[kMaxDevices] = {};
int g_static_sms[kMaxDevices] = {};
}  // namespace

extern "C" bb_status bb_radix_sort_pairs_static(const uint32_t* keys_in, const uint32_t* vals_in,
                                                uint32_t* keys_out, uint32_t* vals_out, uint32_t n,
                                                uint32_t key_bits, void* stream) {
  bb_status st = bb_check_sort_args(keys_in, vals_in, keys_out, vals_out, n, key_bits);
  if (st != BB_OK || n == 0) return st;
  if (n > kMaxKeys) return bb_fail(BB_E_INVALID, "radix sort (static scratch): n exceeds BB_SORT_STATIC_MAX_KEYS");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return bb_fail(BB_E_INVALID, "radix sort (static scratch): device index too large");
  char* base;
  int sms;
  {
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_base[dev]) {
      void* addr = nullptr;
      e = cudaGetSymbolAddress(&addr, g_sort_static);
      if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
      int count = 0;
      e = cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
      g_static_sms[dev] = count;
      g_static_base[dev] = static_cast<char*>(addr);
    }
    base = g_static_base[dev];
    sms = g_static_sms[dev];
  }
  const int passes = int((key_bits + 7) / 8);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DevCounters* ctr;
  uint32_t *hist, *tile_ctr, *status, *tk, *tv;
  size_t zero_bytes;
  bb_sort_carve(base, n, passes, &ctr, &hist, &tile_ctr, &status, &tk, &tv, &zero_bytes);
  // counters, histograms, tile counters and look-back status must start at zero; the
  // temporary key/value arrays need no clearing
  e = cudaMemsetAsync(base, 0, zero_bytes, s);
  if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
  uint32_t* dk[2] = {keys_out, tk};
  uint32_t* dv[2] = {vals_out, tv};
  bb_launch_sort_to(s, keys_in, vals_in, dk, dv, n, passes, hist, status, tile_ctr, ctr, sms);
  e = cudaGetLastError();
  if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
  return BB_OK;
}
