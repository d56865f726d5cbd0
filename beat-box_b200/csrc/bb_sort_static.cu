// bb_sort_static.cu -- bb_radix_sort_pairs_static: the same onesweep radix sort as
// bb_radix_sort_pairs, with its scratch in a fixed file-scope device array instead of a
// cudaMalloc'd block, so that a call allocates nothing (for callers that must not allocate
// device memory on their path, e.g. a real-time loop with a fixed memory budget).
//
// Scratch: BB_SORT_STATIC_MAX_KEYS keys at most.  Its address is looked up once per device
// with cudaGetSymbolAddress while that device is current; that first call loads the module's
// globals and so belongs before any stream capture.  The address is kept with the unique id of
// the CUDA context it was looked up in: after cudaDeviceReset the device gets a new context
// (new id), the array is reloaded at a new address, and the next call looks it up again.  All
// calls on one device share the array, so calls must not overlap in time (issue them on one
// stream, or order them with events).
#include <cstddef>
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
unsigned long long g_static_ctx[kMaxDevices] = {};

// Unique id of the calling thread's current CUDA context (0 if none or unknown), through the
// driver's cuCtxGetCurrent / cuCtxGetId fetched from the runtime (no link against libcuda).
unsigned long long current_context_id() {
  typedef int (*GetCurrent)(void**);
  typedef int (*GetId)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}
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
    const unsigned long long ctx = current_context_id();
    if (!g_static_base[dev] || ctx == 0 || ctx != g_static_ctx[dev]) {
      void* addr = nullptr;
      e = cudaGetSymbolAddress(&addr, g_sort_static);
      if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
      int count = 0;
      e = cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
      g_static_sms[dev] = count;
      g_static_base[dev] = static_cast<char*>(addr);
      g_static_ctx[dev] = current_context_id();  // the lookup made the device's context current
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

// Device error bits of the last sort on the current device (BB_ERRF_*; 0 = the sort ran to the
// end).  Waits for `stream`, then copies one word from the scratch's counters to the host.
extern "C" bb_status bb_radix_sort_error_flags(uint32_t static_scratch, void* stream, uint32_t* error_flags) {
  if (!error_flags) return bb_fail(BB_E_INVALID, "bb_radix_sort_error_flags: null output");
  *error_flags = 0;
  char* base = nullptr;
  if (static_scratch) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return bb_fail(BB_E_INVALID, "bb_radix_sort_error_flags: device index too large");
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (g_static_ctx[dev] == current_context_id()) base = g_static_base[dev];
  } else {
    base = bb_sort_scratch_base();
  }
  if (!base) return BB_OK;  // no sort has run on this device (in this context)
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(error_flags, base + offsetof(DevCounters, error_flags), sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
  return BB_OK;
}
