// bb_sort_api.cu -- stand-alone device radix sort: the step's Morton-code sort (onesweep,
// decoupled look-back, warp multisplit) exposed on caller-owned device arrays.
//
// No single reference entry point corresponds to it: the reference sorts its Morton codes inside
// the task graph (histogram + scatter per digit, src/shaders/simulation/RB_sim.slang:113-203,
// LBVH.slang:34-152, passes at src/rigid_body_manager.cpp:1288-1295).
#include <mutex>
#include <vector>

#include "bb_common.cuh"
#include "bb_kernels.cuh"

namespace {
constexpr uint32_t kTile = BB_SORT_TILE;

struct SortScratch {
  int device = -1;
  char* base = nullptr;
  size_t bytes = 0;
};
std::mutex g_sort_mu;
std::vector<SortScratch> g_sort_cache;

size_t sort_scratch_bytes(uint32_t n, int passes) {
  size_t tiles = n / kTile + 1;
  return 256 + sizeof(DevCounters) + 2 * 8 * 256 * 4 + 16 * 4 + size_t(passes) * tiles * 256 * 4 + 8ull * n;
}
}  // namespace

// Carves a scratch block into the sort's working arrays; everything before tmp must start
// at zero and is cleared by the caller.
void bb_sort_carve(char* base, uint32_t n, int passes, DevCounters** ctr, uint32_t** hist, uint32_t** tile_ctr,
                   uint32_t** status, uint32_t** tmp_keys, uint32_t** tmp_vals, size_t* zero_bytes) {
  size_t tiles = n / kTile + 1;
  char* p = base;
  *ctr = reinterpret_cast<DevCounters*>(p);
  p += (sizeof(DevCounters) + 255) / 256 * 256;
  *hist = reinterpret_cast<uint32_t*>(p);
  p += 2 * 8 * 256 * 4;
  *tile_ctr = reinterpret_cast<uint32_t*>(p);
  p += 16 * 4;
  *status = reinterpret_cast<uint32_t*>(p);
  p += size_t(passes) * tiles * 256 * 4;
  *zero_bytes = size_t(p - base);
  *tmp_keys = reinterpret_cast<uint32_t*>(p);
  *tmp_vals = *tmp_keys + n;
}

// Scratch block of bb_radix_sort_pairs on the current device (nullptr before its first call).
char* bb_sort_scratch_base() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(g_sort_mu);
  for (auto& c : g_sort_cache)
    if (c.device == dev) return c.base;
  return nullptr;
}

bb_status bb_check_sort_args(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                             uint32_t n, uint32_t key_bits) {
  if (key_bits == 0 || key_bits > 32) return bb_fail(BB_E_INVALID, "radix sort: key_bits must be 1..32");
  if (n == 0) return BB_OK;
  if (!keys_in || !vals_in || !keys_out || !vals_out) return bb_fail(BB_E_INVALID, "radix sort: null array");
  if (keys_in == keys_out || vals_in == vals_out) return bb_fail(BB_E_INVALID, "radix sort: input and output alias");
  if (n > (1u << 30) - 1) return bb_fail(BB_E_INVALID, "radix sort: n must be below 2^30");
  return BB_OK;
}

extern "C" bb_status bb_radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                         uint32_t* vals_out, uint32_t n, uint32_t key_bits, void* stream) {
  bb_status st = bb_check_sort_args(keys_in, vals_in, keys_out, vals_out, n, key_bits);
  if (st != BB_OK || n == 0) return st;
  const int passes = int((key_bits + 7) / 8);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> lk(g_sort_mu);
  SortScratch* sc = nullptr;
  for (auto& c : g_sort_cache)
    if (c.device == dev) sc = &c;
  if (!sc) {
    g_sort_cache.push_back(SortScratch{dev, nullptr, 0});
    sc = &g_sort_cache.back();
  }
  const size_t need = sort_scratch_bytes(n, passes);
  if (sc->bytes < need) {
    // the previous block may still be in use by earlier calls on any stream
    if (sc->base) {
      cudaDeviceSynchronize();
      cudaFree(sc->base);
    }
    sc->base = nullptr;
    sc->bytes = 0;
    cudaError_t e = cudaMalloc(&sc->base, need);
    if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
    sc->bytes = need;
  }
  DevCounters* ctr;
  uint32_t *hist, *tile_ctr, *status, *tk, *tv;
  size_t zero_bytes;
  bb_sort_carve(sc->base, n, passes, &ctr, &hist, &tile_ctr, &status, &tk, &tv, &zero_bytes);
  cudaError_t e = cudaMemsetAsync(sc->base, 0, zero_bytes, s);
  if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
  uint32_t* dk[2] = {keys_out, tk};
  uint32_t* dv[2] = {vals_out, tv};
  bb_launch_sort_to(s, keys_in, vals_in, dk, dv, n, passes, hist, status, tile_ctr, ctr, sms);
  e = cudaGetLastError();
  if (e != cudaSuccess) return bb_fail(BB_E_CUDA, cudaGetErrorString(e));
  return BB_OK;
}
