// bb_scan_sort.cu -- single-pass prefix scan and onesweep LSD radix sort.
//
// Replaces the reference's radix sort (histogram + scatter per 8-bit digit with a host
// transfer between passes, src/shaders/simulation/RB_sim.slang:113-203,
// src/shaders/simulation/LBVH.slang:34-152, RBM:1288-1295) with:
//   * one histogram kernel that counts all digit positions in a single read of the keys,
//   * one onesweep kernel per digit: tiles of 8192 keys rank themselves with warp-level
//     multisplit (one ballot per digit bit), publish per-digit tile totals, resolve their global
//     offsets by decoupled look-back over the preceding tiles, reorder the tile by digit in
//     shared memory and write each digit's run contiguously (coalesced stores).
// Both are stable, so the result equals a stable sort by key -- the reference's semantics.
// Element counts are read from device memory so the kernels can sit in a CUDA graph.
#include "bb_common.cuh"
#include "bb_kernels.cuh"

namespace {
constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;  // 2048 (scan)
constexpr int kSortThreads = 512;  // onesweep block
constexpr int kSortItems = BB_SORT_TILE / kSortThreads;  // 16 keys per thread in a onesweep tile
static_assert(kSortItems * kSortThreads == BB_SORT_TILE, "onesweep tile");
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1u;
}  // namespace

// ---------------------------------------------------------------------------------------
// exclusive scan of n u32 values: out[i] = sum(in[0..i)), *total = sum(in)
__global__ void __launch_bounds__(kThreads) k_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                   const uint32_t* __restrict__ n_ptr, uint32_t n_fixed,
                                                   uint32_t* total, unsigned long long* status, uint32_t* tile_ctr,
                                                   DevCounters* ctr, const uint32_t* __restrict__ skip) {
  __shared__ uint32_t s_tile, s_excl;
  __shared__ uint32_t s_warp[kThreads / 32];
  if (skip && *skip) return;
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
  __syncthreads();
  const uint32_t n = n_ptr ? min(*n_ptr, n_fixed) : n_fixed;
  const uint32_t tile = s_tile;
  const uint32_t base = tile * kTile;
  if (base >= n && !(n == 0 && tile == 0)) return;
  uint32_t v[kItems];
  uint32_t local = 0;
  const uint32_t i0 = base + threadIdx.x * kItems;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    uint32_t i = i0 + k;
    v[k] = i < n ? in[i] : 0u;
    local += v[k];
  }
  // block exclusive scan of the per-thread sums
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kThreads / 32 ? s_warp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kThreads / 32) s_warp[lane] = w;  // inclusive warp sums
  }
  __syncthreads();
  uint32_t block_total = s_warp[kThreads / 32 - 1];
  uint32_t excl_in_block = x - local + (warp > 0 ? s_warp[warp - 1] : 0u);
  // decoupled look-back by thread 0
  if (threadIdx.x == 0) {
    volatile unsigned long long* st = status;
    if (tile == 0) {
      st[0] = (2ull << 32) | block_total;
      s_excl = 0;
    } else {
      st[tile] = (1ull << 32) | block_total;
      uint32_t excl = 0;
      int32_t j = int32_t(tile) - 1;
      uint32_t spins = 0;
      while (j >= 0) {
        unsigned long long w = st[j];
        uint32_t flag = uint32_t(w >> 32);
        if (flag == 0) {
          if (++spins > BB_SPIN_LIMIT) {
            raise_wait_error(ctr, BB_SITE_SCAN);
            break;
          }
          continue;
        }
        excl += uint32_t(w);
        if (flag == 2) break;
        --j;
      }
      st[tile] = (2ull << 32) | (excl + block_total);
      s_excl = excl;
    }
  }
  __syncthreads();
  uint32_t run = s_excl + excl_in_block;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    uint32_t i = i0 + k;
    if (i < n) out[i] = run;
    run += v[k];
  }
  // the tile holding element n-1 (or tile 0 when n == 0) publishes the total
  if (total && threadIdx.x == 0 && (n == 0 ? tile == 0 : (n - 1) / kTile == tile)) *total = s_excl + block_total;
}

// ---------------------------------------------------------------------------------------
// Global histograms of `passes` 8-bit key digits starting at bit shift0, followed by
// `lut_passes` digits of lut[value] (world ids in batched worlds).  Rows: up to 8.
__global__ void __launch_bounds__(kThreads) k_sort_hist(const uint32_t* __restrict__ keys,
                                                        const uint32_t* __restrict__ vals,
                                                        const uint32_t* __restrict__ lut,
                                                        const uint32_t* __restrict__ n_ptr, uint32_t n_fixed,
                                                        uint32_t* hist, int passes, int lut_passes, int shift0) {
  __shared__ uint32_t s_hist[8][256];
  for (int i = threadIdx.x; i < 8 * 256; i += kThreads) (&s_hist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t n = n_ptr ? min(*n_ptr, n_fixed) : n_fixed;
  auto count = [&](uint32_t k, uint32_t v) {
    for (int p = 0; p < passes; ++p) atomicAdd(&s_hist[p][(k >> (shift0 + 8 * p)) & 255u], 1u);
    if (lut_passes) {
      uint32_t w = lut[v];
      for (int p = 0; p < lut_passes; ++p) atomicAdd(&s_hist[passes + p][(w >> (8 * p)) & 255u], 1u);
    }
  };
  // four keys per 16-byte load, two loads in flight per thread; arrays that do not start on a
  // 16-byte boundary (caller pointers into a buffer) take the scalar loop for every key
  const bool aligned = (reinterpret_cast<uintptr_t>(keys) & 15u) == 0 &&
                       (!lut_passes || (reinterpret_cast<uintptr_t>(vals) & 15u) == 0);
  const uint32_t n4 = aligned ? n / 4 : 0u, stride = gridDim.x * kThreads;
  const uint4* k4 = reinterpret_cast<const uint4*>(keys);
  const uint4* v4 = reinterpret_cast<const uint4*>(vals);
  uint32_t q = blockIdx.x * kThreads + threadIdx.x;
  for (; q + stride < n4; q += 2 * stride) {
    const uint4 a = k4[q], b = k4[q + stride];
    uint4 va = make_uint4(0, 0, 0, 0), vb = make_uint4(0, 0, 0, 0);
    if (lut_passes) {
      va = v4[q];
      vb = v4[q + stride];
    }
    count(a.x, va.x); count(a.y, va.y); count(a.z, va.z); count(a.w, va.w);
    count(b.x, vb.x); count(b.y, vb.y); count(b.z, vb.z); count(b.w, vb.w);
  }
  if (q < n4) {
    const uint4 a = k4[q];
    const uint4 va = lut_passes ? v4[q] : make_uint4(0, 0, 0, 0);
    count(a.x, va.x); count(a.y, va.y); count(a.z, va.z); count(a.w, va.w);
  }
  for (uint32_t r = 4 * n4 + blockIdx.x * kThreads + threadIdx.x; r < n; r += stride)  // the rest
    count(keys[r], lut_passes ? vals[r] : 0u);
  __syncthreads();
  for (int p = 0; p < passes + lut_passes; ++p) {
    uint32_t c = s_hist[p][threadIdx.x];
    if (c) atomicAdd(&hist[p * 256 + threadIdx.x], c);
  }
}

// exclusive scan of each 256-bin histogram row into hist_scan (count rows kept)
__global__ void k_sort_hist_scan(const uint32_t* hist, uint32_t* hist_scan, int passes) {
  __shared__ uint32_t s[256];
  for (int p = 0; p < passes; ++p) {
    uint32_t v = hist[p * 256 + threadIdx.x];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
      uint32_t y = threadIdx.x >= uint32_t(o) ? s[threadIdx.x - o] : 0u;
      __syncthreads();
      s[threadIdx.x] += y;
      __syncthreads();
    }
    hist_scan[p * 256 + threadIdx.x] = s[threadIdx.x] - v;
    __syncthreads();
  }
}

// one stable onesweep pass on digit (key >> shift) & 255, or (lut[value] >> shift) & 255
// when lut is given
__device__ __forceinline__ uint32_t sort_digit(uint32_t key, uint32_t val, const uint32_t* __restrict__ lut, int shift) {
  return ((lut ? lut[val] : key) >> shift) & 255u;
}

// Decoupled look-back for digit t of tile `tile`: the sum of digit t over all preceding tiles.
// The status words of 8 predecessors are loaded at once and walked in order (aggregates are
// added until an inclusive prefix), so a chain of tiles still in flight costs one load
// latency per 8 tiles instead of one per tile.  A word not yet published is re-read.
constexpr int kLookback = 8;
__device__ __forceinline__ uint32_t sort_lookback(volatile uint32_t* st, uint32_t tile, uint32_t t, DevCounters* ctr) {
  uint32_t excl = 0, spins = 0;
  int32_t j = int32_t(tile) - 1;
  while (j >= 0) {
    uint32_t w[kLookback];
#pragma unroll
    for (int k = 0; k < kLookback; ++k) {
      w[k] = 2u << 30;  // before tile 0: an empty inclusive prefix
      if (j - k >= 0) w[k] = st[uint32_t(j - k) * 256u + t];
    }
    int k = 0;
    for (; k < kLookback; ++k) {
      const uint32_t flag = w[k] & ~kValMask;
      if (flag == 0) break;  // not yet published: re-read from here
      excl += w[k] & kValMask;
      if (flag == kFlagPrefix) return excl;
    }
    j -= k;
    if (k < kLookback && ++spins > BB_SPIN_LIMIT) {
      raise_wait_error(ctr, BB_SITE_SORT);
      return excl;
    }
  }
  return excl;
}

// one stable onesweep pass on digit (key >> shift) & 255, or (lut[value] >> shift) & 255
// when lut is given.  A tile is BB_SORT_TILE = 8192 keys on kSortThreads = 512 threads (16 keys
// each), so each digit's run in a tile averages 32 keys (128-byte lines when written out).  The
// values are read when the tile is reordered, not held through the ranking (registers: two
// blocks per SM); with a lut the digit needs the value, which the ranking reads then.
// Shared memory (dynamic, kSortSmem bytes): per-warp digit counts 16 x 256, keys and values of
// the tile, the digit of each reordered position.
constexpr int kSortWarps = kSortThreads / 32;
constexpr size_t kSortSmem = size_t(kSortWarps) * 256 * 4 + size_t(BB_SORT_TILE) * (4 + 4 + 1);
__global__ void __launch_bounds__(kSortThreads, 2) k_onesweep(const uint32_t* __restrict__ keys_in,
                                                              const uint32_t* __restrict__ vals_in,
                                                              uint32_t* __restrict__ keys_out,
                                                              uint32_t* __restrict__ vals_out,
                                                              const uint32_t* __restrict__ n_ptr, uint32_t n_fixed,
                                                              const uint32_t* __restrict__ digit_start, int shift,
                                                              const uint32_t* __restrict__ lut, uint32_t* status,
                                                              uint32_t* tile_ctr, DevCounters* ctr) {
  extern __shared__ __align__(16) uint8_t s_dyn[];
  uint32_t(*s_warp_hist)[256] = reinterpret_cast<uint32_t(*)[256]>(s_dyn);
  uint32_t* s_keys = reinterpret_cast<uint32_t*>(s_dyn + size_t(kSortWarps) * 256 * 4);
  uint32_t* s_vals = s_keys + BB_SORT_TILE;
  uint8_t* s_dig = reinterpret_cast<uint8_t*>(s_vals + BB_SORT_TILE);
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_offset[256];  // global position of this tile's first key of digit d
  __shared__ uint32_t s_local[256];   // tile position of its first key of digit d
  __shared__ uint32_t s_wsum[8];
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
  for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&s_warp_hist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t n = n_ptr ? min(*n_ptr, n_fixed) : n_fixed;
  const uint32_t tile = s_tile;
  const uint32_t base = tile * BB_SORT_TILE;
  if (base >= n) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt_mask = (1u << lane) - 1u;
  const uint32_t first = base + warp * (32 * kSortItems) + lane;
  uint32_t key[kSortItems], rank[kSortItems];
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const uint32_t i = first + k * 32;
    key[k] = i < n ? keys_in[i] : 0u;
  }
  // warp-level multisplit: rank of each key among its warp's keys of the same digit, in order.
  // The lanes holding the same digit are found with one ballot per digit bit (plus one for the
  // keys past n); only the lowest of them reads and advances the warp's count of that digit, and
  // the others take the old count from it by a shuffle.  rank keeps the digit in its top 8 bits.
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const bool valid = first + k * 32 < n;
    const uint32_t d = valid ? sort_digit(key[k], lut ? vals_in[first + k * 32] : 0u, lut, shift) : 0u;
    uint32_t peers = __ballot_sync(0xFFFFFFFFu, valid);
    if (!valid) peers = ~peers;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const uint32_t bal = __ballot_sync(0xFFFFFFFFu, (d >> b) & 1u);
      peers &= ((d >> b) & 1u) ? bal : ~bal;
    }
    const int leader = __ffs(peers) - 1;
    uint32_t prior = 0;
    if (valid && lane == leader) {
      prior = s_warp_hist[warp][d];
      s_warp_hist[warp][d] = prior + __popc(peers);
    }
    prior = __shfl_sync(0xFFFFFFFFu, prior, leader);
    rank[k] = (d << 24) | (prior + __popc(peers & lt_mask));
    __syncwarp();
  }
  __syncthreads();
  // per digit t (threads 0..255): exclusive prefix over warps, and the tile's count of digit t
  const uint32_t t = threadIdx.x;
  volatile uint32_t* st = status;
  uint32_t sum = 0, x = 0;
  if (t < 256) {
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = s_warp_hist[w][t];
      s_warp_hist[w][t] = sum;
      sum += c;
    }
    // publish the tile's counts first, so that later tiles can look past this one early
    st[tile * 256 + t] = (tile == 0 ? kFlagPrefix : kFlagAgg) | sum;
    // tile-local start of each digit: block exclusive scan of the counts (warps 0..7)
    x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_wsum[warp] = x;
  }
  __syncthreads();
  if (t < 256) {
    uint32_t wo = 0;
    for (int w = 0; w < warp; ++w) wo += s_wsum[w];
    s_local[t] = wo + x - sum;
    // keys of digit t in the preceding tiles
    uint32_t excl = 0;
    if (tile > 0) {
      excl = sort_lookback(st, tile, t, ctr);
      st[tile * 256 + t] = kFlagPrefix | (excl + sum);
    }
    s_offset[t] = digit_start[t] + excl;
  }
  __syncthreads();
  // reorder the tile by digit (stable: warps and ranks follow the input order) ...
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const uint32_t i = first + k * 32;
    if (i < n) {
      const uint32_t d = rank[k] >> 24;
      const uint32_t lp = s_local[d] + s_warp_hist[warp][d] + (rank[k] & 0xFFFFFFu);
      s_keys[lp] = key[k];
      s_vals[lp] = vals_in[i];
      s_dig[lp] = uint8_t(d);
    }
  }
  __syncthreads();
  // ... and write each digit's run of the tile contiguously
  const uint32_t nt = min(uint32_t(BB_SORT_TILE), n - base);
  for (uint32_t i = t; i < nt; i += kSortThreads) {
    const uint32_t d = s_dig[i];
    const uint32_t dst = s_offset[d] + (i - s_local[d]);
    keys_out[dst] = s_keys[i];
    vals_out[dst] = s_vals[i];
  }
}

// dynamic shared memory of k_onesweep above the 48 KB default: set once per device (the first
// sort on a device should come before any stream capture; bb_world_create makes that call)
void onesweep_smem_attr() {
  static bool done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !done[dev]) {
    cudaFuncSetAttribute((const void*)k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSortSmem));
    done[dev] = true;
  }
}

// ---------------------------------------------------------------------------------------
// host launchers
void bb_launch_scan(cudaStream_t s, const uint32_t* in, uint32_t* out, const uint32_t* n_dev, uint32_t n_cap,
                    uint32_t* total, unsigned long long* status, uint32_t* tile_ctr, DevCounters* ctr,
                    const uint32_t* skip) {
  uint32_t tiles = (n_cap + kTile - 1) / kTile;
  if (tiles == 0) tiles = 1;
  k_scan<<<tiles, kThreads, 0, s>>>(in, out, n_dev, n_cap, total, status, tile_ctr, ctr, skip);
}

uint32_t bb_scan_tiles(uint32_t n_cap) { return n_cap / kTile + 1; }
uint32_t bb_sort_tiles(uint32_t n_cap) { return n_cap / BB_SORT_TILE + 1; }

// Sorts `passes` digits: pass 0 reads (keys_in, vals_in); pass k writes buffer
// dst[(passes - 1 - k) & 1] and the next pass reads it, so the last pass lands in dst[0].
// hist: 2 x 4 x 256 words (counts, exclusive starts), zeroed; status: passes x tiles x 256
// words, zeroed; tile_ctr: passes words, zeroed.
void bb_launch_sort_to(cudaStream_t s, const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* dst_keys[2],
                       uint32_t* dst_vals[2], uint32_t n, int passes, uint32_t* hist, uint32_t* status,
                       uint32_t* tile_ctr, DevCounters* ctr, int sms) {
  onesweep_smem_attr();
  uint32_t tiles = (n + BB_SORT_TILE - 1) / BB_SORT_TILE;
  if (tiles == 0) tiles = 1;
  k_sort_hist<<<sms * 4, kThreads, 0, s>>>(keys_in, vals_in, nullptr, nullptr, n, hist, passes, 0, 0);
  k_sort_hist_scan<<<1, 256, 0, s>>>(hist, hist + 8 * 256, passes);
  const uint32_t* ik = keys_in;
  const uint32_t* iv = vals_in;
  for (int p = 0; p < passes; ++p) {
    int o = (passes - 1 - p) & 1;
    k_onesweep<<<tiles, kSortThreads, kSortSmem, s>>>(ik, iv, dst_keys[o], dst_vals[o], nullptr, n, hist + 8 * 256 + p * 256, 8 * p,
                                          nullptr, status + size_t(p) * tiles * 256, tile_ctr + p, ctr);
    ik = dst_keys[o];
    iv = dst_vals[o];
  }
}

// Sorts `passes` key digits (from bit shift0) and then `lut_passes` digits of lut[value] in
// place between buffers 0 and 1; result in buffer (passes + lut_passes) % 2.  hist: one region
// of 2 x 8 x 256 words (counts, exclusive starts), zeroed; status: (passes + lut_passes) x
// tiles x 256 words, zeroed; tile_ctr: one word per pass, zeroed.
void bb_launch_sort(cudaStream_t s, uint32_t* keys[2], uint32_t* vals[2], const uint32_t* n_dev, uint32_t n_cap,
                    int passes, int shift0, uint32_t* hist, uint32_t* status, uint32_t* tile_ctr, DevCounters* ctr,
                    int sms, const uint32_t* lut, int lut_passes) {
  onesweep_smem_attr();
  uint32_t tiles = (n_cap + BB_SORT_TILE - 1) / BB_SORT_TILE;
  if (tiles == 0) tiles = 1;
  const int total = passes + (lut ? lut_passes : 0);
  k_sort_hist<<<sms * 4, kThreads, 0, s>>>(keys[0], vals[0], lut, n_dev, n_cap, hist, passes, lut ? lut_passes : 0,
                                           shift0);
  k_sort_hist_scan<<<1, 256, 0, s>>>(hist, hist + 8 * 256, total);
  for (int p = 0; p < total; ++p) {
    int in = p & 1, out = in ^ 1;
    bool by_lut = p >= passes;
    k_onesweep<<<tiles, kSortThreads, kSortSmem, s>>>(keys[in], vals[in], keys[out], vals[out], n_dev, n_cap,
                                          hist + 8 * 256 + p * 256, by_lut ? 8 * (p - passes) : shift0 + 8 * p,
                                          by_lut ? lut : nullptr, status + size_t(p) * tiles * 256, tile_ctr + p,
                                          ctr);
  }
}
