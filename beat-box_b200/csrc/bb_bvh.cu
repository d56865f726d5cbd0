// bb_bvh.cu -- Morton codes, radix sort, Karras LBVH build, atomic bottom-up refit and the
// broad phase.
//
// Reference: entry_generate_morton_codes (src/shaders/simulation/RB_sim.slang:75-111),
// MortonCodeGenerator (src/shaders/simulation/LBVH.slang:4-32), entry_generate_hierarchy_
// linear_bvh + LBVH::determine_range/find_split/delta (RB_sim.slang:206-278, LBVH.slang:
// 155-221), entry_build/convert_bounding_boxes_linear_bvh (RB_sim.slang:282-349),
// entry_broad_phase + LBVH::broad_phase (RB_sim.slang:413-437, LBVH.slang:223-286).
//
// B200 design: the body state is never gathered into Morton order (the reference copies its
// 184-byte AoS bodies every step, RB_sim.slang:351-386); the sort carries body ids and every
// later stage indexes the SoA arrays by id.  Keys are emitted in the previous substep's
// sorted order, so ties break exactly like the reference's scratch-array order.  The refit
// uses one arrival counter per internal node (second arriver merges) instead of the
// reference's O(N depth) per-leaf atomic min/max walk; float min/max is exact, so the boxes
// are identical.  The broad phase traverses left-first and prunes subtrees whose leaf range
// ends at or before the query, so each query emits its partners j > i in ascending order and
// the pair list comes out sorted by (a, b) with no global atomic per pair.
#include "bb_common.cuh"
#include "bb_kernels.cuh"

// ---- FP32-exact geometry (no contraction) -------------------------------------------------
__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}
__device__ __forceinline__ float morton_axis(float p, float mn, float ext) {
  float x = __fdiv_rn(__fsub_rn(p, mn), ext);
  x = __fmul_rn(x, 1024.0f);
  x = fminf(fmaxf(x, 0.0f), 1023.0f);
  return x;
}
__device__ __forceinline__ uint32_t morton_code(float3 p, const float wmin[3], const float wext[3]) {
  uint32_t xx = expand_bits(__float2uint_rz(morton_axis(p.x, wmin[0], wext[0])));
  uint32_t yy = expand_bits(__float2uint_rz(morton_axis(p.y, wmin[1], wext[1])));
  uint32_t zz = expand_bits(__float2uint_rz(morton_axis(p.z, wmin[2], wext[2])));
  return xx * 4 + yy * 2 + zz;
}

// RigidBody::get_AABB_from_OBB (src/shaders/extensions.slang:195-210): the 8 corners of the
// box [minimum, maximum] rotated by the quaternion sandwich q c q* (include/shared.inl:455-475)
// plus position.  Boxes have [minimum, maximum] = [-half, half]; voxel bodies their grid box,
// which is off-centre (the body origin is the centre of mass).
__device__ __forceinline__ void leaf_box(const DevState& d, float4 shp, float4 p4, float4 q4, float4& mn, float4& mx) {
  uint32_t type = __float_as_uint(shp.w);
  if (type == BB_SHAPE_SPHERE) {
    float r = shp.x;
    mn = make_float4(__fsub_rn(p4.x, r), __fsub_rn(p4.y, r), __fsub_rn(p4.z, r), 0.f);
    mx = make_float4(__fadd_rn(p4.x, r), __fadd_rn(p4.y, r), __fadd_rn(p4.z, r), 0.f);
    return;
  }
  float lo[3] = {-shp.x, -shp.y, -shp.z}, hi[3] = {shp.x, shp.y, shp.z};
  if (BB_SHAPE_KIND(type) == BB_SHAPE_VOXEL) {
    const VoxDev& v = d.vox[BB_SHAPE_VOXEL_INDEX(type)];
    lo[0] = v.ox;
    lo[1] = v.oy;
    lo[2] = v.oz;
    hi[0] = v.hx;
    hi[1] = v.hy;
    hi[2] = v.hz;
  }
  Quatf q = q_from(q4);
  Quatf qc = q_conj(q);
  float blo[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
  float bhi[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    Quatf c{(i & 1) ? hi[0] : lo[0], (i & 2) ? hi[1] : lo[1], (i & 4) ? hi[2] : lo[2], 0.f};
    Quatf r = q_mul_exact(q_mul_exact(q, c), qc);
    float w[3] = {__fadd_rn(r.x, p4.x), __fadd_rn(r.y, p4.y), __fadd_rn(r.z, p4.z)};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      blo[k] = w[k] < blo[k] ? w[k] : blo[k];
      bhi[k] = w[k] > bhi[k] ? w[k] : bhi[k];
    }
  }
  mn = make_float4(blo[0], blo[1], blo[2], 0.f);
  mx = make_float4(bhi[0], bhi[1], bhi[2], 0.f);
}

__device__ __forceinline__ bool box_overlap(float4 amn, float4 amx, float4 bmn, float4 bmx) {
  return amn.x <= bmx.x && amx.x >= bmn.x && amn.y <= bmx.y && amx.y >= bmn.y && amn.z <= bmx.z && amx.z >= bmn.z;
}

// ---- kernels ---------------------------------------------------------------------------------
__global__ void k_bounds(const DevState d, uint32_t n) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = d.pos[i];
  atomicMin(&d.ctr->bounds_min[0], f2ord(p.x));
  atomicMin(&d.ctr->bounds_min[1], f2ord(p.y));
  atomicMin(&d.ctr->bounds_min[2], f2ord(p.z));
  atomicMax(&d.ctr->bounds_max[0], f2ord(p.x));
  atomicMax(&d.ctr->bounds_max[1], f2ord(p.y));
  atomicMax(&d.ctr->bounds_max[2], f2ord(p.z));
}

// keys[0][i] = Morton code of body vals[0][i] (the previous substep's sorted order).
__global__ void k_morton(const DevState d, uint32_t n, Params p) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float wmin[3], wext[3];
  if (p.bounds_mode == BB_BOUNDS_AUTO) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float lo = ord2f(d.ctr->bounds_min[k]), hi = ord2f(d.ctr->bounds_max[k]);
      float e = __fsub_rn(hi, lo);
      wmin[k] = lo;
      wext[k] = e > 0.0f ? e : 1.0f;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      wmin[k] = p.world_min[k];
      wext[k] = p.world_extent[k];
    }
  }
  uint32_t id = d.vals[0][i];
  if (d.n_worlds >= 1) {  // batched worlds: each world normalises by its own box
    uint32_t w = d.world_of[id];
    float4 a = d.world_bounds[2 * w], b = d.world_bounds[2 * w + 1];
    wmin[0] = a.x; wmin[1] = a.y; wmin[2] = a.z;
    wext[0] = b.x; wext[1] = b.y; wext[2] = b.z;
  }
  d.keys[0][i] = morton_code(f3(d.pos[id]), wmin, wext);
}

// world of every sorted position (batched worlds only)
__global__ void k_sorted_world(const DevState d, uint32_t n) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d.sworld[i] = d.world_of[d.vals[0][i]];
}

// LBVH::delta (LBVH.slang:158-170) on the key (world, code): with batched worlds the world id
// forms the 32 high bits, so a pair of different worlds shares fewer prefix bits than any pair
// inside one world, and each world's range is one subtree.  sw == nullptr: single world.
__device__ __forceinline__ int clz_delta(const uint32_t* codes, const uint32_t* sw, int n, int i, uint32_t ci,
                                         uint32_t wi, int j) {
  if (j < 0 || j > n - 1) return -1;
  int base = 0;
  if (sw) {
    uint32_t wj = sw[j];
    if (wi != wj) return __clz(wi ^ wj);
    base = 32;
  }
  uint32_t cj = codes[j];
  if (ci == cj) return base + 32 + __clz(uint32_t(i ^ j));
  return base + __clz(ci ^ cj);
}

// leaves in sorted order + Karras internal nodes (LBVH.slang:155-221, RB_sim.slang:206-278)
__global__ void k_build(const DevState d, uint32_t n) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* codes = d.keys[0];
  const uint32_t* sw = d.n_worlds > 1 ? d.sworld : nullptr;
  uint32_t id = d.vals[0][i];
  d.rank[id] = i;
  float4 mn, mx;
  leaf_box(d, d.shape[id], d.pos[id], d.rot[id], mn, mx);
  uint32_t leaf = n - 1 + i;
  d.node_box[2 * leaf] = mn;
  d.node_box[2 * leaf + 1] = mx;
  if (i == 0) d.parent[0] = -1;
  if (i + 1 >= n) return;
  const int N = int(n), idx = int(i);
  uint32_t code = codes[idx];
  uint32_t wi = sw ? sw[idx] : 0u;
  int dl = clz_delta(codes, sw, N, idx, code, wi, idx - 1);
  int dr = clz_delta(codes, sw, N, idx, code, wi, idx + 1);
  int dir = dr >= dl ? 1 : -1;
  int dmin = min(dl, dr);
  int lmax = 2;
  while (clz_delta(codes, sw, N, idx, code, wi, idx + lmax * dir) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t > 0; t >>= 1)
    if (clz_delta(codes, sw, N, idx, code, wi, idx + (l + t) * dir) > dmin) l += t;
  int j = idx + l * dir;
  int first = min(idx, j), last = max(idx, j);
  uint32_t fc = codes[first];
  uint32_t fw = sw ? sw[first] : 0u;
  int common = clz_delta(codes, sw, N, first, fc, fw, last);
  int split = first, step = last - first;
  do {
    step = (step + 1) >> 1;
    int ns = split + step;
    if (ns < last && clz_delta(codes, sw, N, first, fc, fw, ns) > common) split = ns;
  } while (step > 1);
  int ca = split == first ? N - 1 + split : split;
  int cb = split + 1 == last ? N - 1 + split + 1 : split + 1;
  d.child[i] = make_int2(ca, cb);
  d.parent[ca] = idx;
  d.parent[cb] = idx;
  d.range_last[i] = last;
  d.range_first[i] = first;
  d.visit[i] = 0;
}

__device__ __forceinline__ uint32_t atom_add_acq_rel_gpu(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Bottom-up refit: the second child to arrive at a node merges both boxes and climbs on.  The
// arrival counter is one acquire-release atomic: its release publishes the arriving thread's
// box, its acquire makes the sibling's box visible to the second arriver.  The thread that
// merges a node also writes the node's traversal record (below), so the records cost no pass
// of their own over the node boxes.
__device__ __forceinline__ void write_node_rec(const DevState& d, int p, int2 c, int leaf0, float4 lmn, float4 lmx,
                                               float4 rmn, float4 rmx);

__global__ void k_refit(const DevState d, uint32_t n) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || n < 2) return;
  const int leaf0 = int(n) - 1;
  int node = d.parent[leaf0 + i];
  uint32_t guard = 0;
  while (node >= 0) {
    if (atom_add_acq_rel_gpu(&d.visit[node], 1u) == 0u) return;  // first arriver: sibling not ready
    int2 c = d.child[node];
    float4 amn = __ldcg(&d.node_box[2 * c.x]), amx = __ldcg(&d.node_box[2 * c.x + 1]);
    float4 bmn = __ldcg(&d.node_box[2 * c.y]), bmx = __ldcg(&d.node_box[2 * c.y + 1]);
    float4 mn = make_float4(bmn.x < amn.x ? bmn.x : amn.x, bmn.y < amn.y ? bmn.y : amn.y,
                            bmn.z < amn.z ? bmn.z : amn.z, 0.f);
    float4 mx = make_float4(bmx.x > amx.x ? bmx.x : amx.x, bmx.y > amx.y ? bmx.y : amx.y,
                            bmx.z > amx.z ? bmx.z : amx.z, 0.f);
    __stcg(&d.node_box[2 * node], mn);
    __stcg(&d.node_box[2 * node + 1], mx);
    write_node_rec(d, node, c, leaf0, amn, amx, bmn, bmx);
    node = d.parent[node];
    if (++guard > 128u) {  // a Karras tree over 30-bit codes + 32 index bits is < 64 deep
      raise_error(d.ctr, BB_ERRF_STACK_OVERFLOW);
      return;
    }
  }
}

// A query that visits more than BB_BP_BUDGET nodes (a huge static body: floor, walls) is
// handed to k_broad_heavy, which splits its traversal over a block.
#define BB_BP_BUDGET 128u  // a serial walk longer than this sets the kernel's tail: hand it off
#define BB_BP_STAGE 32u   // partners per query kept from the counting traversal
#define BB_HEAVY_CAP 8192u
#define BB_FRONTIER 256

// Internal node records for the traversals: both children's boxes, indices and leaf ranges in
// one 80-byte record (5 float4), written by the refit when it merges the node.  A visit is then
// one dependent load (instead of the child indices, then each child's range and box), and a
// leaf child is tested from its parent's record without being visited.  Layout: (lmin.xyz,
// lmax.x), (lmax.yz, rmin.xy), (rmin.z, rmax.xyz), (left, right, left last leaf, right last
// leaf), (left first leaf, right first leaf, -, -).
__device__ __forceinline__ void write_node_rec(const DevState& d, int p, int2 c, int leaf0, float4 lmn, float4 lmx,
                                               float4 rmn, float4 rmx) {
  const int lf = c.x >= leaf0 ? c.x - leaf0 : d.range_first[c.x], ll = c.x >= leaf0 ? c.x - leaf0 : d.range_last[c.x];
  const int rf = c.y >= leaf0 ? c.y - leaf0 : d.range_first[c.y], rl = c.y >= leaf0 ? c.y - leaf0 : d.range_last[c.y];
  float4* r = d.node_rec + 5 * size_t(p);
  r[0] = make_float4(lmn.x, lmn.y, lmn.z, lmx.x);
  r[1] = make_float4(lmx.y, lmx.z, rmn.x, rmn.y);
  r[2] = make_float4(rmn.z, rmx.x, rmx.y, rmx.z);
  r[3] = make_float4(__int_as_float(c.x), __int_as_float(c.y), __int_as_float(ll), __int_as_float(rl));
  r[4] = make_float4(__int_as_float(lf), __int_as_float(rf), 0.f, 0.f);
}

struct Kids {
  int l, r;       // child nodes
  bool tl, tr;    // worth visiting from query qi: leaves in (qi, wend) and a box overlapping the query's
  int lspan, rspan;  // leaves under each
};
// wend = n for one world; the end of the query's world otherwise
__device__ __forceinline__ Kids rec_take(const DevState& d, int p, int qi, int wend, float4 qmn, float4 qmx) {
  const float4* r = d.node_rec + 5 * size_t(p);
  const float4 a = r[0], b = r[1], c = r[2], e = r[3], f = r[4];
  Kids k;
  k.l = __float_as_int(e.x);
  k.r = __float_as_int(e.y);
  const int ll = __float_as_int(e.z), rl = __float_as_int(e.w), lf = __float_as_int(f.x), rf = __float_as_int(f.y);
  k.lspan = ll - lf + 1;
  k.rspan = rl - rf + 1;
  k.tl = ll > qi && lf < wend &&
         box_overlap(qmn, qmx, make_float4(a.x, a.y, a.z, 0.f), make_float4(a.w, b.x, b.y, 0.f));
  k.tr = rl > qi && rf < wend &&
         box_overlap(qmn, qmx, make_float4(b.z, b.w, c.x, 0.f), make_float4(c.y, c.z, c.w, 0.f));
  return k;
}

// Left-first walk of the subtree at `root` (taken by the query already) for query qi: calls
// leaf(j) for every partner j in ascending order.  Taken leaf children are reported from their
// parent's record at once when nothing to their left is still pending; a right leaf child whose
// left sibling subtree is pending goes on the stack as a marker.  Stops and returns false after
// `budget` pops (the caller hands the query to a wider path).
template <class F>
__device__ __forceinline__ bool walk_query(const DevState& d, int root, int leaf0, int qi, int wend, float4 qmn,
                                           float4 qmx, uint32_t budget, F&& leaf) {
  if (root >= leaf0) {
    leaf(uint32_t(root - leaf0));
    return true;
  }
  int stack[BB_BVH_STACK];
  int sp = 0;
  stack[sp++] = root;
  uint32_t pops = 0;
  while (sp > 0) {
    if (++pops > budget) return false;
    const int node = stack[--sp];
    if (node >= leaf0) {  // a marker: a taken leaf whose left neighbours are done
      leaf(uint32_t(node - leaf0));
      continue;
    }
    const Kids k = rec_take(d, node, qi, wend, qmn, qmx);
    const bool l_leaf = k.l >= leaf0, r_leaf = k.r >= leaf0;
    const bool l_push = k.tl && !l_leaf;
    if (k.tl && l_leaf) leaf(uint32_t(k.l - leaf0));
    if (k.tr) {
      if (r_leaf && !l_push) {
        leaf(uint32_t(k.r - leaf0));
      } else if (sp < BB_BVH_STACK) {
        stack[sp++] = k.r;
      } else {
        raise_error(d.ctr, BB_ERRF_STACK_OVERFLOW);
      }
    }
    if (l_push) {
      if (sp < BB_BVH_STACK) stack[sp++] = k.l;
      else raise_error(d.ctr, BB_ERRF_STACK_OVERFLOW);
    }
  }
  return true;
}

__device__ __forceinline__ int world_end(const DevState& d, uint32_t qi, uint32_t n) {
  if (d.n_worlds <= 1) return int(n);
  uint32_t w = d.sworld[qi];
  return int(d.world_first[w] + d.world_count[w]);
}

// Left-first traversal for sorted query i.  EMIT=false counts every partner and keeps the first
// BB_BP_STAGE of them in bp_stage (so k_broad_copy can place them once offsets are known);
// EMIT=true re-walks only the queries that had more (is_heavy == 2) and writes their pairs.
template <bool EMIT>
__global__ void __launch_bounds__(128) k_broad(const DevState d, uint32_t n) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (n < 2) {
    if (!EMIT) {
      d.pair_cnt[i] = 0;
      d.is_heavy[i] = 0;
    }
    return;
  }
  if (EMIT && d.is_heavy[i] != 2u) return;
  const int N = int(n);
  const int leaf0 = N - 1;
  float4 qmn = d.node_box[2 * (leaf0 + i)], qmx = d.node_box[2 * (leaf0 + i) + 1];
  const int wend = world_end(d, i, n);
  const uint32_t out = EMIT ? d.pair_off[i] : 0u;
  const uint32_t cap = d.pair_capacity;
  uint32_t count = 0;
  auto leaf = [&](uint32_t j) {
    if (EMIT) {
      const uint32_t k = out + count;
      if (k < cap) d.pairs[k] = make_uint2(i, j);
      else raise_error(d.ctr, BB_ERRF_PAIR_OVERFLOW);
    } else if (count < BB_BP_STAGE) {
      d.bp_stage[size_t(i) * BB_BP_STAGE + count] = j;
    }
    ++count;
  };
  if (!walk_query(d, 0, leaf0, int(i), wend, qmn, qmx, EMIT ? 0xFFFFFFFFu : BB_BP_BUDGET, leaf)) {
    const uint32_t slot = atomicAdd(&d.ctr->heavy_n, 1u);
    if (slot < BB_HEAVY_CAP) {
      d.heavy_list[slot] = i;
      d.is_heavy[i] = 1;
      return;  // pair_cnt[i] is written by the heavy path
    }
    count = 0;  // heavy list full: walk it here after all
    walk_query(d, 0, leaf0, int(i), wend, qmn, qmx, 0xFFFFFFFFu, leaf);
  }
  if (!EMIT) {
    d.pair_cnt[i] = count;
    d.is_heavy[i] = count > BB_BP_STAGE ? 2u : 0u;
  }
}

// pairs of the queries whose partners all fit in bp_stage.  A warp takes 32 consecutive queries,
// scans their counts, and its lanes then write the warp's pairs 32 at a time, each lane finding
// its query by a binary search over the scanned counts (shuffles): every lane has work, and a
// pair's place pair_off[i] + k and value are those of the staged slot.
__global__ void k_broad_copy(const DevState d, uint32_t n) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  const uint32_t cap = d.pair_capacity;
  const int lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t q0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; q0 < n; q0 += nwarps * 32u) {  // warp-uniform
    const uint32_t i = q0 + lane;
    uint32_t cnt = 0, off = 0;
    if (i < n && d.is_heavy[i] == 0u) {
      cnt = d.pair_cnt[i];
      off = d.pair_off[i];
    }
    uint32_t inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
      if (lane >= o) inc += y;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, inc, 31);
    const uint32_t exc = inc - cnt;
    for (uint32_t r0 = 0; r0 < total; r0 += 32u) {
      const uint32_t r = r0 + uint32_t(lane);
      int j = 0;  // the first lane whose inclusive count exceeds r
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const uint32_t v = __shfl_sync(0xFFFFFFFFu, inc, j + step - 1);
        if (v <= r) j += step;
      }
      const uint32_t ej = __shfl_sync(0xFFFFFFFFu, exc, j), oj = __shfl_sync(0xFFFFFFFFu, off, j);
      if (r < total) {
        const uint32_t k = r - ej, o = oj + k;
        const uint32_t partner = d.bp_stage[size_t(q0 + uint32_t(j)) * BB_BP_STAGE + k];
        if (o < cap) d.pairs[o] = make_uint2(q0 + uint32_t(j), partner);
        else raise_error(d.ctr, BB_ERRF_PAIR_OVERFLOW);
      }
    }
  }
}

// block-wide exclusive scan of one value per thread (blockDim.x == NT)
template <int NT>
__device__ __forceinline__ uint32_t block_scan_nt(uint32_t v, uint32_t* s_warp, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < NT / 32 ? s_warp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < NT / 32) s_warp[lane] = w;
  }
  __syncthreads();
  total = s_warp[NT / 32 - 1];
  uint32_t excl = x - v + (warp > 0 ? s_warp[warp - 1] : 0u);
  __syncthreads();
  return excl;
}
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t& total) {
  return block_scan_nt<BB_FRONTIER>(v, s_warp, total);
}

// One block per heavy query: expand an ordered frontier of overlapping subtrees level by
// level (each level a block scan, so left-to-right order is kept), then every thread walks
// one frontier subtree left-first.  Per-thread counts are scanned so the emitted pairs keep
// ascending partner order.
template <bool EMIT>
__global__ void __launch_bounds__(BB_FRONTIER) k_broad_heavy(const DevState d, uint32_t n, int all) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  __shared__ int s_fr[2][BB_FRONTIER];
  __shared__ uint32_t s_warp[BB_FRONTIER / 32];
  __shared__ uint32_t s_size;
  const uint32_t hc = min(d.ctr->heavy_n, BB_HEAVY_CAP);
  if (blockIdx.x >= hc || (!all && d.hv_n[blockIdx.x] != BB_NONE)) return;  // pool path took this query
  const uint32_t qi = d.heavy_list[blockIdx.x];
  const int N = int(n), leaf0 = N - 1;
  const float4 qmn = d.node_box[2 * (leaf0 + qi)], qmx = d.node_box[2 * (leaf0 + qi) + 1];
  const int wend = world_end(d, qi, n);
  const int t = threadIdx.x;
  if (t == 0) {
    s_fr[0][0] = 0;
    s_size = 1;
  }
  __syncthreads();
  int cur = 0;
  for (int level = 0; level < 64; ++level) {
    const uint32_t size = s_size;
    const int node = t < int(size) ? s_fr[cur][t] : -1;
    int kid[2] = {-1, -1};
    uint32_t c = 0;
    if (node >= leaf0) {
      kid[c++] = node;  // a leaf entry stays in place
    } else if (node >= 0) {
      const Kids k = rec_take(d, node, int(qi), wend, qmn, qmx);
      if (k.tl) kid[c++] = k.l;
      if (k.tr) kid[c++] = k.r;
    }
    uint32_t total;
    const uint32_t pos = block_excl_scan(c, s_warp, total);
    if (total > BB_FRONTIER || total == 0) break;  // uniform: keep the current frontier
    bool internal = false;
    for (uint32_t k = 0; k < c; ++k) {
      s_fr[cur ^ 1][pos + k] = kid[k];
      internal |= kid[k] < leaf0;
    }
    const int more = __syncthreads_or(internal);
    cur ^= 1;
    if (t == 0) s_size = total;
    __syncthreads();
    if (!more) break;
  }
  const uint32_t size = s_size;
  // count (and emit) the leaves under frontier entry t, left-first
  const int root = t < int(size) ? s_fr[cur][t] : -1;
  uint32_t count = 0;
  uint32_t out = 0;
  for (int pass = EMIT ? 0 : 1; pass < 2; ++pass) {
    // EMIT: pass 0 counts (for the scan), pass 1 writes
    uint32_t cnt = 0;
    if (root >= 0) {
      walk_query(d, root, leaf0, int(qi), wend, qmn, qmx, 0xFFFFFFFFu, [&](uint32_t j) {
        if (EMIT && pass == 1) {
          const uint32_t k = out + cnt;
          if (k < d.pair_capacity) d.pairs[k] = make_uint2(qi, j);
          else raise_error(d.ctr, BB_ERRF_PAIR_OVERFLOW);
        }
        ++cnt;
      });
    }
    count = cnt;
    if (EMIT && pass == 0) {
      uint32_t total;
      out = d.pair_off[qi] + block_excl_scan(cnt, s_warp, total);
    }
  }
  if (!EMIT) {
    uint32_t total;
    block_excl_scan(count, s_warp, total);
    if (t == 0) d.pair_cnt[qi] = total;
  }
}

// ---- heavy queries over the whole GPU -------------------------------------------------------
// A query with a huge box (floor, walls) can overlap a large share of all leaves.  One block
// per heavy query expands an ordered frontier of overlapping subtrees, up to BB_HV_FRONTIER
// entries, and appends it to a pool; then every pool entry is walked by its own thread (count,
// scan over the pool, walk again to emit), so one query's walk is spread over the GPU.  The
// frontier keeps left-to-right order and each entry covers a contiguous leaf range, so the
// concatenated walks emit ascending partners, as the single-thread traversal does.  A query
// whose frontier does not fit the pool, or whose world or remaining frontier covers few leaves,
// goes to k_broad_heavy (hv_n = BB_NONE).
// Thread t holds frontier entries [4t, 4t+4); the loads of all four (child, then child range
// and box) are issued together, so a level costs a few load latencies whatever its size.
#define BB_HV_THREADS 1024
#define BB_HV_PER_THREAD 4
// Queries whose world (or remaining frontier) covers at most this many leaves go to the block
// traversal k_broad_heavy: its 256-entry frontier then leaves at most 512 leaves per walk.
#define BB_HV_BLOCK_LEAVES (512u * BB_FRONTIER)
#define BB_HV_FRONTIER (BB_HV_THREADS * BB_HV_PER_THREAD)
// With at most BB_FLAT_MAX heavy queries (a floor and a few walls) the flat pass below answers
// them all; their slots read hv_n = BB_HV_FLAT and the pool and block paths leave them alone.
#define BB_FLAT_MAX 4u
#define BB_HV_FLAT 0xFFFFFFFEu

__global__ void __launch_bounds__(BB_HV_THREADS) k_heavy_frontier(const DevState d, uint32_t n) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  __shared__ int s_fr[2][BB_HV_FRONTIER];
  __shared__ uint32_t s_warp[BB_HV_THREADS / 32];
  __shared__ uint32_t s_size, s_off, s_fits;
  const uint32_t hc = min(d.ctr->heavy_n, BB_HEAVY_CAP);
  const int N = int(n), leaf0 = N - 1;
  const int t = threadIdx.x;
  for (uint32_t slot = blockIdx.x; slot < hc; slot += gridDim.x) {
    if (d.ctr->heavy_n <= BB_FLAT_MAX) {  // few heavy queries: the flat pass takes them
      if (t == 0) d.hv_n[slot] = BB_HV_FLAT;
      __syncthreads();
      continue;
    }
    const uint32_t qi = d.heavy_list[slot];
    const float4 qmn = d.node_box[2 * (leaf0 + qi)], qmx = d.node_box[2 * (leaf0 + qi) + 1];
    const int wend = world_end(d, qi, n);
    const int wbeg = d.n_worlds > 1 ? int(d.world_first[d.sworld[qi]]) : 0;
    if (uint32_t(wend - wbeg) <= BB_HV_BLOCK_LEAVES) {  // a world this small: block traversal
      if (t == 0) d.hv_n[slot] = BB_NONE;
      __syncthreads();
      continue;
    }
    if (t == 0) {
      s_fr[0][0] = 0;
      s_size = 1;
    }
    __syncthreads();
    int cur = 0;
    bool block_path = false;
    for (int level = 0; level < 64; ++level) {
      const uint32_t size = s_size;
      int node[BB_HV_PER_THREAD];
      int2 ch[BB_HV_PER_THREAD];
#pragma unroll
      for (int e = 0; e < BB_HV_PER_THREAD; ++e) {
        const uint32_t idx = uint32_t(t) * BB_HV_PER_THREAD + e;
        node[e] = idx < size ? s_fr[cur][idx] : -1;
      }
      // take test of both children of every internal entry (one record load each, issued
      // together); leaves stay in place
      bool tk[2 * BB_HV_PER_THREAD];
      uint32_t span[2 * BB_HV_PER_THREAD];
      uint32_t c = 0;
#pragma unroll
      for (int e = 0; e < BB_HV_PER_THREAD; ++e) {
        tk[2 * e] = tk[2 * e + 1] = false;
        span[2 * e] = span[2 * e + 1] = 0;
        ch[e] = make_int2(-1, -1);
        if (node[e] < 0 || node[e] >= leaf0) continue;
        const Kids k = rec_take(d, node[e], int(qi), wend, qmn, qmx);
        ch[e] = make_int2(k.l, k.r);
        tk[2 * e] = k.tl;
        tk[2 * e + 1] = k.tr;
        span[2 * e] = k.l >= leaf0 ? 0u : uint32_t(k.lspan);
        span[2 * e + 1] = k.r >= leaf0 ? 0u : uint32_t(k.rspan);
      }
#pragma unroll
      for (int e = 0; e < BB_HV_PER_THREAD; ++e) c += node[e] >= leaf0 ? 1u : uint32_t(tk[2 * e]) + uint32_t(tk[2 * e + 1]);
      uint32_t total;
      uint32_t pos = block_scan_nt<BB_HV_THREADS>(c, s_warp, total);
      if (total > BB_HV_FRONTIER || total == 0) {  // uniform: keep the current frontier (or none)
        if (total == 0 && t == 0) s_size = 0;
        __syncthreads();
        break;
      }
      uint32_t work = 0;  // leaves under this thread's new internal entries
      bool internal = false;
#pragma unroll
      for (int e = 0; e < BB_HV_PER_THREAD; ++e) {
        if (node[e] >= leaf0) {
          s_fr[cur ^ 1][pos++] = node[e];
          continue;
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          if (!tk[2 * e + h]) continue;
          const int k = h ? ch[e].y : ch[e].x;
          s_fr[cur ^ 1][pos++] = k;
          if (k < leaf0) {
            internal = true;
            work += span[2 * e + h];
          }
        }
      }
      const int more = __syncthreads_or(internal);
      cur ^= 1;
      if (t == 0) s_size = total;
      uint32_t total_work;
      block_scan_nt<BB_HV_THREADS>(work, s_warp, total_work);  // ends with a CTA barrier
      // stop expanding once the entries are leaves or each entry's walk is short (32 leaves
      // under an entry on average), whatever the frontier's width: a thin overlap set (a wall)
      // then stops after about log2(N / 32) levels instead of descending the whole tree one
      // block-wide level at a time
      if (!more || total_work <= 32u * total) break;
      // few leaves left under the frontier: a block traversal (k_broad_heavy) costs less than
      // more levels here plus a pool walk; the pool is for queries over very many leaves
      if (total_work <= BB_HV_BLOCK_LEAVES) {
        block_path = true;
        break;
      }
    }
    if (block_path) {
      if (t == 0) d.hv_n[slot] = BB_NONE;
      __syncthreads();
      continue;
    }
    const uint32_t size = s_size;
    if (t == 0) {
      const uint32_t off = size ? atomicAdd(&d.ctr->hv_pool_n, size) : 0u;
      const bool fits = uint64_t(off) + size <= d.hv_cap;
      s_off = off;
      s_fits = fits ? 1u : 0u;
      d.hv_first[slot] = fits ? off : 0u;
      d.hv_n[slot] = fits ? size : BB_NONE;
    }
    __syncthreads();
    const uint32_t off = s_off;
    if (s_fits) {
      for (uint32_t k = t; k < size; k += blockDim.x) {
        d.hv_pool[off + k] = uint32_t(s_fr[cur][k]);
        d.hv_slot[off + k] = slot;
      }
    } else {  // the reservation ran past the pool: mark the part of it inside the pool unused
      for (uint32_t k = t; k < size && uint64_t(off) + k < d.hv_cap; k += blockDim.x) d.hv_slot[off + k] = BB_NONE;
    }
    __syncthreads();
  }
}

// EMIT=false: partners under each pool entry; EMIT=true: write them
template <bool EMIT>
__global__ void k_heavy_walk(const DevState d, uint32_t n) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  const uint32_t E = min(d.ctr->hv_pool_n, d.hv_cap);
  const int N = int(n), leaf0 = N - 1;
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
    const uint32_t slot = d.hv_slot[e];
    if (slot == BB_NONE || d.hv_n[slot] == BB_NONE) {  // the slot's reservation failed (fallback path)
      if (!EMIT) d.hv_cnt[e] = 0;
      continue;
    }
    const uint32_t qi = d.heavy_list[slot];
    const float4 qmn = d.node_box[2 * (leaf0 + qi)], qmx = d.node_box[2 * (leaf0 + qi) + 1];
    const int wend = world_end(d, qi, n);
    uint32_t out = 0;
    if (EMIT) out = d.pair_off[qi] + d.hv_off[e] - d.hv_off[d.hv_first[slot]];
    uint32_t cnt = 0;
    walk_query(d, int(d.hv_pool[e]), leaf0, int(qi), wend, qmn, qmx, 0xFFFFFFFFu, [&](uint32_t j) {
      if (EMIT) {
        const uint32_t k = out + cnt;
        if (k < d.pair_capacity) d.pairs[k] = make_uint2(qi, j);
        else raise_error(d.ctr, BB_ERRF_PAIR_OVERFLOW);
      }
      ++cnt;
    });
    if (!EMIT) d.hv_cnt[e] = cnt;
  }
}

// pair count of every heavy query with a pool frontier
__global__ void k_heavy_totals(const DevState d) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  const uint32_t hc = min(d.ctr->heavy_n, BB_HEAVY_CAP);
  for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < hc; slot += gridDim.x * blockDim.x) {
    const uint32_t m = d.hv_n[slot];
    if (m == BB_NONE || m == BB_HV_FLAT) continue;
    const uint32_t f = d.hv_first[slot];
    d.pair_cnt[d.heavy_list[slot]] = m ? d.hv_off[f + m - 1] + d.hv_cnt[f + m - 1] - d.hv_off[f] : 0u;
  }
}

// ---- a few heavy queries: one flat pass over the leaves ------------------------------------------
// With at most BB_FLAT_MAX heavy queries, each is answered by testing every leaf j of its range
// (qi, world end) against the query box.  That is the traversal's answer: every internal box is
// the exact min/max union of its children's, so no ancestor of an overlapping leaf is pruned
// (only a non-finite box could make the two differ), and ascending j is the traversal's order.
// Block b takes tiles of BB_FLAT_TILE leaves, thread t leaves j0 + k * BB_FLAT_THREADS + t, so
// the reads coalesce and leaf order is (k, warp, lane).  EMIT=false counts per (query, tile)
// into flat_cnt; k_heavy_flat_scan turns the counts into offsets and the query's pair count;
// EMIT=true runs the same tests and writes the pairs.  One read of every leaf box per query
// replaces the pool's frontier levels and walks, which for a floor cover most of the world.
#define BB_FLAT_THREADS 256
#define BB_FLAT_PER 8
#define BB_FLAT_TILE (BB_FLAT_THREADS * BB_FLAT_PER)
template <bool EMIT>
__global__ void __launch_bounds__(BB_FLAT_THREADS) k_heavy_flat(const DevState d, uint32_t n) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  const uint32_t hc = d.ctr->heavy_n;
  if (hc == 0 || hc > BB_FLAT_MAX) return;
  __shared__ uint32_t s_cnt[BB_FLAT_PER][BB_FLAT_THREADS / 32];
  const int leaf0 = int(n) - 1;
  const uint32_t tiles = (n + BB_FLAT_TILE - 1) / BB_FLAT_TILE;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t h = 0; h < hc; ++h) {
    const uint32_t qi = d.heavy_list[h];
    const float4 qmn = d.node_box[2 * (leaf0 + qi)], qmx = d.node_box[2 * (leaf0 + qi) + 1];
    const uint32_t wend = uint32_t(world_end(d, qi, n));
    const uint32_t out = EMIT ? d.pair_off[qi] : 0u;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {  // block-uniform
      const uint32_t j0 = tile * BB_FLAT_TILE;
      if (j0 + BB_FLAT_TILE <= qi + 1u || j0 >= wend) {  // no leaf of the tile in (qi, wend)
        if (!EMIT && threadIdx.x == 0) d.flat_cnt[h * tiles + tile] = 0;
        continue;
      }
      bool f[BB_FLAT_PER];
#pragma unroll
      for (int k = 0; k < BB_FLAT_PER; ++k) {
        const uint32_t j = j0 + uint32_t(k) * BB_FLAT_THREADS + threadIdx.x;
        f[k] = false;
        if (j > qi && j < wend)
          f[k] = box_overlap(qmn, qmx, d.node_box[2 * (leaf0 + j)], d.node_box[2 * (leaf0 + j) + 1]);
      }
      unsigned m[BB_FLAT_PER];
#pragma unroll
      for (int k = 0; k < BB_FLAT_PER; ++k) {
        m[k] = __ballot_sync(0xFFFFFFFFu, f[k]);
        if (lane == 0) s_cnt[k][warp] = uint32_t(__popc(m[k]));
      }
      __syncthreads();
      if (threadIdx.x == 0) {  // exclusive prefix in leaf order (k, then warp); the tile's count
        uint32_t run = 0;
        for (int k = 0; k < BB_FLAT_PER; ++k)
          for (int w = 0; w < BB_FLAT_THREADS / 32; ++w) {
            const uint32_t c = s_cnt[k][w];
            s_cnt[k][w] = run;
            run += c;
          }
        if (!EMIT) d.flat_cnt[h * tiles + tile] = run;
      }
      __syncthreads();
      if (EMIT) {
        const uint32_t base = out + d.flat_off[h * tiles + tile];
#pragma unroll
        for (int k = 0; k < BB_FLAT_PER; ++k) {
          if (!f[k]) continue;
          const uint32_t j = j0 + uint32_t(k) * BB_FLAT_THREADS + threadIdx.x;
          const uint32_t o = base + s_cnt[k][warp] + uint32_t(__popc(m[k] & ((1u << lane) - 1u)));
          if (o < d.pair_capacity) d.pairs[o] = make_uint2(qi, j);
          else raise_error(d.ctr, BB_ERRF_PAIR_OVERFLOW);
        }
      }
      __syncthreads();  // s_cnt is rewritten by the next tile
    }
  }
}
// block h: exclusive scan of query h's tile counts into flat_off, and its pair count
__global__ void __launch_bounds__(1024) k_heavy_flat_scan(const DevState d, uint32_t n) {
  if (d.ctr->front_skip) return;  // nothing moved since the last front end
  const uint32_t hc = d.ctr->heavy_n;
  if (hc == 0 || hc > BB_FLAT_MAX || blockIdx.x >= hc) return;
  __shared__ uint32_t s_warp[32];
  const uint32_t tiles = (n + BB_FLAT_TILE - 1) / BB_FLAT_TILE, h = blockIdx.x;
  uint32_t carry = 0;
  for (uint32_t b = 0; b < tiles; b += blockDim.x) {  // block-uniform
    const uint32_t i = b + threadIdx.x;
    const uint32_t v = i < tiles ? d.flat_cnt[h * tiles + i] : 0u;
    uint32_t total;
    const uint32_t ex = block_scan_nt<1024>(v, s_warp, total);
    if (i < tiles) d.flat_off[h * tiles + i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) d.pair_cnt[d.heavy_list[h]] = carry;
}

void bb_front_end(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, const StepScratch& sc, int sms,
                  int cur, uint32_t max_world_bodies, cudaEvent_t* marks) {
  (void)cur;
  if (n == 0) return;
  const int T = BB_THREADS;
  uint32_t blocks = (n + T - 1) / T;
  if (p.bounds_mode == BB_BOUNDS_AUTO) k_bounds<<<blocks, T, 0, s>>>(d, n);
  k_morton<<<blocks, T, 0, s>>>(d, n, p);
  if (marks) cudaEventRecord(marks[0], s);
  uint32_t* keys[2] = {d.keys[0], d.keys[1]};
  uint32_t* vals[2] = {d.vals[0], d.vals[1]};
  if (d.n_worlds > 1) {
    // stable sort by code, then by world id (two digits of world_of[id]): key order (world, code)
    bb_launch_sort(s, keys, vals, &d.ctr->front_n, n, 4, 0, sc.sort_hist, sc.sort_status, sc.sort_tile_ctr, d.ctr,
                   sms, d.world_of, 2);
    k_sorted_world<<<blocks, T, 0, s>>>(d, n);
  } else {
    bb_launch_sort(s, keys, vals, &d.ctr->front_n, n, 4, 0, sc.sort_hist, sc.sort_status, sc.sort_tile_ctr, d.ctr, sms);
  }
  if (marks) cudaEventRecord(marks[1], s);
  k_build<<<blocks, T, 0, s>>>(d, n);
  if (marks) cudaEventRecord(marks[2], s);
  k_refit<<<blocks, T, 0, s>>>(d, n);
  if (marks) cudaEventRecord(marks[3], s);
  const uint32_t bt = p.broad_threads ? p.broad_threads : 128u;
  uint32_t bb = (n + bt - 1) / bt;
  uint32_t hb = min(n, BB_HEAVY_CAP);
  k_broad<false><<<bb, bt, 0, s>>>(d, n);
  // The frontier pool is for worlds over BB_HV_BLOCK_LEAVES bodies; when no world is that large
  // every heavy query takes the block traversal and the pool kernels are not launched at all
  // (their GPU-wide 1024-thread blocks would only stall other streams' work).
  const bool pool = max_world_bodies > BB_HV_BLOCK_LEAVES;
  if (pool) {
    // two co-resident 1024-thread blocks per SM loop over the heavy slots
    k_heavy_frontier<<<min(hb, 2u * uint32_t(sms)), BB_HV_THREADS, 0, s>>>(d, n);
    k_heavy_walk<false><<<sms * 8, 128, 0, s>>>(d, n);
    bb_launch_scan(s, d.hv_cnt, d.hv_off, &d.ctr->hv_pool_n, d.hv_cap, nullptr,
                   sc.scan_status + 5 * size_t(sc.scan_tiles), sc.scan_tile_ctr + 5, d.ctr, &d.ctr->front_skip);
    k_heavy_totals<<<(hb + 255) / 256, 256, 0, s>>>(d);
    k_heavy_flat<false><<<min((n + BB_FLAT_TILE - 1) / BB_FLAT_TILE, uint32_t(sms) * 8u), BB_FLAT_THREADS, 0, s>>>(d, n);
    k_heavy_flat_scan<<<BB_FLAT_MAX, 1024, 0, s>>>(d, n);
  }
  k_broad_heavy<false><<<hb, BB_FRONTIER, 0, s>>>(d, n, pool ? 0 : 1);
  bb_launch_scan(s, d.pair_cnt, d.pair_off, nullptr, n, &d.ctr->pair_count, sc.scan_status, sc.scan_tile_ctr, d.ctr,
                 &d.ctr->front_skip);
  k_broad_copy<<<sms * 16, 256, 0, s>>>(d, n);
  k_broad<true><<<bb, bt, 0, s>>>(d, n);
  k_broad_heavy<true><<<hb, BB_FRONTIER, 0, s>>>(d, n, pool ? 0 : 1);
  if (pool) {
    k_heavy_walk<true><<<sms * 8, 128, 0, s>>>(d, n);
    k_heavy_flat<true><<<min((n + BB_FLAT_TILE - 1) / BB_FLAT_TILE, uint32_t(sms) * 8u), BB_FLAT_THREADS, 0, s>>>(d, n);
  }
}
