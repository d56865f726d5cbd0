// bb_common.cuh -- shared device definitions of the B200 rigid-body step.
//
// Layout (all arrays in HBM, indexed by body id unless noted):
//   pos      float4  position.xyz, inverse mass
//   rot      float4  quaternion x y z w
//   vel      float4  linear velocity.xyz, mass
//   omega    float4  angular velocity.xyz, 0
//   pvel     float4  previous-step velocity (AVBD adaptive warm start)
//   shape    float4  half extents (sphere: radius in x), w = shape type bits
//   iinv     float4  body-frame inverse inertia diagonal.xyz, friction
//   flags    u32     BB_BODY_* ; sleep u32 timer (bit 31 = partner veto)
// Manifolds live in pair slots (one slot per broad-phase pair); slot p owns contact rows
// 8p .. 8p+7.  A compact list man_slot[m] (pair order) names the slots that collided.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/beatbox.h"

#define BB_MAX_CONTACTS 8
#define BB_MAX_COLORS 32
#define BB_UNCOLORED BB_EDGE_COLOR_OVERFLOW
#define BB_RESTING BB_EDGE_COLOR_RESTING  // a manifold whose island has no awake body (not coloured)
#define BB_NONE 0xFFFFFFFFu
#define BB_SLEEP_VETO 0x80000000u
#define BB_SLEEP_MASK 0x7FFFFFFFu
#define BB_SPIN_LIMIT (1u << 22)
#define BB_BODY_PAUSE_AWAKE (1u << 6)  // a paused body that was awake when its world was paused
#define BB_BVH_STACK 64

#define BB_KEY_SPHERE_SPHERE 20
#define BB_KEY_BOX_SPHERE 21
#define BB_KEY_SPHERE_BOX 22

// ---- device counters (one struct per world, zeroed per substep where noted) ---------
struct DevCounters {
  uint32_t n_bodies;       // host-set
  uint32_t n_dynamic;      // host-set
  uint32_t pair_count;     // broad phase output (per substep)
  uint32_t manifold_count; // per substep
  uint32_t contact_count;
  uint32_t fresh;
  uint32_t max_pen_bits;   // float bits of the deepest penetration (positive)
  uint32_t island_count;
  uint32_t sleeping;
  uint32_t gc_colors;
  uint32_t gc_overflow;
  uint32_t gc_violations;
  uint32_t gc_rounds_run;  // colouring rounds the last edge colouring ran
  uint32_t avbd_colors;
  uint32_t avbd_violations;
  uint32_t stick;
  uint32_t error_flags;    // sticky until read
  uint32_t gc_epoch;       // colouring round epoch (never reset)
  uint32_t barrier_count;  // grid barrier
  uint32_t barrier_gen;
  uint32_t bounds_min[3];  // BB_BOUNDS_AUTO: ordered-float min/max of positions
  uint32_t bounds_max[3];
  uint32_t avbd_body_count;
  uint32_t substeps;       // substeps run since the world was created
  uint32_t wait_limit;     // polls before a bounded device wait gives up (0 = BB_SPIN_LIMIT)
  uint32_t abandon_block;  // test switch: the PGS solver's last block leaves before its first barrier
  uint32_t pgs_manifolds;  // per substep: colour-sweep items with an awake body (solved manifolds)
  uint32_t pgs_contacts;   // their contacts
  uint32_t round_flags[2]; // per-round flags / counters: components' "changed", then the AVBD colouring's uncoloured counts
  uint32_t heavy_n;        // broad phase: heavy queries of this substep
  uint32_t error_site;     // where the first bounded wait gave up (bb_step_stats.error_site)
  uint32_t prev_manifolds; // manifold count of the last substep (its buffer is the previous one)
  uint32_t gc_coloured;    // substep number of the last edge colouring (0: none to reuse)
  uint32_t sync_count[8];  // grid_sync arrival counters, one per persistent launch of a substep
                           // (zeroed at substep start): 0 edge colouring, 1 PGS, 2.. AVBD,
                           // 7 connected components
  uint32_t np_counts[4];   // narrow-phase work lists: box-box, with a sphere, voxel pairs, carried
  uint32_t gc_list_n[2];   // edge colouring: sizes of the alternating uncoloured-manifold lists
  uint32_t hv_pool_n;      // broad phase: frontier entries of the heavy queries
  uint32_t slot_count;     // worlds with voxel shapes: manifold slots (6 per voxel pair, else 1)
  uint32_t slots_of[2];    // manifold slots of the narrow phase that last wrote contact buffer 0 / 1
  // Front-end skip: when no body was awake after the last substep's sleep stage, nothing was
  // integrated, so every pose (and the sort, tree and pair list built from them) is as the last
  // front end left it.  front_valid is cleared by every host-side change of bodies, poses or
  // parameters; front_n is the front-end sort's key count (0 when skipped, else all).
  uint32_t front_skip, front_valid, front_n, sleep_ran, awake_after;
};

// Voxel shape on the device (VoxelShape, include/shared.inl:938-951) with the body-frame box
// RigidBody::minimum = origin, maximum = hi precomputed on the host.
struct VoxDev {
  float ox, oy, oz, vs;   // grid origin (corner of cell 0), cell size
  float hx, hy, hz;       // grid box maximum
  uint32_t surf_count;
  uint32_t dx, dy, dz;    // cells per axis
  uint32_t occ_off;       // first word of the occupancy bits in vox_occ
  uint32_t surf_off;      // first entry of the surface list in vox_surf
  uint32_t pad[3];
};
#define BB_SHAPE_KIND(t) ((t) & 0xFFu)
#define BB_SHAPE_VOXEL_INDEX(t) ((t) >> 8)

// ---- pointers of one world's device state ------------------------------------------------
struct DevState {
  // bodies
  float4 *pos, *rot, *vel, *omega, *pvel, *shape, *iinv;
  uint32_t *flags, *sleep;
  float4* iw;  // world inverse inertia cache: 2 float4 per body (xx xy xz yy | yz zz - -)
  // front end
  uint32_t *keys[2], *vals[2];  // vals[0] holds the sorted ids (= next substep's order)
  uint32_t* rank;               // body id -> sorted position
  float4* node_box;             // 2 float4 per node (min, max); internal 0..N-2, leaves N-1..
  float4* node_rec;             // 5 float4 per internal node: both children's boxes, indices, leaf ranges
  int2* child;                  // internal node children
  int32_t* parent;              // parent of every node (root: -1)
  int32_t* range_last;          // last leaf covered by each internal node
  uint32_t* visit;              // refit arrival counters
  uint32_t *pair_cnt, *pair_off;  // per query
  uint32_t *is_heavy, *heavy_list;  // 1: over the visit budget (block-cooperative), 2: staging spilled
  uint32_t* bp_stage;           // first 32 partners of each query (counting traversal)
  // heavy queries split over the whole GPU: per slot its frontier range in the pool; per pool
  // entry the subtree root, the slot, the partner count and its exclusive scan
  uint32_t *hv_first, *hv_n, *hv_pool, *hv_slot, *hv_cnt, *hv_off;
  uint32_t *flat_cnt, *flat_off;  // flat pass of a few heavy queries: per (query, leaf tile) counts, offsets
  uint32_t hv_cap;              // pool entries
  uint2* pairs;                 // (sorted a, sorted b)
  uint32_t* np_list;            // narrow-phase work list (pair indices; see k_np_classify)
  // manifolds (two buffers: [cur], [prev] chosen by parity)
  uint2* m_bodies[2];    // body ids (a, b) per slot
  int2* m_keycc[2];      // key, contact count per slot
  float4* m_normal[2];   // normal.xyz, error (int bits)
  float4* m_t0[2];
  float4* m_t1[2];
  float4* m_anchor_a[2]; // body positions at narrow-phase time
  float4* m_anchor_b[2];
  uint32_t* man_slot[2]; // compact manifold -> slot
  uint32_t* man_count_prev; // not used (count kept in counters)
  // contacts (8 per slot)
  float4* c_pos[2];      // position.xyz, penetration
  float4* c_lam[2];      // normal impulse / lambda, tangent impulse 0/1, AVBD normal penalty k
  float4* c_kt[2];       // AVBD tangent penalties 0/1, stick (bits), warm-start count (bits)
  float4* c_anc_a[2];    // AVBD local anchor on a .xyz, feature pair (bits)
  float4* c_anc_b[2];    // AVBD local anchor on b .xyz, 0
  // PGS rows (current only)
  float4 *c_r1, *c_r2, *c_k;
  // dataflow schedule: per compact manifold (slot, a, b, rank_a | rank_b << 16); per-body counters
  uint4* flow_rec;
  uint32_t* flow_counter;
  // barrier schedule: colour-ordered items, rec = (slot, a, b, cc | dyn_a << 8 | dyn_b << 9 |
  // skip << 10), mass = (inverse mass a, inverse mass b, friction, -)
  uint4* pgs_rec;
  float4* pgs_mass;
  float4* pgs_frame;   // 3 per item: normal, tangent 0, tangent 1
  float4* pgs_lam;     // compact impulses, pgs_coff[k] + j
  uint32_t *pgs_cnt, *pgs_coff, *pgs_slot;
  // per-body manifold lists (CSR over compact manifold indices) [cur], [prev]
  uint32_t* csr_start[2];
  uint32_t* csr_list[2];
  uint32_t* csr_partner[2];  // other body of each list entry
  uint32_t* csr_slot[2];     // slot of each list entry's manifold
  uint32_t* csr_cursor;
  uint32_t* hit;         // per pair slot: 1 if it produced a manifold
  uint32_t* man_index;   // per pair slot: exclusive scan of hit
  // islands
  uint32_t *uf_parent, *is_root, *root_rank, *island;
  uint32_t* cc_mark;       // per body id: substep number when its old component must start over
  uint32_t* island_start;  // per-island path: first sorted manifold of each island
  // colouring
  uint32_t* gc_color;    // per compact manifold
  uint32_t* gc_pid;      // pair-identity hash
  uint32_t* gc_choice;
  uint4* gc_rec;         // per compact manifold: body a, body b, pair hash, static bits
  uint32_t* gc_list[2];  // manifolds still uncoloured after a round (alternating)
  uint32_t* gc_mask;     // per body
  uint32_t* gc_island_tag; // per island: colouring epoch + 1 when one of its bodies is awake
  unsigned long long* gc_owner; // 32 colours x (body capacity + 1) bodies: (epoch << 32) | priority
  uint32_t *bucket_keys[2], *bucket_vals[2]; // colour sort of manifolds / bodies
  uint32_t* bucket_start; // 34 + 32*L entries
  uint32_t* colour_awake; // per colour (32 = overflow): 1 if one of its manifolds has an awake body
  // colour reuse: an island whose manifolds (bodies and key) are exactly last substep's keeps
  // last substep's colours (the colouring of an island depends on that set alone)
  uint32_t* gc_slot_color[2]; // per manifold slot of each buffer: the colour the colouring gave it
  uint32_t* gc_reuse;      // per slot of this substep: the colour of the same manifold last substep, or BB_NONE
  uint32_t* gc_survived;   // per slot of the previous buffer: substep number when a manifold took it over
  uint32_t* gc_body_chg;   // per body: substep number when one of its manifolds of last substep ended
  uint32_t* gc_island_chg; // per island: colouring epoch + 1 when it must be coloured afresh
  // AVBD
  uint32_t* body_color;   // per body
  uint32_t* body_color_round;
  float4 *a_pos_start, *a_rot_start, *a_pos_tilde, *a_rot_tilde;
  uint32_t* a_depth;
  uint32_t *a_bucket_keys[2], *a_bucket_vals[2];
  uint32_t* a_bucket_start;
  // scan / sort scratch
  uint32_t* scan_status;  // decoupled look-back status words
  uint32_t* scan_tile_ctr;
  uint32_t* sort_hist;    // 4 x 256 global digit histograms
  uint32_t* sort_status;  // tiles x 256 per pass
  uint32_t* sort_tile_ctr;
  // batched worlds (n_worlds > 1): world w owns body ids [world_first[w], +world_count[w]),
  // which is also its range of sorted positions (keys sort by (world, Morton code))
  uint32_t n_worlds;
  uint32_t* world_of;     // per body
  uint32_t* world_first;  // per world
  uint32_t* world_count;  // per world
  float4* world_bounds;   // per world: (min.xyz, -), (extent.xyz, -)
  uint32_t* sworld;       // world of each sorted position
  int32_t* range_first;   // first leaf covered by each internal node
  DevCounters* ctr;
  float* staging;  // host state exchange: rot 4N | pos 3N | vel 3N | omega 3N
  uint32_t pair_capacity;
  uint32_t body_capacity;
  // voxel bodies (shape.w = BB_SHAPE_VOXEL | index << 8) and full inverse inertia
  const VoxDev* vox;
  const uint32_t* vox_occ;
  const uint32_t* vox_surf;
  uint32_t vox_on;         // the world has voxel shapes: slots are expanded per pair
  uint32_t full_inertia;   // some body has a non-zero off-diagonal in iinv_off
  uint32_t* slot_cnt;      // per pair: manifold slots (vox_on)
  uint32_t* slot_off;      // per pair: first slot
  uint32_t* slot_pair;     // per slot: pair << 3 | face code
  uint32_t* vox_list;      // narrow-phase work list of the voxel slots
  float4* iinv_off;        // per body: body-frame inverse inertia off-diagonal (xy, xz, yz, -)
  uint32_t* frozen;        // per body: 1 if asleep or static at the last narrow phase, state unwritten since
  uint32_t* carry_list;    // narrow-phase work list of the frozen pairs: slot | paused << 31
  uint2* carry_ids;        // the two bodies of each carry_list entry
  uint32_t* carry_tag;     // per slot: the substep that last carried it in place (short carry)
};

// ---- small vector helpers -------------------------------------------------------------------
__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float4 f4(float3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float comp(float3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__device__ __forceinline__ void set_comp(float3& a, int i, float v) {
  if (i == 0) a.x = v;
  else if (i == 1) a.y = v;
  else a.z = v;
}

struct Quatf {
  float x, y, z, w;
};
__device__ __forceinline__ Quatf q_from(float4 a) { return Quatf{a.x, a.y, a.z, a.w}; }
__device__ __forceinline__ float4 q_to4(Quatf q) { return make_float4(q.x, q.y, q.z, q.w); }
__device__ __forceinline__ Quatf q_conj(Quatf q) { return Quatf{-q.x, -q.y, -q.z, q.w}; }
// Hamilton product (include/math.hpp:357-364), contraction allowed.
__device__ __forceinline__ Quatf q_mul(Quatf a, Quatf b) {
  return Quatf{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
               a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
__device__ __forceinline__ Quatf q_normalize(Quatf q) {
  float m = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  return Quatf{q.x / m, q.y / m, q.z / m, q.w / m};
}
__device__ __forceinline__ float3 q_rotate(Quatf q, float3 v) {  // q v q*
  Quatf r = q_mul(q_mul(q, Quatf{v.x, v.y, v.z, 0.f}), q_conj(q));
  return make_float3(r.x, r.y, r.z);
}
__device__ __forceinline__ float3 q_rotate_inv(Quatf q, float3 v) {  // q* v q
  Quatf r = q_mul(q_mul(q_conj(q), Quatf{v.x, v.y, v.z, 0.f}), q);
  return make_float3(r.x, r.y, r.z);
}

// Exact (no contraction) Hamilton product for the bit-exact AABB path: the reference order
// ((a + b) + c) - d with every product rounded separately.
__device__ __forceinline__ float ex4(float a1, float b1, float a2, float b2, float a3, float b3, float a4, float b4) {
  return __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(a1, b1), __fmul_rn(a2, b2)), __fmul_rn(a3, b3)), __fmul_rn(a4, b4));
}
__device__ __forceinline__ Quatf q_mul_exact(Quatf a, Quatf b) {
  Quatf r;
  r.x = ex4(a.w, b.x, a.x, b.w, a.y, b.z, a.z, b.y);
  r.y = ex4(a.w, b.y, a.y, b.w, a.z, b.x, a.x, b.z);
  r.z = ex4(a.w, b.z, a.z, b.w, a.x, b.y, a.y, b.x);
  r.w = __fsub_rn(__fsub_rn(__fsub_rn(__fmul_rn(a.w, b.w), __fmul_rn(a.x, b.x)), __fmul_rn(a.y, b.y)),
                  __fmul_rn(a.z, b.z));
  return r;
}

// 3x3 symmetric helpers: world inverse inertia stored as (xx, xy, xz, yy) (yz, zz).
struct Sym3 {
  float xx, xy, xz, yy, yz, zz;
};
__device__ __forceinline__ float3 sym_mul(const Sym3& s, float3 v) {
  return make_float3(s.xx * v.x + s.xy * v.y + s.xz * v.z, s.xy * v.x + s.yy * v.y + s.yz * v.z,
                     s.xz * v.x + s.yz * v.y + s.zz * v.z);
}
// Rotation matrix rows of to_matrix (include/math.hpp:287-304).
__device__ __forceinline__ void q_matrix(Quatf q, float m[3][3]) {
  float x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
  float xx = q.x * x2, xy = q.x * y2, xz = q.x * z2, yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
  float wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
  m[0][0] = 1.f - (yy + zz); m[0][1] = xy - wz; m[0][2] = xz + wy;
  m[1][0] = xy + wz; m[1][1] = 1.f - (xx + zz); m[1][2] = yz - wx;
  m[2][0] = xz - wy; m[2][1] = yz + wx; m[2][2] = 1.f - (xx + yy);
}
// World inverse inertia from the body-frame diagonal d.  transpose_quirk: R^T D R
// (get_transformed_inertia, extensions.slang:184-188); else R D R^T.
__device__ __forceinline__ Sym3 world_inv_inertia(Quatf q, float3 d, bool transpose_quirk) {
  float R[3][3];
  q_matrix(q, R);
  float M[3][3];  // rows of the matrix S with world = S^T D S
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) M[i][j] = transpose_quirk ? R[i][j] : R[j][i];
  // world[a][b] = sum_k M[k][a] d_k M[k][b]
  float dd[3] = {d.x, d.y, d.z};
  Sym3 s;
  auto e = [&](int a, int b) { return M[0][a] * dd[0] * M[0][b] + M[1][a] * dd[1] * M[1][b] + M[2][a] * dd[2] * M[2][b]; };
  s.xx = e(0, 0); s.xy = e(0, 1); s.xz = e(0, 2); s.yy = e(1, 1); s.yz = e(1, 2); s.zz = e(2, 2);
  return s;
}

// Body with a full symmetric body-frame inverse inertia B (diagonal d, off-diagonal o = xy, xz,
// yz): world = S^T B S with S as above.  Used only for bodies whose o is not zero, so boxes and
// spheres keep the diagonal formula's bits.
__device__ __forceinline__ Sym3 world_inv_inertia_full(Quatf q, float3 d, float3 o, bool transpose_quirk) {
  float R[3][3];
  q_matrix(q, R);
  float M[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) M[i][j] = transpose_quirk ? R[i][j] : R[j][i];
  const float B[3][3] = {{d.x, o.x, o.y}, {o.x, d.y, o.z}, {o.y, o.z, d.z}};
  float T[3][3];  // B * M
  for (int k = 0; k < 3; ++k)
    for (int b = 0; b < 3; ++b) T[k][b] = B[k][0] * M[0][b] + B[k][1] * M[1][b] + B[k][2] * M[2][b];
  auto e = [&](int a, int b) { return M[0][a] * T[0][b] + M[1][a] * T[1][b] + M[2][a] * T[2][b]; };
  Sym3 s;
  s.xx = e(0, 0); s.xy = e(0, 1); s.xz = e(0, 2); s.yy = e(1, 1); s.yz = e(1, 2); s.zz = e(2, 2);
  return s;
}
__device__ __forceinline__ Sym3 body_world_inv_inertia(const float4* iinv, const float4* iinv_off, bool full, uint32_t i,
                                                       Quatf q, bool tq) {
  if (full) {
    const float4 o = iinv_off[i];
    if (o.x != 0.f || o.y != 0.f || o.z != 0.f) return world_inv_inertia_full(q, f3(iinv[i]), f3(o), tq);
  }
  return world_inv_inertia(q, f3(iinv[i]), tq);
}

// Sites of bounded waits, recorded in DevCounters::error_site by the first one that gives up
// (bb_step_stats.error_site): the sort's and the scan's look-backs, the dataflow PGS wait,
// the generation barrier, and BB_SITE_GRID + k for the grid barrier on sync_count[k] (0 edge colouring, 1
// PGS_SOFT, 2 AVBD colouring, 3..5 AVBD solve phases, 7 connected components).
#define BB_SITE_SORT 1u
#define BB_SITE_FLOW 2u
#define BB_SITE_GEN_BARRIER 3u
#define BB_SITE_SCAN 4u
#define BB_SITE_GRID 16u
__device__ __forceinline__ void raise_error(DevCounters* c, uint32_t bit) { atomicOr(&c->error_flags, bit); }
// a bounded wait at `site` (BB_SITE_*) gave up
__device__ __forceinline__ void raise_wait_error(DevCounters* c, uint32_t site) {
  atomicCAS(&c->error_site, 0u, site);
  atomicOr(&c->error_flags, BB_ERRF_SPIN_LIMIT);
}

// id of a body inside its own world (batched worlds hash world-local ids, so a world's
// colouring does not depend on where it sits in the batch)
__device__ __forceinline__ uint32_t local_id(const DevState& d, uint32_t id) {
  return d.n_worlds > 1 ? id - d.world_first[d.world_of[id]] : id;
}

// order-preserving float <-> uint (include/math.hpp:228-256)
__device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t u = __float_as_uint(f);
  uint32_t mask = uint32_t(-int32_t(u >> 31)) | 0x80000000u;
  return u ^ mask;
}
__device__ __forceinline__ float ord2f(uint32_t v) {
  uint32_t mask = ((v >> 31) - 1u) | 0x80000000u;
  return __uint_as_float(v ^ mask);
}

// ---- grid barrier for persistent cooperative kernels ------------------------------------
// Sense by generation counter; the spin is bounded: on timeout the block raises
// BB_ERRF_SPIN_LIMIT and every later barrier returns at once (results are then invalid and
// the host reports BB_E_DEVICE_LIMIT).
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Bound of every grid-barrier wait: checked once per 64 polls (a barrier that completes within
// them never reads it).  Gives up past the world's wait_limit (BB_SPIN_LIMIT when 0), raising
// BB_ERRF_SPIN_LIMIT, or at once when another wait of the launch already gave up.
__device__ __forceinline__ bool spin_gave_up(DevCounters* c, uint32_t spins, uint32_t site) {
  if ((spins & 63u) != 0u) return false;
  const uint32_t lim = *reinterpret_cast<volatile const uint32_t*>(&c->wait_limit);
  if (spins > (lim ? lim : BB_SPIN_LIMIT)) {
    atomicCAS(&c->error_site, 0u, site);
    atomicOr(&c->error_flags, BB_ERRF_SPIN_LIMIT);
    return true;
  }
  return (ld_acquire_gpu(&c->error_flags) & BB_ERRF_SPIN_LIMIT) != 0;
}

__device__ __forceinline__ void grid_barrier(DevCounters* c) {
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t g = ld_acquire_gpu(&c->barrier_gen);
    fence_acq_rel_gpu();  // publish this block's writes (cumulative over the CTA barrier)
    uint32_t arrived = atomicAdd(&c->barrier_count, 1u);
    if (arrived == gridDim.x - 1) {
      c->barrier_count = 0;
      fence_acq_rel_gpu();
      atomicAdd(&c->barrier_gen, 1u);
    } else {
      uint32_t spins = 0;
      while (ld_acquire_gpu(&c->barrier_gen) == g)
        if (spin_gave_up(c, ++spins, BB_SITE_GEN_BARRIER)) break;
    }
    fence_acq_rel_gpu();
  }
  __syncthreads();
}

// Grid barrier on a monotonic arrival counter that is zero when the kernel starts (one counter
// per persistent launch of a substep): block thread 0 publishes the block's writes and adds one
// without waiting for a reply, then polls until all blocks of this epoch arrived.  Two round
// trips fewer than the generation barrier above (no generation read, no atomic reply).
__device__ __forceinline__ void red_relaxed_add(uint32_t* p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void grid_sync(DevCounters* c, uint32_t* count, uint32_t& epoch) {
  __syncthreads();
  ++epoch;
  if (gridDim.x == 1) return;  // one block: the CTA barrier is the grid barrier
  if (threadIdx.x == 0) {
    fence_acq_rel_gpu();  // release this block's writes (cumulative over the CTA barrier)
    red_relaxed_add(count, 1u);
    const uint32_t target = epoch * gridDim.x;
    uint32_t spins = 0;
    while (ld_acquire_gpu(count) < target)
      if (spin_gave_up(c, ++spins, BB_SITE_GRID + uint32_t(count - c->sync_count))) break;
  }
  __syncthreads();
}

// grid_sync split in two: arrive publishes this block's writes and counts it in; wait returns
// once every block of the epoch has arrived.  Work placed between them must neither read what
// other blocks write in this epoch nor write what they read.
__device__ __forceinline__ void grid_arrive(uint32_t* count, uint32_t& epoch) {
  __syncthreads();
  ++epoch;
  if (threadIdx.x == 0 && gridDim.x > 1) {
    fence_acq_rel_gpu();
    red_relaxed_add(count, 1u);
  }
}
__device__ __forceinline__ void grid_wait(DevCounters* c, const uint32_t* count, uint32_t epoch) {
  if (threadIdx.x == 0 && gridDim.x > 1) {
    const uint32_t target = epoch * gridDim.x;
    uint32_t spins = 0;
    while (ld_acquire_gpu(count) < target)
      if (spin_gave_up(c, ++spins, BB_SITE_GRID + uint32_t(count - c->sync_count))) break;
  }
  __syncthreads();
}

// kernel-side solver parameters (a plain copy of bb_solver_params)
typedef bb_solver_params Params;

// ---- host-side launch helpers (defined in bb_world.cu) ----------------------------------
#define BB_THREADS 256
// persistent cooperative kernels: one 512-thread block per SM (fewer barrier participants)
#define BB_COOP_THREADS 512
