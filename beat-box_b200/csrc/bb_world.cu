// bb_world.cu -- the world object behind the C ABI of include/beatbox.h.
//
// Replaces RigidBodyManager (src/rigid_body_manager.{hpp,cpp}): buffer allocation
// (RBM:121-283), the per-step program (RBM:1284-1427, here the substep sequence in
// World::substep) and the SimConfig readback (RBM:1681-1693).  Bodies are added through
// bb_add_bodies, which restates SceneManager::load_scene's id / mass / inertia assignment
// (src/scene_manager.hpp:850-887).
//
// Execution: a step of S substeps is captured once into a CUDA graph keyed by
// (S, buffer parity, warm start, dt, parameters) and replayed; all per-substep counts stay on
// the device.  Persistent solver kernels are launched cooperatively.
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "bb_common.cuh"
#include "bb_kernels.cuh"
#include "bb_voxel_build.hpp"

namespace {
thread_local std::string g_last_error = "no error";
bb_status fail(bb_status code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
#define CU(call)                                                                                       \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess) return fail(BB_E_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

struct Shape {
  uint32_t type;
  float half[3];
  uint32_t vox = 0;          // voxel shapes: index in the world's voxel table
  float unit_mass = 0;       // voxel shapes: mass at density 1
  float unit_inv[6] = {0, 0, 0, 0, 0, 0};  // voxel shapes: inverse inertia at density 1
};

thread_local size_t t_alloc_bytes = 0;  // device bytes allocated by dalloc on this thread
thread_local bool t_count_only = false;  // dalloc only counts (bb_world_bytes_for)

// device arrays of a world with their sizes (a saved state is an image of all of them)
typedef std::vector<std::pair<void*, size_t>> Owned;

template <class T> T* dalloc(size_t n, Owned& owned, cudaError_t& err, cudaStream_t stream) {
  void* p = nullptr;
  if (n == 0) n = 1;
  t_alloc_bytes += n * sizeof(T);
  if (t_count_only) return nullptr;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess) {
    err = e;
    return nullptr;
  }
  cudaMemsetAsync(p, 0, n * sizeof(T), stream);
  owned.emplace_back(p, n * sizeof(T));
  return static_cast<T*>(p);
}

uint64_t fnv(const void* data, size_t bytes, uint64_t h = 1469598103934665603ull) {
  const uint8_t* b = static_cast<const uint8_t*>(data);
  for (size_t i = 0; i < bytes; ++i) h = (h ^ b[i]) * 1099511628211ull;
  return h;
}
}  // namespace

bb_status bb_fail(bb_status code, const char* msg) { return fail(code, msg); }

int bb_coop_blocks(const void* kernel, int threads, int sms) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  if (per_sm < 1) per_sm = 1;
  return sms * std::min(per_sm, 1);
}

cudaError_t bb_launch_coop(const void* kernel, int blocks, int threads, void** args, cudaStream_t s,
                           size_t smem_bytes) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem_bytes;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, kernel, args);
}

// state exchange with the host through one staging buffer: rot 4N | pos 3N | vel 3N | omega 3N
// (rotations first: float4 accesses need the 16-byte-aligned base)
__global__ void k_pack_state(const DevState d, uint32_t n, float* st) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = d.pos[i], q = d.rot[i], v = d.vel[i], w = d.omega[i];
  float* Q = st;
  float* P = st + 4 * size_t(n);
  float* V = st + 7 * size_t(n);
  float* W = st + 10 * size_t(n);
  P[3 * i] = p.x; P[3 * i + 1] = p.y; P[3 * i + 2] = p.z;
  reinterpret_cast<float4*>(Q)[i] = q;
  V[3 * i] = v.x; V[3 * i + 1] = v.y; V[3 * i + 2] = v.z;
  W[3 * i] = w.x; W[3 * i + 1] = w.y; W[3 * i + 2] = w.z;
}
// bodies [o, o + n) into the staging buffer (the k_pack_state layout for n bodies), and their
// flags as the caller sees them: a paused body reads asleep as it was when its world stopped
__global__ void k_pack_range(const DevState d, uint32_t o, uint32_t n, float* st, uint32_t* flags) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t b = o + i;
  float4 p = d.pos[b], q = d.rot[b], v = d.vel[b], w = d.omega[b];
  float* P = st + 4 * size_t(n);
  float* V = st + 7 * size_t(n);
  float* W = st + 10 * size_t(n);
  P[3 * i] = p.x; P[3 * i + 1] = p.y; P[3 * i + 2] = p.z;
  reinterpret_cast<float4*>(st)[i] = q;
  V[3 * i] = v.x; V[3 * i + 1] = v.y; V[3 * i + 2] = v.z;
  W[3 * i] = w.x; W[3 * i + 1] = w.y; W[3 * i + 2] = w.z;
  uint32_t f = d.flags[b];
  if (f & BB_BODY_PAUSED) f = (f & BB_BODY_PAUSE_AWAKE) ? (f & ~BB_BODY_SLEEPING) : f;
  flags[i] = f & (BB_BODY_DYNAMIC | BB_BODY_GRAVITY | BB_BODY_SLEEPING);
}
__global__ void k_unpack_state(const DevState d, uint32_t n, const float* st, uint32_t mask) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* Q = st;
  const float* P = st + 4 * size_t(n);
  const float* V = st + 7 * size_t(n);
  const float* W = st + 10 * size_t(n);
  if (mask & 1) d.pos[i] = make_float4(P[3 * i], P[3 * i + 1], P[3 * i + 2], d.pos[i].w);
  if (mask & 2) d.rot[i] = reinterpret_cast<const float4*>(Q)[i];
  if (mask & 4) d.vel[i] = make_float4(V[3 * i], V[3 * i + 1], V[3 * i + 2], d.vel[i].w);
  if (mask & 8) d.omega[i] = make_float4(W[3 * i], W[3 * i + 1], W[3 * i + 2], 0.f);
}

__global__ void k_extend_contacts(const DevState d, uint32_t o, uint32_t count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  d.vals[0][o + i] = o + i;
  d.frozen[o + i] = 0;
  if (i == 0) d.ctr->front_valid = 0;
  for (int k = 0; k < 2; ++k) d.csr_start[k][o + 1 + i] = d.csr_start[k][o];
}

// host-side counts and one world's range and Morton box of a batch, as kernel parameters (no
// host buffer to keep alive while the stream catches up)
__global__ void k_set_counts(const DevState d, uint32_t n, uint32_t n_dyn) {
  d.ctr->n_bodies = n;
  d.ctr->n_dynamic = n_dyn;
}
__global__ void k_set_world(const DevState d, uint32_t widx, uint32_t first, uint32_t count, float4 lo, float4 ext) {
  d.world_first[widx] = first;
  d.world_count[widx] = count;
  d.world_bounds[2 * widx] = lo;
  d.world_bounds[2 * widx + 1] = ext;
}
__global__ void k_fill_u32(uint32_t* p, uint32_t count, uint32_t v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) p[i] = v;
}
__global__ void k_iota(uint32_t* p, uint32_t count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) p[i] = i;
}

// Bodies [so, so + count) of world `s` into [o, o + count) of world `d` (both on one stream), as
// an upload of the same bodies would write them: flags as the caller sees them, the previous
// velocity equal to the velocity, sleep timers at zero.  Bodies [o + count, o + slot) are
// parked as static specks on a line well outside the Morton box starting at `lo`, as
// bb_world_refill parks them.
__global__ void k_move_bodies(const DevState d, const DevState s, uint32_t o, uint32_t so, uint32_t count,
                              uint32_t slot, float3 lo, float4 park_shape) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= slot) return;
  const uint32_t b = o + i;
  if (i < count) {
    const uint32_t a = so + i;
    const float4 v = s.vel[a];
    d.pos[b] = s.pos[a];
    d.rot[b] = s.rot[a];
    d.vel[b] = v;
    d.pvel[b] = v;
    d.omega[b] = s.omega[a];
    d.shape[b] = s.shape[a];
    d.iinv[b] = s.iinv[a];
    d.iinv_off[b] = s.iinv_off[a];
    uint32_t f = s.flags[a];
    if (f & BB_BODY_PAUSED) f = (f & BB_BODY_PAUSE_AWAKE) ? (f & ~BB_BODY_SLEEPING) : f;
    d.flags[b] = f & (BB_BODY_DYNAMIC | BB_BODY_GRAVITY | BB_BODY_SLEEPING);
  } else {
    const float z = 0.f;
    d.pos[b] = make_float4(lo.x - 1000.0f - 0.01f * float(i - count), lo.y - 1000.0f, lo.z - 1000.0f, z);
    d.rot[b] = make_float4(z, z, z, 1.0f);
    d.vel[b] = make_float4(z, z, z, z);
    d.pvel[b] = make_float4(z, z, z, z);
    d.omega[b] = make_float4(z, z, z, z);
    d.shape[b] = park_shape;
    d.iinv[b] = make_float4(z, z, z, z);
    d.iinv_off[b] = make_float4(z, z, z, z);
    d.flags[b] = 0u;
  }
  d.sleep[b] = 0u;
}

// Pause (on = 1) or resume the dynamic bodies [o, o + count): a paused body is flagged asleep
// and remembers whether it was awake, so resuming gives back its flags exactly.
__global__ void k_pause(const DevState d, uint32_t o, uint32_t count, uint32_t on) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) d.ctr->front_valid = 0;
  if (i >= count) return;
  const uint32_t f = d.flags[o + i];
  if (!(f & BB_BODY_DYNAMIC)) return;
  if (on && !(f & BB_BODY_PAUSED)) {
    d.flags[o + i] = f | BB_BODY_PAUSED | BB_BODY_SLEEPING | ((f & BB_BODY_SLEEPING) ? 0u : BB_BODY_PAUSE_AWAKE);
  } else if (!on && (f & BB_BODY_PAUSED)) {
    uint32_t g = f & ~(BB_BODY_PAUSED | BB_BODY_PAUSE_AWAKE);
    if (f & BB_BODY_PAUSE_AWAKE) g &= ~BB_BODY_SLEEPING;
    d.flags[o + i] = g;
  }
}

// Bodies [o, o + count) were replaced (a refilled batch slot): the manifolds of both buffers
// that involve them are dropped from the warm-start lookups (per-body list entries and the
// manifold's bodies), they start unfrozen, and their sorted order restarts as the identity, as
// for a world just added.
__global__ void k_refill_contacts(const DevState d, uint32_t o, uint32_t count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) d.ctr->front_valid = 0;
  if (i >= count) return;
  const uint32_t id = o + i;
  d.vals[0][id] = id;
  d.frozen[id] = 0;
  for (int k = 0; k < 2; ++k) {
    const uint32_t s0 = d.csr_start[k][id], s1 = d.csr_start[k][id + 1];
    for (uint32_t e = s0; e < s1; ++e) {
      const uint32_t slot = d.man_slot[k][d.csr_list[k][e]];
      d.m_bodies[k][slot] = make_uint2(BB_NONE, BB_NONE);
      d.m_keycc[k][slot] = make_int2(-1, 0);
      d.csr_partner[k][e] = BB_NONE;
    }
  }
}

// Render feed: per body the affine transform [R | t] (3 x 4, row-major: the layout of a ray
// tracing instance transform), R from the quaternion (to_matrix, include/math.hpp:292-309),
// so that world = R * local + t.  The reference writes the same per-body transform into its
// TLAS instances (src/shaders/AS_mngr.slang:5-36, shared.inl:377-419).
__global__ void k_transforms(const DevState d, uint32_t n, float* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float R[3][3];
  q_matrix(q_from(d.rot[i]), R);
  const float4 p = d.pos[i];
  float* o = out + 12 * size_t(i);
  o[0] = R[0][0]; o[1] = R[0][1]; o[2] = R[0][2]; o[3] = p.x;
  o[4] = R[1][0]; o[5] = R[1][1]; o[6] = R[1][2]; o[7] = p.y;
  o[8] = R[2][0]; o[9] = R[2][1]; o[10] = R[2][2]; o[11] = p.z;
}

// Debug contact points of the last substep in manifold order, 8 slots per manifold (position,
// depth; unused slots get a NaN depth), written into the solver-row scratch (free between steps).
__global__ void k_contact_points(const DevState d, int cur, float4* out) {
  const uint32_t M = d.ctr->manifold_count;
  const size_t total = size_t(M) * BB_MAX_CONTACTS;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    const uint32_t m = uint32_t(t / BB_MAX_CONTACTS), j = uint32_t(t % BB_MAX_CONTACTS);
    const uint32_t slot = d.man_slot[cur][m];
    const int cc = d.m_keycc[cur][slot].y;
    out[t] = int(j) < cc ? d.c_pos[cur][size_t(slot) * BB_MAX_CONTACTS + j] : make_float4(0.f, 0.f, 0.f, __int_as_float(0x7FC00000));
  }
}

__global__ void k_begin_substep(DevCounters* c) {
  if (threadIdx.x != 0) return;
  const bool still = c->front_valid != 0u && c->sleep_ran != 0u && c->awake_after == 0u;
  c->front_skip = still ? 1u : 0u;
  c->front_n = still ? 0u : 0xFFFFFFFFu;
  c->front_valid = 1u;
  c->sleep_ran = 0;
  c->awake_after = 0;
  if (!still) {  // the skipped front end's outputs stay: its pair count and bounds
    c->pair_count = 0;
    c->hv_pool_n = 0;
    for (int k = 0; k < 3; ++k) {
      c->bounds_min[k] = 0xFFFFFFFFu;
      c->bounds_max[k] = 0u;
    }
  }
  c->prev_manifolds = c->manifold_count;
  c->manifold_count = 0;
  c->contact_count = 0;
  c->pgs_manifolds = 0;
  c->pgs_contacts = 0;
  c->fresh = 0;
  c->max_pen_bits = 0;
  c->island_count = 0;
  c->sleeping = 0;
  c->gc_colors = 0;
  c->gc_overflow = 0;
  c->gc_violations = 0;
  c->avbd_colors = 0;
  c->avbd_violations = 0;
  c->stick = 0;
  c->barrier_count = 0;
  c->round_flags[0] = 0;
  c->round_flags[1] = 0;
  c->heavy_n = 0;
  for (int k = 0; k < 8; ++k) c->sync_count[k] = 0;
  c->np_counts[0] = 0;
  c->np_counts[1] = 0;
  c->np_counts[2] = 0;
  c->np_counts[3] = 0;
  c->slot_count = 0;
  c->gc_list_n[0] = 0;
  c->gc_list_n[1] = 0;
  c->substeps += 1;
}

struct bb_world_impl {
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint32_t cap_n = 0, cap_p = 0, n = 0, n_dyn = 0;
  uint32_t max_world_n = 0;  // batched worlds: bodies of the largest world
  uint32_t max_world_bodies() const { return d.n_worlds > 1 ? max_world_n : n; }
  std::vector<Shape> shapes;
  std::vector<float> restitution;
  // batched worlds: first body id, body count (the slot's capacity) and dynamic bodies of each
  std::vector<uint32_t> wfirst, wcount, wdyn;
  uint32_t park_shape = 0xFFFFFFFFu;  // tiny box that parks a refilled slot's unused bodies
  // capacity regrow (bb_world_set_auto_regrow): a device snapshot of every array before the first
  // step since the last bb_sync, the steps issued since, and the host fields the steps change
  uint32_t ppb = 16, regrow_max_ppb = 0, regrows = 0;
  void* shadow = nullptr;
  size_t shadow_cap = 0;
  std::vector<size_t> shadow_sizes;
  std::vector<std::pair<float, uint32_t>> step_log;
  bool snapped = false;
  int snap_parity = 0, snap_last_cur = 0;
  bool snap_ran_any = false, snap_skip_warm = false;
  bb_solver_params params;
  DevState d = {};
  StepScratch sc = {};
  Owned owned;
  int parity = 0;    // manifold buffer of the last committed substep
  int last_cur = 0;  // manifold buffer the last (partial or full) substep wrote
  bool skip_warm_once = false;
  bool ran_any = false;
  int coop_edge = 0, coop_pgs = 0, coop_avbd = 0, coop_cc = 0;
  size_t scratch_bytes = 0;
  void* scratch_base = nullptr;
  size_t dev_bytes = 0;  // device memory held by this world
  float* xforms = nullptr;  // render feed: 12 floats per body
  // Pinned host staging for uploads issued while steps may be queued on the stream: a chunk is
  // reused once the copies issued from it have run (its event), so adding, refilling or
  // writing bodies does not wait for the queued steps.
  struct Stage {
    char* p = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
  };
  std::vector<Stage> stages;
  char* stage_get(size_t bytes, int* idx) {
    for (size_t k = 0; k < stages.size(); ++k)
      if (stages[k].cap >= bytes && cudaEventQuery(stages[k].ev) == cudaSuccess) {
        *idx = int(k);
        return stages[k].p;
      }
    if (stages.size() < 8) {
      Stage s;
      s.cap = std::max<size_t>(bytes, size_t(1) << 20);
      if (cudaMallocHost(&s.p, s.cap) != cudaSuccess) return nullptr;
      if (cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaFreeHost(s.p);
        return nullptr;
      }
      stages.push_back(s);
      *idx = int(stages.size() - 1);
      return stages.back().p;
    }
    Stage& s = stages[0];  // all in flight: wait for the oldest, grow it if needed
    cudaEventSynchronize(s.ev);
    if (s.cap < bytes) {
      cudaFreeHost(s.p);
      s.p = nullptr;
      s.cap = 0;
      if (cudaMallocHost(&s.p, bytes) != cudaSuccess) return nullptr;
      s.cap = bytes;
    }
    std::rotate(stages.begin(), stages.begin() + 1, stages.end());
    *idx = int(stages.size() - 1);
    return stages.back().p;
  }
  void stage_done(int idx) { cudaEventRecord(stages[size_t(idx)].ev, stream); }
  void stages_free() {
    for (auto& s : stages) {
      if (s.ev) cudaEventDestroy(s.ev);
      if (s.p) cudaFreeHost(s.p);
    }
    stages.clear();
  }
  // graph cache
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;
  };
  std::map<std::tuple<uint32_t, int, int, uint32_t, uint64_t, uint32_t>, GraphEntry> graphs;
  bool use_graphs = true;
  uint64_t launches = 0;
  // voxel shapes: host copies of the device table and pools
  std::vector<VoxDev> vox_table;
  std::vector<uint32_t> vox_occ, vox_surf;
  void* vox_buf = nullptr;     // device: table | occupancy | surface list
  void* slot_buf = nullptr;    // device: slot_cnt | slot_off | slot_pair | vox_list (pair capacity each)
  // profiling
  bool profiling = false;
  std::vector<std::string> stage_names;
  std::vector<float> stage_ms;

  ~bb_world_impl() {
    stages_free();
    for (auto& g : graphs)
      if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
    for (auto& o : owned) cudaFree(o.first);
    if (vox_buf) cudaFree(vox_buf);
    if (slot_buf) cudaFree(slot_buf);
    if (shadow) cudaFree(shadow);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }

  bb_status allocate() {
    cudaError_t err = cudaSuccess;
    const size_t N = cap_n + 1, P = cap_p;
    const size_t C = P * BB_MAX_CONTACTS;
    auto f4 = [&](size_t k) { return dalloc<float4>(k, owned, err, stream); };
    auto u32 = [&](size_t k) { return dalloc<uint32_t>(k, owned, err, stream); };
    d.pos = f4(N); d.rot = f4(N); d.vel = f4(N); d.omega = f4(N); d.pvel = f4(N); d.shape = f4(N); d.iinv = f4(N);
    d.flags = u32(N); d.sleep = u32(N); d.iw = f4(2 * N); d.iinv_off = f4(N); d.frozen = u32(N);
    for (int k = 0; k < 2; ++k) { d.keys[k] = u32(N); d.vals[k] = u32(N); }
    d.rank = u32(N);
    d.node_box = f4(4 * N);
    d.node_rec = f4(5 * N);
    d.child = dalloc<int2>(N, owned, err, stream);
    d.parent = dalloc<int32_t>(2 * N, owned, err, stream);
    d.range_last = dalloc<int32_t>(N, owned, err, stream);
    d.visit = u32(N);
    d.pair_cnt = u32(N); d.pair_off = u32(N + 1);
    d.is_heavy = u32(N); d.heavy_list = u32(8192);
    d.bp_stage = u32(size_t(N) * 32);
    d.hv_first = u32(8192); d.hv_n = u32(8192);
    d.hv_cap = uint32_t(P);
    d.hv_pool = u32(P); d.hv_slot = u32(P); d.hv_cnt = u32(P); d.hv_off = u32(P);
    d.flat_cnt = u32(4 * (N / 2048 + 2)); d.flat_off = u32(4 * (N / 2048 + 2));  // 4 queries x leaf tiles
    d.pairs = dalloc<uint2>(P, owned, err, stream);
    for (int k = 0; k < 2; ++k) {
      d.m_bodies[k] = dalloc<uint2>(P, owned, err, stream);
      d.m_keycc[k] = dalloc<int2>(P, owned, err, stream);
      d.m_normal[k] = f4(P); d.m_t0[k] = f4(P); d.m_t1[k] = f4(P); d.m_anchor_a[k] = f4(P); d.m_anchor_b[k] = f4(P);
      d.man_slot[k] = u32(P);
      d.c_pos[k] = f4(C); d.c_lam[k] = f4(C); d.c_kt[k] = f4(C); d.c_anc_a[k] = f4(C); d.c_anc_b[k] = f4(C);
      d.csr_start[k] = u32(N + 1);
      d.csr_list[k] = u32(2 * P);
      d.csr_partner[k] = u32(2 * P);
      d.csr_slot[k] = u32(2 * P);
    }
    d.c_r1 = f4(C); d.c_r2 = f4(C); d.c_k = f4(C);
    d.flow_rec = dalloc<uint4>(P, owned, err, stream);
    d.pgs_rec = dalloc<uint4>(P, owned, err, stream);
    d.np_list = u32(P); d.carry_list = u32(P);
    d.carry_ids = dalloc<uint2>(P, owned, err, stream);
    d.carry_tag = u32(P);
    d.gc_rec = dalloc<uint4>(P, owned, err, stream);
    d.gc_list[0] = u32(P); d.gc_list[1] = u32(P);
    d.pgs_mass = f4(P);
    d.pgs_frame = f4(3 * P);
    d.pgs_lam = f4(8 * P);
    d.pgs_cnt = u32(P); d.pgs_coff = u32(P); d.pgs_slot = u32(P);
    d.flow_counter = u32(N);
    d.range_first = dalloc<int32_t>(N, owned, err, stream);
    d.sworld = u32(N);
    d.world_of = u32(N); d.world_first = u32(N); d.world_count = u32(N);
    d.world_bounds = f4(2 * N);
    d.n_worlds = 0;
    d.csr_cursor = u32(N + 1);
    d.hit = u32(P); d.man_index = u32(P);
    d.uf_parent = u32(N); d.is_root = u32(N); d.root_rank = u32(N); d.island = u32(N);
    d.island_start = u32(N + 2);
    d.gc_color = u32(P); d.gc_pid = u32(P); d.gc_choice = u32(P); d.gc_mask = u32(N);
    d.gc_island_tag = u32(N); d.cc_mark = u32(N);
    d.gc_owner = dalloc<unsigned long long>(N * BB_MAX_COLORS, owned, err, stream);
    for (int k = 0; k < 2; ++k) { d.bucket_keys[k] = u32(P); d.bucket_vals[k] = u32(P); }
    d.bucket_start = u32(64);
    d.colour_awake = u32(BB_MAX_COLORS + 1);
    d.gc_slot_color[0] = u32(P); d.gc_slot_color[1] = u32(P);
    d.gc_reuse = u32(P); d.gc_survived = u32(P);
    d.gc_body_chg = u32(N); d.gc_island_chg = u32(N);
    d.body_color = u32(N); d.body_color_round = u32(N);
    d.a_pos_start = f4(N); d.a_rot_start = f4(N); d.a_pos_tilde = f4(N); d.a_rot_tilde = f4(N);
    d.a_depth = u32(N);
    for (int k = 0; k < 2; ++k) { d.a_bucket_keys[k] = u32(N); d.a_bucket_vals[k] = u32(N); }
    d.a_bucket_start = u32(64 * BB_MAX_COLORS + 2);
    d.ctr = dalloc<DevCounters>(1, owned, err, stream);
    d.staging = dalloc<float>(14 * N + 4, owned, err, stream);  // 13 floats of state + flags per body
    xforms = dalloc<float>(12 * N, owned, err, stream);
    d.pair_capacity = cap_p;
    d.body_capacity = cap_n;
    // scratch zeroed at every substep: scan status (7 scans), sort hists / status (12 slots)
    sc.scan_tiles = bb_scan_tiles(std::max<size_t>(P, N + 1));
    sc.sort_tiles = bb_sort_tiles(std::max<size_t>(P, N));
    size_t scan_words = size_t(7) * sc.scan_tiles;  // 64-bit
    size_t sort_status_words = size_t(12) * sc.sort_tiles * 256;
    size_t hist_words = 5 * BB_HIST_REGION;
    scratch_bytes = scan_words * 8 + 16 * 4 + hist_words * 4 + sort_status_words * 4 + 16 * 4;
    char* base = static_cast<char*>(static_cast<void*>(dalloc<uint8_t>(scratch_bytes + 256, owned, err, stream)));
    if (err != cudaSuccess) return fail(BB_E_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(err));
    scratch_base = base;
    sc.scan_status = reinterpret_cast<unsigned long long*>(base);
    base += scan_words * 8;
    sc.scan_tile_ctr = reinterpret_cast<uint32_t*>(base);
    base += 16 * 4;
    sc.sort_hist = reinterpret_cast<uint32_t*>(base);
    base += hist_words * 4;
    sc.sort_status = reinterpret_cast<uint32_t*>(base);
    base += sort_status_words * 4;
    sc.sort_tile_ctr = reinterpret_cast<uint32_t*>(base);
    return BB_OK;
  }

  void reset_contacts() {
    cudaMemsetAsync(d.frozen, 0, sizeof(uint32_t) * (cap_n + 1), stream);
    cudaMemsetAsync(&d.ctr->front_valid, 0, sizeof(uint32_t), stream);
    cudaMemsetAsync(&d.ctr->gc_coloured, 0, sizeof(uint32_t), stream);
    cudaMemsetAsync(d.csr_start[0], 0, sizeof(uint32_t) * (cap_n + 2), stream);
    cudaMemsetAsync(d.csr_start[1], 0, sizeof(uint32_t) * (cap_n + 2), stream);
    if (n) k_iota<<<(n + 255) / 256, 256, 0, stream>>>(d.vals[0], n);
  }

  // bodies [o, o + count) were appended: they start with empty contact lists and take the
  // next sorted positions; existing bodies keep their warm-start state and order
  void extend_contacts(uint32_t o, uint32_t count) {
    k_extend_contacts<<<(count + 255) / 256, 256, 0, stream>>>(d, o, count);
  }

  // device copy of every array (and the host fields a step changes), taken on the world's stream
  bb_status snapshot() {
    size_t total = 0;
    for (auto& o : owned) total += o.second;
    if (shadow_cap < total) {
      if (shadow) cudaFree(shadow);
      shadow = nullptr;
      shadow_cap = 0;
      cudaError_t e = cudaMalloc(&shadow, total);
      if (e != cudaSuccess) return fail(BB_E_CUDA, std::string("auto-regrow snapshot: ") + cudaGetErrorString(e));
      shadow_cap = total;
    }
    shadow_sizes.clear();
    size_t off = 0;
    for (auto& o : owned) {
      cudaMemcpyAsync(static_cast<char*>(shadow) + off, o.first, o.second, cudaMemcpyDeviceToDevice, stream);
      shadow_sizes.push_back(o.second);
      off += o.second;
    }
    snap_parity = parity;
    snap_last_cur = last_cur;
    snap_ran_any = ran_any;
    snap_skip_warm = skip_warm_once;
    snapped = true;
    step_log.clear();
    return BB_OK;
  }
  void forget_snapshot() {
    snapped = false;
    step_log.clear();
  }

  // Pair capacity raised to new_ppb pairs per body: every array reallocated, the snapshot copied
  // back into it (pair-, slot- and contact-indexed arrays keep their indices, so each array takes
  // the snapshot's bytes up to the smaller size), host fields back to the snapshot's.
  bb_status regrow(uint32_t new_ppb) {
    CU(cudaStreamSynchronize(stream));
    const DevState keep = d;
    for (auto& o : owned) cudaFree(o.first);
    owned.clear();
    ppb = new_ppb;
    cap_p = uint32_t(std::min<uint64_t>(uint64_t(ppb) * cap_n + 1024, 0x3FFFFFFFull));
    t_alloc_bytes = 0;
    bb_status st = allocate();
    if (st != BB_OK) return st;
    dev_bytes = t_alloc_bytes;
    d.n_worlds = keep.n_worlds;
    d.vox = keep.vox;
    d.vox_occ = keep.vox_occ;
    d.vox_surf = keep.vox_surf;
    d.vox_on = keep.vox_on;
    d.full_inertia = keep.full_inertia;
    if (slot_buf) {
      cudaFree(slot_buf);
      slot_buf = nullptr;
      CU(cudaMalloc(&slot_buf, 16ull * cap_p));
      uint32_t* sb = static_cast<uint32_t*>(slot_buf);
      d.slot_cnt = sb;
      d.slot_off = sb + cap_p;
      d.slot_pair = sb + 2ull * cap_p;
      d.vox_list = sb + 3ull * cap_p;
      dev_bytes += 16ull * cap_p;
    }
    if (owned.size() != shadow_sizes.size()) return fail(BB_E_CUDA, "auto-regrow: array layout changed");
    size_t off = 0;
    for (size_t k = 0; k < owned.size(); ++k) {
      CU(cudaMemcpyAsync(owned[k].first, static_cast<char*>(shadow) + off, std::min(owned[k].second, shadow_sizes[k]),
                         cudaMemcpyDeviceToDevice, stream));
      off += shadow_sizes[k];
    }
    parity = snap_parity;
    last_cur = snap_last_cur;
    ran_any = snap_ran_any;
    skip_warm_once = snap_skip_warm;
    invalidate_graphs();
    ++regrows;
    return BB_OK;
  }

  void invalidate_graphs() {
    for (auto& g : graphs)
      if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
    graphs.clear();
  }

  // one full pipeline pass (RBM:1284-1427) at h; commit = flip the manifold parity
  void substep(float h, bool warm, uint32_t stop_stage, bool commit) {
    const int cur = parity ^ 1;
    k_begin_substep<<<1, 32, 0, stream>>>(d.ctr);
    cudaMemsetAsync(scratch_base, 0, scratch_bytes, stream);
    bb_front_end(stream, d, params, n, sc, sms, cur, max_world_bodies());
    if (stop_stage >= 2) bb_narrow_phase(stream, d, params, n, sc, sms, cur, warm);
    last_cur = cur;
    if (stop_stage < 3) return;
    bb_advect(stream, d, params, n, h, sms);
    bb_islands(stream, d, params, n, sc, sms, cur, coop_cc);
    bb_sleep(stream, d, params, n, sms, cur);
    const bool coloured = (params.flags & BB_SIM_USE_GRAPH_COLORING) != 0;
    if (coloured || params.solver == BB_SOLVER_AVBD) bb_edge_coloring(stream, d, params, n, sc, sms, cur, coop_edge);
    if (params.solver == BB_SOLVER_AVBD) bb_solve_avbd(stream, d, params, n, h, sc, sms, cur, coop_avbd);
    else if (!coloured) bb_solve_islands(stream, d, params, n, h, cur, sc, sms);
    else bb_solve_pgs_soft(stream, d, params, n, h, cur, sc, coop_pgs, sms);
    if (commit) parity = cur;
  }
};

using World = bb_world_impl;

static World* W(void* w) { return static_cast<World*>(w); }

namespace {
struct StateHeader {
  uint32_t magic, version;
  uint32_t cap_n, cap_p, n, n_dyn, n_worlds, vox_on, full_inertia;
  int32_t parity, last_cur;
  uint32_t ran_any, skip_warm_once, arrays;
  uint64_t slot_bytes, total;
  bb_solver_params params;
};
constexpr uint32_t kStateMagic = 0x31534242u;  // "BBS1"
constexpr uint32_t kStateVersion = 2;  // the array set of this build (frozen-pair carry and list slots)
uint64_t state_bytes(const World* w) {
  uint64_t t = sizeof(StateHeader) + 8ull * w->owned.size();
  for (auto& o : w->owned) t += o.second;
  if (w->slot_buf) t += 16ull * w->cap_p;
  return t;
}
}  // namespace

extern "C" {

const char* bb_last_error_string(void) { return g_last_error.c_str(); }
const char* bb_version(void) { return "beatbox-b200 0.1 (sm_100a)"; }

void bb_default_solver_params(bb_solver_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->solver = BB_SOLVER_AVBD;
  p->flags = BB_SIM_DEFAULT_FLAGS;
  p->quirks = BB_QUIRKS_REFERENCE;
  p->iterations = 5;
  p->relax_iterations = 5;
  p->gc_rounds = 32;
  p->gravity = -9.81f;
  p->linear_damping = 0.1f;
  p->angular_damping = 0.1f;
  p->contact_hertz = 30.0f;
  p->penetration_cap = -0.25f;
  p->sleep_lin_vel2 = 0.0144f;
  p->sleep_ang_vel2 = 0.0225f;
  p->sleep_steps = 30;
  p->avbd_iterations = 10;
  p->avbd_beta = 100000.0f;
  p->avbd_gamma = 0.99f;
  p->avbd_k_min = 1.0f;
  p->avbd_k_max = 1000000000.0f;
  p->avbd_margin = 0.0005f;
  p->avbd_stick_thresh = 0.01f;
  p->avbd_stick_slop = 0.001f;
  p->avbd_color_rounds = 16;
  p->avbd_shock_layers = 12;
  p->avbd_post_stab_sweeps = 4;
  p->schedule = BB_SCHEDULE_COLOUR_BARRIER;
  p->broad_threads = 128;
  p->narrow_blocks_per_sm = 16;
  p->pgs_stage_next = 0;
  p->bounds_mode = BB_BOUNDS_FIXED;
  for (int k = 0; k < 3; ++k) {
    p->world_min[k] = -64.0f;
    p->world_extent[k] = 128.0f;
  }
}

bb_status bb_world_create(const bb_world_desc* desc, void** out_world) {
  if (!desc || !out_world || desc->max_bodies == 0) return fail(BB_E_INVALID, "bb_world_create: bad arguments");
  World* w = new World();
  if (desc->device >= 0) {
    cudaError_t e = cudaSetDevice(desc->device);
    if (e != cudaSuccess) {
      delete w;
      return fail(BB_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
  }
  cudaGetDevice(&w->device);
  cudaDeviceGetAttribute(&w->sms, cudaDevAttrMultiProcessorCount, w->device);
  if (desc->stream) {
    w->stream = static_cast<cudaStream_t>(desc->stream);
  } else {
    cudaError_t e = cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete w;
      return fail(BB_E_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    w->own_stream = true;
  }
  w->cap_n = desc->max_bodies;
  uint32_t ppb = desc->pairs_per_body ? desc->pairs_per_body : 16;
  w->ppb = ppb;
  w->cap_p = uint32_t(std::min<uint64_t>(uint64_t(ppb) * w->cap_n + 1024, 0x3FFFFFFFull));
  bb_default_solver_params(&w->params);
  t_alloc_bytes = 0;
  bb_status st = w->allocate();
  w->dev_bytes = t_alloc_bytes;
  if (st != BB_OK) {
    delete w;
    return st;
  }
  // Persistent grids sized to the world's capacity: about one thread per item of the largest
  // colour (~half the bodies) for the sweeps, about one per body for colouring and components.
  // A small world then runs on a block or two (its barriers become CTA barriers) and leaves
  // the rest of the GPU to other worlds' streams.  Results do not depend on the grid.
  auto fit = [](int max_blocks, uint64_t items, int threads) {
    return int(std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(max_blocks), (items + threads - 1) / threads)));
  };
  w->coop_edge = fit(bb_edge_coloring_blocks(w->sms), w->cap_n, 1024);
  w->coop_pgs = fit(bb_pgs_soft_blocks(w->sms), w->cap_n / 2, 256);
  onesweep_smem_attr();
  w->coop_avbd = fit(bb_avbd_blocks(w->sms), w->cap_n / 2, 512);
  w->coop_cc = fit(bb_components_blocks(w->sms), w->cap_n, 512);
  // The zero fills run on the world's stream ahead of everything the world does later.  On a
  // stream of its own, wait for them here (no device-wide wait); on the caller's stream, which may
  // hold queued work of other worlds, only check that they were issued.
  cudaError_t e = w->own_stream ? cudaStreamSynchronize(w->stream) : cudaGetLastError();
  if (e != cudaSuccess) {
    delete w;
    return fail(BB_E_CUDA, std::string("create: ") + cudaGetErrorString(e));
  }
  *out_world = w;
  return BB_OK;
}

bb_status bb_world_destroy(void* world) {
  if (!world) return fail(BB_E_INVALID, "bb_world_destroy: null world");
  cudaStreamSynchronize(W(world)->stream);
  delete W(world);
  return BB_OK;
}

void* bb_world_stream(void* world) { return world ? W(world)->stream : nullptr; }
uint64_t bb_world_device_bytes(void* world) { return world ? W(world)->dev_bytes : 0; }

uint64_t bb_world_bytes_for(uint32_t max_bodies, uint32_t pairs_per_body) {
  World probe;
  probe.cap_n = max_bodies;
  const uint32_t ppb = pairs_per_body ? pairs_per_body : 16;
  probe.cap_p = uint32_t(std::min<uint64_t>(uint64_t(ppb) * max_bodies + 1024, 0x3FFFFFFFull));
  t_alloc_bytes = 0;
  t_count_only = true;
  probe.allocate();
  t_count_only = false;
  probe.owned.clear();
  return t_alloc_bytes;
}

// Remove every body and shape; allocations, stream and parameters stay (for reuse of a world
// object by a server).  Persistent contact state restarts as for a new world.
bb_status bb_world_clear(void* world) {
  World* w = W(world);
  if (!w) return fail(BB_E_INVALID, "bb_world_clear: null world");
  CU(cudaStreamSynchronize(w->stream));
  w->n = 0;
  w->n_dyn = 0;
  w->max_world_n = 0;
  w->shapes.clear();
  w->restitution.clear();
  w->wfirst.clear();
  w->wcount.clear();
  w->wdyn.clear();
  w->park_shape = 0xFFFFFFFFu;
  w->vox_table.clear();
  w->vox_occ.clear();
  w->vox_surf.clear();
  w->d.vox_on = 0;
  w->d.full_inertia = 0;
  w->d.n_worlds = 0;
  w->parity = 0;
  w->last_cur = 0;
  w->skip_warm_once = false;
  w->ran_any = false;
  w->forget_snapshot();
  w->invalidate_graphs();
  uint32_t nn[2] = {0, 0};
  CU(cudaMemcpyAsync(w->d.ctr, nn, sizeof(nn), cudaMemcpyHostToDevice, w->stream));
  // the next substep rebuilds the front end whatever the bodies added later; the sticky
  // device error bits of earlier steps go with the bodies
  CU(cudaMemsetAsync(&w->d.ctr->front_valid, 0, sizeof(uint32_t), w->stream));
  CU(cudaMemsetAsync(&w->d.ctr->error_flags, 0, sizeof(uint32_t), w->stream));
  CU(cudaMemsetAsync(&w->d.ctr->error_site, 0, sizeof(uint32_t), w->stream));
  CU(cudaStreamSynchronize(w->stream));
  return BB_OK;
}
uint32_t bb_body_count(void* world) { return world ? W(world)->n : 0; }

bb_status bb_add_box_shape(void* world, float hx, float hy, float hz, uint32_t* out_shape) {
  if (!world || !out_shape || !(hx > 0) || !(hy > 0) || !(hz > 0)) return fail(BB_E_INVALID, "bb_add_box_shape: bad arguments");
  W(world)->shapes.push_back(Shape{BB_SHAPE_BOX, {hx, hy, hz}});
  *out_shape = uint32_t(W(world)->shapes.size() - 1);
  return BB_OK;
}

bb_status bb_add_sphere_shape(void* world, float radius, uint32_t* out_shape) {
  if (!world || !out_shape || !(radius > 0)) return fail(BB_E_INVALID, "bb_add_sphere_shape: bad arguments");
  W(world)->shapes.push_back(Shape{BB_SHAPE_SPHERE, {radius, radius, radius}});
  *out_shape = uint32_t(W(world)->shapes.size() - 1);
  return BB_OK;
}

bb_status bb_voxel_shape_info(uint32_t nx, uint32_t ny, uint32_t nz, float voxel_size, const uint8_t* solid,
                              bb_voxel_info* out, uint32_t* surface, uint32_t surface_capacity) {
  VoxelBuild b;
  if (!out || !voxel_build(nx, ny, nz, voxel_size, solid, b))
    return fail(BB_E_INVALID, "bb_voxel_shape_info: bad grid (dims 1..256, voxel_size > 0, one solid cell)");
  for (int k = 0; k < 3; ++k) {
    out->grid_origin[k] = b.origin[k];
    out->box_min[k] = b.origin[k];
    out->box_max[k] = b.hi[k];
  }
  out->solid_count = b.solid;
  out->surface_count = uint32_t(b.surf.size());
  out->unit_mass = b.unit_mass;
  for (int k = 0; k < 6; ++k) out->unit_inv_inertia[k] = b.unit_inv[k];
  if (surface) {
    if (surface_capacity < b.surf.size()) return fail(BB_E_INVALID, "bb_voxel_shape_info: surface buffer too small");
    std::memcpy(surface, b.surf.data(), 4 * b.surf.size());
  }
  return BB_OK;
}

// Appends the shape to the world's voxel table and re-uploads table and pools (shapes are
// added while building a scene, not per step).  The first voxel shape also allocates the
// per-slot arrays of the narrow phase (six manifold slots per voxel pair).
bb_status bb_add_voxel_shape(void* world, uint32_t nx, uint32_t ny, uint32_t nz, float voxel_size,
                             const uint8_t* solid, uint32_t* out_shape) {
  World* w = W(world);
  VoxelBuild b;
  if (!w || !out_shape || !voxel_build(nx, ny, nz, voxel_size, solid, b))
    return fail(BB_E_INVALID, "bb_add_voxel_shape: bad arguments (dims 1..256, voxel_size > 0, one solid cell)");
  if (w->vox_table.size() >= (1u << 24)) return fail(BB_E_INVALID, "bb_add_voxel_shape: too many voxel shapes");
  VoxDev v = {};
  v.ox = b.origin[0];
  v.oy = b.origin[1];
  v.oz = b.origin[2];
  v.vs = b.vs;
  v.hx = b.hi[0];
  v.hy = b.hi[1];
  v.hz = b.hi[2];
  v.surf_count = uint32_t(b.surf.size());
  v.dx = nx;
  v.dy = ny;
  v.dz = nz;
  v.occ_off = uint32_t(w->vox_occ.size());
  v.surf_off = uint32_t(w->vox_surf.size());
  w->vox_table.push_back(v);
  w->vox_occ.insert(w->vox_occ.end(), b.occ.begin(), b.occ.end());
  w->vox_surf.insert(w->vox_surf.end(), b.surf.begin(), b.surf.end());
  CU(cudaStreamSynchronize(w->stream));
  if (!w->slot_buf) {
    CU(cudaMalloc(&w->slot_buf, 16ull * w->cap_p));
    uint32_t* sb = static_cast<uint32_t*>(w->slot_buf);
    w->d.slot_cnt = sb;
    w->d.slot_off = sb + w->cap_p;
    w->d.slot_pair = sb + 2ull * w->cap_p;
    w->d.vox_list = sb + 3ull * w->cap_p;
    w->dev_bytes += 16ull * w->cap_p;
  }
  const size_t tb = sizeof(VoxDev) * w->vox_table.size(), ob = 4 * w->vox_occ.size(), sb = 4 * w->vox_surf.size();
  if (w->vox_buf) {
    CU(cudaFree(w->vox_buf));
    w->vox_buf = nullptr;
  }
  CU(cudaMalloc(&w->vox_buf, tb + ob + sb + 16));
  char* base = static_cast<char*>(w->vox_buf);
  CU(cudaMemcpyAsync(base, w->vox_table.data(), tb, cudaMemcpyHostToDevice, w->stream));
  CU(cudaMemcpyAsync(base + tb, w->vox_occ.data(), ob, cudaMemcpyHostToDevice, w->stream));
  CU(cudaMemcpyAsync(base + tb + ob, w->vox_surf.data(), sb, cudaMemcpyHostToDevice, w->stream));
  CU(cudaStreamSynchronize(w->stream));
  w->d.vox = reinterpret_cast<const VoxDev*>(base);
  w->d.vox_occ = reinterpret_cast<const uint32_t*>(base + tb);
  w->d.vox_surf = reinterpret_cast<const uint32_t*>(base + tb + ob);
  w->d.vox_on = 1;
  Shape sh{BB_SHAPE_VOXEL, {0.5f * (b.hi[0] - b.origin[0]), 0.5f * (b.hi[1] - b.origin[1]), 0.5f * (b.hi[2] - b.origin[2])}};
  sh.vox = uint32_t(w->vox_table.size() - 1);
  sh.unit_mass = b.unit_mass;
  for (int k = 0; k < 6; ++k) sh.unit_inv[k] = b.unit_inv[k];
  w->shapes.push_back(sh);
  w->invalidate_graphs();
  *out_shape = uint32_t(w->shapes.size() - 1);
  return BB_OK;
}

// Bodies converted to the device layout (SoA float4 rows), ready to upload at some offset.
struct BodyRows {
  std::vector<float4> pos, rot, vel, om, shp, ii, io;
  std::vector<uint32_t> fl;
  std::vector<float> restitution;
  bool any_off = false;
  uint32_t ndyn = 0;
  void resize(uint32_t count) {
    for (auto* v : {&pos, &rot, &vel, &om, &shp, &ii, &io}) v->assign(count, make_float4(0.f, 0.f, 0.f, 0.f));
    fl.assign(count, 0u);
    restitution.assign(count, 0.f);
  }
};

static bb_status pack_bodies(World* w, const bb_body_desc* bodies, uint32_t count, BodyRows& r) {
  r.resize(count);
  std::vector<float4>&pos = r.pos, &rot = r.rot, &vel = r.vel, &om = r.om, &shp = r.shp, &ii = r.ii, &io = r.io;
  std::vector<uint32_t>& fl = r.fl;
  bool& any_off = r.any_off;
  uint32_t& ndyn = r.ndyn;
  for (uint32_t i = 0; i < count; ++i) {
    const bb_body_desc& b = bodies[i];
    if (b.shape >= w->shapes.size()) return fail(BB_E_INVALID, "bb_add_bodies: unknown shape handle");
    const Shape& s = w->shapes[b.shape];
    bool dyn = (b.flags & BB_BODY_DYNAMIC) != 0;
    double vol = s.type == BB_SHAPE_BOX ? 8.0 * s.half[0] * s.half[1] * s.half[2]
                                        : 4.0 / 3.0 * 3.14159265358979 * double(s.half[0]) * s.half[0] * s.half[0];
    float mass = b.mass > 0 ? b.mass : (s.type == BB_SHAPE_VOXEL ? b.density * s.unit_mass : float(b.density * vol));
    if (!dyn) mass = 0;
    if (dyn && !(mass > 0)) return fail(BB_E_INVALID, "bb_add_bodies: dynamic body needs mass or density");
    float inv_mass = dyn ? 1.0f / mass : 0.0f;
    float inv_i[3] = {0, 0, 0}, inv_o[3] = {0, 0, 0};
    if (dyn) {
      if (b.inertia_mode == BB_INERTIA_EXPLICIT) {
        for (int k = 0; k < 3; ++k) {
          inv_i[k] = b.inv_inertia[k];
          inv_o[k] = b.inv_inertia_off[k];
        }
      } else if (s.type == BB_SHAPE_VOXEL) {
        const float scale = s.unit_mass / mass;  // inertia scales with mass at fixed shape
        for (int k = 0; k < 3; ++k) {
          inv_i[k] = s.unit_inv[k] * scale;
          inv_o[k] = s.unit_inv[3 + k] * scale;
        }
      } else if (b.inertia_mode == BB_INERTIA_REFERENCE) {
        // cuboid_get_inverse_intertia(inv_mass, min, max) (include/math.hpp:106-130)
        float w_ = 2 * s.half[0], h_ = 2 * s.half[1], d_ = 2 * s.half[2];
        float t = 1.0f / 12.0f;
        inv_i[0] = 1.0f / (t * inv_mass * (h_ * h_ + d_ * d_));
        inv_i[1] = 1.0f / (t * inv_mass * (w_ * w_ + d_ * d_));
        inv_i[2] = 1.0f / (t * inv_mass * (w_ * w_ + h_ * h_));
      } else if (s.type == BB_SHAPE_BOX) {
        double w_ = 2.0 * s.half[0], h_ = 2.0 * s.half[1], d_ = 2.0 * s.half[2];
        inv_i[0] = float(12.0 / (mass * (h_ * h_ + d_ * d_)));
        inv_i[1] = float(12.0 / (mass * (w_ * w_ + d_ * d_)));
        inv_i[2] = float(12.0 / (mass * (w_ * w_ + h_ * h_)));
      } else {
        float v = float(5.0 / (2.0 * mass * double(s.half[0]) * s.half[0]));
        inv_i[0] = inv_i[1] = inv_i[2] = v;
      }
    }
    pos[i] = make_float4(b.position[0], b.position[1], b.position[2], inv_mass);
    rot[i] = make_float4(b.rotation[0], b.rotation[1], b.rotation[2], b.rotation[3]);
    vel[i] = make_float4(b.velocity[0], b.velocity[1], b.velocity[2], mass);
    om[i] = make_float4(b.omega[0], b.omega[1], b.omega[2], 0.f);
    uint32_t tbits = s.type | (s.type == BB_SHAPE_VOXEL ? s.vox << 8 : 0u);
    float tf;
    std::memcpy(&tf, &tbits, 4);
    shp[i] = make_float4(s.half[0], s.half[1], s.half[2], tf);
    ii[i] = make_float4(inv_i[0], inv_i[1], inv_i[2], b.friction);
    io[i] = make_float4(inv_o[0], inv_o[1], inv_o[2], 0.f);
    if (inv_o[0] != 0.f || inv_o[1] != 0.f || inv_o[2] != 0.f) any_off = true;
    fl[i] = b.flags & (BB_BODY_DYNAMIC | BB_BODY_GRAVITY | BB_BODY_SLEEPING);
    if (dyn) ++ndyn;
    r.restitution[i] = b.restitution;
  }
  return BB_OK;
}

// rows of `r` into body ids [o, o + count) on the world's stream (sleep timers start at 0),
// copied through the world's pinned staging: nothing waits for the steps queued before
static bb_status upload_bodies(World* w, uint32_t o, const BodyRows& r) {
  const uint32_t count = uint32_t(r.fl.size());
  if (count == 0) return BB_OK;
  const size_t f4 = size_t(count) * sizeof(float4);
  int si = 0;
  char* h = w->stage_get(8 * f4 + size_t(count) * sizeof(uint32_t), &si);
  if (!h) return fail(BB_E_CUDA, "upload: pinned staging could not be allocated");
  const std::vector<float4>* rows[7] = {&r.pos, &r.rot, &r.vel, &r.om, &r.shp, &r.ii, &r.io};
  for (int k = 0; k < 7; ++k) std::memcpy(h + k * f4, rows[k]->data(), f4);
  std::memcpy(h + 7 * f4, r.fl.data(), size_t(count) * sizeof(uint32_t));
  float4* dst[7] = {w->d.pos, w->d.rot, w->d.vel, w->d.omega, w->d.shape, w->d.iinv, w->d.iinv_off};
  for (int k = 0; k < 7; ++k) CU(cudaMemcpyAsync(dst[k] + o, h + k * f4, f4, cudaMemcpyHostToDevice, w->stream));
  CU(cudaMemcpyAsync(w->d.pvel + o, h + 2 * f4, f4, cudaMemcpyHostToDevice, w->stream));
  CU(cudaMemcpyAsync(w->d.flags + o, h + 7 * f4, size_t(count) * sizeof(uint32_t), cudaMemcpyHostToDevice, w->stream));
  CU(cudaMemsetAsync(w->d.sleep + o, 0, size_t(count) * sizeof(uint32_t), w->stream));
  w->stage_done(si);
  if (r.any_off) w->d.full_inertia = 1;
  return BB_OK;
}

static bb_status add_bodies_impl(World* w, const bb_body_desc* bodies, uint32_t count, uint32_t* out_first_id,
                                 bool keep_contacts = false) {
  if (!w || (!bodies && count)) return fail(BB_E_INVALID, "bb_add_bodies: bad arguments");
  if (uint64_t(w->n) + count > w->cap_n) return fail(BB_E_CAPACITY, "bb_add_bodies: max_bodies exceeded");
  BodyRows r;
  bb_status st = pack_bodies(w, bodies, count, r);
  if (st != BB_OK) return st;
  const uint32_t o = w->n;
  st = upload_bodies(w, o, r);
  if (st != BB_OK) return st;
  w->restitution.insert(w->restitution.end(), r.restitution.begin(), r.restitution.end());
  const uint32_t ndyn = r.ndyn;
  w->n += count;
  w->n_dyn += ndyn;
  if (out_first_id) *out_first_id = o;
  // new bodies restart the persistent state (sorted order, warm-start contacts), as a scene
  // load does in the reference; a world added to a batch leaves the other worlds' state alone
  if (keep_contacts) w->extend_contacts(o, count);
  else w->reset_contacts();
  w->invalidate_graphs();
  k_set_counts<<<1, 1, 0, w->stream>>>(w->d, w->n, w->n_dyn);
  CU(cudaGetLastError());
  return BB_OK;
}

bb_status bb_add_bodies(void* world, const bb_body_desc* bodies, uint32_t count, uint32_t* out_first_id) {
  World* w = W(world);
  if (w) w->forget_snapshot();
  if (w && w->d.n_worlds > 0) return fail(BB_E_INVALID, "bb_add_bodies: this object holds batched worlds");
  return add_bodies_impl(w, bodies, count, out_first_id);
}

bb_status bb_add_world(void* world, const bb_batch_world_desc* desc, const bb_body_desc* bodies, uint32_t count,
                       uint32_t* out_world_index, uint32_t* out_first_id) {
  World* w = W(world);
  if (!w || !desc || count == 0) return fail(BB_E_INVALID, "bb_add_world: bad arguments");
  w->forget_snapshot();
  if (w->d.n_worlds == 0 && w->n > 0) return fail(BB_E_INVALID, "bb_add_world: object already holds a plain world");
  for (int k = 0; k < 3; ++k)
    if (!(desc->world_extent[k] > 0)) return fail(BB_E_INVALID, "bb_add_world: world_extent must be positive");
  uint32_t first = 0;
  const uint32_t dyn_before = w->n_dyn;
  bb_status st = add_bodies_impl(w, bodies, count, &first, w->d.n_worlds > 0);
  if (st != BB_OK) return st;
  const uint32_t widx = w->d.n_worlds;
  w->wfirst.push_back(first);
  w->wcount.push_back(count);
  w->wdyn.push_back(w->n_dyn - dyn_before);
  k_fill_u32<<<(count + 255) / 256, 256, 0, w->stream>>>(w->d.world_of + first, count, widx);
  k_set_world<<<1, 1, 0, w->stream>>>(w->d, widx, first, count,
                                      make_float4(desc->world_min[0], desc->world_min[1], desc->world_min[2], 0.f),
                                      make_float4(desc->world_extent[0], desc->world_extent[1], desc->world_extent[2], 0.f));
  CU(cudaGetLastError());
  w->d.n_worlds = widx + 1;
  w->max_world_n = std::max(w->max_world_n, count);
  w->invalidate_graphs();
  if (out_world_index) *out_world_index = widx;
  if (out_first_id) *out_first_id = first;
  return BB_OK;
}

uint32_t bb_world_count(void* world) { return world ? W(world)->d.n_worlds : 0; }

// body id range of world `widx` of a batch, or of the whole plain world (widx 0)
static bool world_range(World* w, uint32_t widx, uint32_t* first, uint32_t* count) {
  if (w->d.n_worlds == 0) {
    if (widx != 0) return false;
    *first = 0;
    *count = w->n;
    return true;
  }
  if (widx >= w->wfirst.size()) return false;
  *first = w->wfirst[widx];
  *count = w->wcount[widx];
  return true;
}

bb_status bb_world_pause(void* world, uint32_t world_index, uint32_t paused) {
  World* w = W(world);
  uint32_t first = 0, count = 0;
  if (!w || !world_range(w, world_index, &first, &count)) return fail(BB_E_INVALID, "bb_world_pause: bad world index");
  w->forget_snapshot();
  if (count == 0) return BB_OK;
  k_pause<<<(count + 255) / 256, 256, 0, w->stream>>>(w->d, first, count, paused ? 1u : 0u);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(BB_E_CUDA, std::string("bb_world_pause: ") + cudaGetErrorString(e));
  return BB_OK;
}

bb_status bb_world_refill(void* world, uint32_t world_index, const bb_batch_world_desc* desc,
                          const bb_body_desc* bodies, uint32_t count) {
  World* w = W(world);
  if (!w || !desc || (!bodies && count)) return fail(BB_E_INVALID, "bb_world_refill: bad arguments");
  if (w->d.n_worlds == 0 || world_index >= w->wfirst.size())
    return fail(BB_E_INVALID, "bb_world_refill: not a world of this batch");
  for (int k = 0; k < 3; ++k)
    if (!(desc->world_extent[k] > 0)) return fail(BB_E_INVALID, "bb_world_refill: world_extent must be positive");
  const uint32_t first = w->wfirst[world_index], slot = w->wcount[world_index];
  if (count > slot) return fail(BB_E_CAPACITY, "bb_world_refill: more bodies than the world's slot holds");
  w->forget_snapshot();
  if (w->park_shape == 0xFFFFFFFFu) {
    w->shapes.push_back(Shape{BB_SHAPE_BOX, {0.001f, 0.001f, 0.001f}});
    w->park_shape = uint32_t(w->shapes.size() - 1);
  }
  // the slot's unused bodies are parked: static specks on a line well outside the world's box
  std::vector<bb_body_desc> all(slot);
  for (uint32_t i = 0; i < count; ++i) all[i] = bodies[i];
  for (uint32_t i = count; i < slot; ++i) {
    bb_body_desc& b = all[i];
    std::memset(&b, 0, sizeof(b));
    b.position[0] = desc->world_min[0] - 1000.0f - 0.01f * float(i - count);
    b.position[1] = desc->world_min[1] - 1000.0f;
    b.position[2] = desc->world_min[2] - 1000.0f;
    b.rotation[3] = 1.0f;
    b.shape = w->park_shape;
  }
  BodyRows r;
  bb_status st = pack_bodies(w, all.data(), slot, r);
  if (st != BB_OK) return st;
  st = upload_bodies(w, first, r);
  if (st != BB_OK) return st;
  for (uint32_t i = 0; i < slot; ++i) w->restitution[first + i] = r.restitution[i];
  w->n_dyn = w->n_dyn - w->wdyn[world_index] + r.ndyn;
  w->wdyn[world_index] = r.ndyn;
  k_set_world<<<1, 1, 0, w->stream>>>(w->d, world_index, first, slot,
                                      make_float4(desc->world_min[0], desc->world_min[1], desc->world_min[2], 0.f),
                                      make_float4(desc->world_extent[0], desc->world_extent[1], desc->world_extent[2], 0.f));
  k_refill_contacts<<<(slot + 255) / 256, 256, 0, w->stream>>>(w->d, first, slot);
  k_set_counts<<<1, 1, 0, w->stream>>>(w->d, w->n, w->n_dyn);
  CU(cudaGetLastError());
  return BB_OK;
}

bb_status bb_set_material(void* world, uint32_t first, uint32_t count, float friction, float restitution) {
  World* w = W(world);
  if (!w || uint64_t(first) + count > w->n) return fail(BB_E_INVALID, "bb_set_material: bad range");
  cudaStreamSynchronize(w->stream);
  w->forget_snapshot();
  std::vector<float4> ii(count);
  CU(cudaMemcpy(ii.data(), w->d.iinv + first, count * sizeof(float4), cudaMemcpyDeviceToHost));
  for (auto& v : ii) v.w = friction;
  CU(cudaMemcpyAsync(w->d.iinv + first, ii.data(), count * sizeof(float4), cudaMemcpyHostToDevice, w->stream));
  CU(cudaStreamSynchronize(w->stream));
  for (uint32_t i = 0; i < count; ++i) w->restitution[first + i] = restitution;
  return BB_OK;
}

bb_status bb_set_solver_params(void* world, const bb_solver_params* p) {
  World* w = W(world);
  if (!w || !p) return fail(BB_E_INVALID, "bb_set_solver_params: bad arguments");
  w->forget_snapshot();
  if (p->solver == BB_SOLVER_PGS && (p->flags & BB_SIM_USE_GRAPH_COLORING))
    return fail(BB_E_INVALID, "BB_SOLVER_PGS runs on the per-island path only: clear BB_SIM_USE_GRAPH_COLORING");
  if (p->solver > BB_SOLVER_AVBD) return fail(BB_E_INVALID, "unknown solver");
  if (p->gc_rounds > 63 || p->avbd_shock_layers == 0 || p->avbd_shock_layers > 64)
    return fail(BB_E_INVALID, "gc_rounds <= 63 and 1 <= avbd_shock_layers <= 64 required");
  for (int k = 0; k < 3; ++k)
    if (!(p->world_extent[k] > 0)) return fail(BB_E_INVALID, "world_extent must be positive");
  if (p->schedule > BB_SCHEDULE_COLOUR_BARRIER) return fail(BB_E_INVALID, "unknown schedule");
  if ((p->broad_threads != 0 && p->broad_threads != 32 && p->broad_threads != 64 && p->broad_threads != 128) ||
      p->narrow_blocks_per_sm > 64 || p->pgs_stage_next > 1)
    return fail(BB_E_INVALID, "launch geometry out of range (broad_threads 32/64/128, narrow <= 64, pgs_stage_next 0/1)");
  // contact geometry depends on these: no pair keeps last substep's manifolds as they were
  if (p->quirks != w->params.quirks || p->penetration_cap != w->params.penetration_cap)
    CU(cudaMemsetAsync(w->d.frozen, 0, 4ull * (w->cap_n + 1), w->stream));
  CU(cudaMemsetAsync(&w->d.ctr->front_valid, 0, sizeof(uint32_t), w->stream));  // bounds, modes
  // the colouring rounds (gc_rounds) may change: the next colouring starts afresh
  CU(cudaMemsetAsync(&w->d.ctr->gc_coloured, 0, sizeof(uint32_t), w->stream));
  w->params = *p;
  if (!w->params.broad_threads) w->params.broad_threads = 128;
  if (!w->params.narrow_blocks_per_sm) w->params.narrow_blocks_per_sm = 16;
  return BB_OK;
}

bb_status bb_get_solver_params(void* world, bb_solver_params* p) {
  if (!world || !p) return fail(BB_E_INVALID, "bb_get_solver_params: bad arguments");
  *p = W(world)->params;
  return BB_OK;
}

bb_status bb_skip_warm_starting_once(void* world) {
  if (!world) return fail(BB_E_INVALID, "null world");
  W(world)->skip_warm_once = true;
  return BB_OK;
}

bb_status bb_step(void* world, float dt, uint32_t substeps) {
  World* w = W(world);
  if (!w || !(dt > 0) || substeps == 0 || substeps > 64) return fail(BB_E_INVALID, "bb_step: bad arguments");
  if (w->n == 0) return BB_OK;
  if (w->regrow_max_ppb) {  // auto-regrow: snapshot before the first step since the last sync
    if (!w->snapped) {
      bb_status st = w->snapshot();
      if (st != BB_OK) return st;
    }
    w->step_log.emplace_back(dt, substeps);
  }
  const float h = dt / float(substeps);
  const bool warm_first = (w->params.flags & BB_SIM_WARM_STARTING) && !w->skip_warm_once;
  const bool warm_rest = (w->params.flags & BB_SIM_WARM_STARTING) != 0;
  w->skip_warm_once = false;
  uint32_t hbits;
  std::memcpy(&hbits, &h, 4);
  auto key = std::make_tuple(substeps, w->parity, warm_first ? 1 : 0, w->n, fnv(&w->params, sizeof(w->params)), hbits);
  if (w->use_graphs && !w->profiling) {
    auto it = w->graphs.find(key);
    if (it == w->graphs.end()) {
      int parity0 = w->parity;
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        for (uint32_t s = 0; s < substeps; ++s) w->substep(h, s == 0 ? warm_first : warm_rest, 99, true);
        e = cudaStreamEndCapture(w->stream, &g);
      }
      w->parity = parity0;
      World::GraphEntry ge;
      if (e == cudaSuccess) e = cudaGraphInstantiate(&ge.exec, g, 0);
      if (e == cudaSuccess) {
        size_t nn = 0;
        cudaGraphGetNodes(g, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        cudaGraphGetNodes(g, nodes.data(), &nn);
        for (auto nd : nodes) {
          cudaGraphNodeType t;
          cudaGraphNodeGetType(nd, &t);
          if (t == cudaGraphNodeTypeKernel) ++ge.kernels;
        }
      }
      if (g) cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        cudaGetLastError();
        w->use_graphs = false;  // fall back to direct launches from now on
      } else {
        it = w->graphs.emplace(key, ge).first;
      }
    }
    if (w->use_graphs) {
      CU(cudaGraphLaunch(it->second.exec, w->stream));
      w->launches += it->second.kernels;
      for (uint32_t s = 0; s < substeps; ++s) w->parity ^= 1;
      w->last_cur = w->parity;
      w->ran_any = true;
      return BB_OK;
    }
  }
  if (w->profiling) {
    // per-stage timing: run the substeps stage by stage with events
    // the front end is split at its sort, tree build and refit (their own rooflines)
    static const char* names[] = {"morton", "sort", "lbvh_build", "refit", "broad_phase", "narrow_phase", "advect",
                                  "islands", "sleep", "edge_coloring", "solve"};
    constexpr int kStages = 11;
    if (w->stage_ms.size() != kStages) {
      w->stage_ms.assign(kStages, 0.f);
      w->stage_names.assign(names, names + kStages);
    }
    for (uint32_t s = 0; s < substeps; ++s) {
      const int cur = w->parity ^ 1;
      cudaEvent_t ev[kStages + 1];
      for (auto& e : ev) cudaEventCreate(&e);
      k_begin_substep<<<1, 32, 0, w->stream>>>(w->d.ctr);
      cudaMemsetAsync(w->scratch_base, 0, w->scratch_bytes, w->stream);
      cudaEventRecord(ev[0], w->stream);
      bb_front_end(w->stream, w->d, w->params, w->n, w->sc, w->sms, cur, w->max_world_bodies(), ev + 1);
      cudaEventRecord(ev[5], w->stream);
      bb_narrow_phase(w->stream, w->d, w->params, w->n, w->sc, w->sms, cur, s == 0 ? warm_first : warm_rest);
      cudaEventRecord(ev[6], w->stream);
      bb_advect(w->stream, w->d, w->params, w->n, h, w->sms);
      cudaEventRecord(ev[7], w->stream);
      bb_islands(w->stream, w->d, w->params, w->n, w->sc, w->sms, cur, w->coop_cc);
      cudaEventRecord(ev[8], w->stream);
      bb_sleep(w->stream, w->d, w->params, w->n, w->sms, cur);
      cudaEventRecord(ev[9], w->stream);
      const bool coloured = (w->params.flags & BB_SIM_USE_GRAPH_COLORING) != 0;
      if (coloured || w->params.solver == BB_SOLVER_AVBD)
        bb_edge_coloring(w->stream, w->d, w->params, w->n, w->sc, w->sms, cur, w->coop_edge);
      cudaEventRecord(ev[10], w->stream);
      if (w->params.solver == BB_SOLVER_AVBD) bb_solve_avbd(w->stream, w->d, w->params, w->n, h, w->sc, w->sms, cur, w->coop_avbd);
      else if (!coloured) bb_solve_islands(w->stream, w->d, w->params, w->n, h, cur, w->sc, w->sms);
      else bb_solve_pgs_soft(w->stream, w->d, w->params, w->n, h, cur, w->sc, w->coop_pgs, w->sms);
      cudaEventRecord(ev[11], w->stream);
      CU(cudaEventSynchronize(ev[11]));
      for (int k = 0; k < kStages; ++k) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
        w->stage_ms[k] += ms;
      }
      for (auto& e : ev) cudaEventDestroy(e);
      w->parity = cur;
      w->last_cur = cur;
    }
    w->ran_any = true;
    return BB_OK;
  }
  for (uint32_t s = 0; s < substeps; ++s) w->substep(h, s == 0 ? warm_first : warm_rest, 99, true);
  w->ran_any = true;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(BB_E_CUDA, std::string("bb_step: ") + cudaGetErrorString(e));
  return BB_OK;
}

bb_status bb_sync(void* world) {
  World* w = W(world);
  if (!w) return fail(BB_E_INVALID, "null world");
  CU(cudaStreamSynchronize(w->stream));
  uint32_t flags = 0;
  CU(cudaMemcpy(&flags, &w->d.ctr->error_flags, 4, cudaMemcpyDeviceToHost));
  // auto-regrow: a pair overflow in the steps since the last sync reruns them from the snapshot
  // with twice the pair capacity, as often as the limit allows
  while ((flags & (BB_ERRF_PAIR_OVERFLOW | BB_ERRF_CONTACT_OVERFLOW)) && w->regrow_max_ppb && w->snapped &&
         w->ppb < w->regrow_max_ppb) {
    bb_status st = w->regrow(std::min(2 * w->ppb, w->regrow_max_ppb));
    if (st != BB_OK) return st;
    const std::vector<std::pair<float, uint32_t>> log = w->step_log;
    w->step_log.clear();
    for (auto& s : log) {
      st = bb_step(world, s.first, s.second);
      if (st != BB_OK) return st;
    }
    CU(cudaStreamSynchronize(w->stream));
    CU(cudaMemcpy(&flags, &w->d.ctr->error_flags, 4, cudaMemcpyDeviceToHost));
  }
  if (!(flags & (BB_ERRF_PAIR_OVERFLOW | BB_ERRF_CONTACT_OVERFLOW))) w->forget_snapshot();
  if (flags & (BB_ERRF_PAIR_OVERFLOW | BB_ERRF_CONTACT_OVERFLOW))
    return fail(BB_E_CAPACITY, "pair capacity exceeded: create the world with a larger pairs_per_body");
  if (flags & (BB_ERRF_SPIN_LIMIT | BB_ERRF_STACK_OVERFLOW | BB_ERRF_CAS_LIMIT))
    return fail(BB_E_DEVICE_LIMIT, "a bounded device loop gave up (error flags " + std::to_string(flags) + ")");
  return BB_OK;
}

// Device pack + one async copy per array on the world's stream (host memory should be pinned
// for full PCIe / C2C bandwidth; pageable memory works, slower).
bb_status bb_read_state(void* world, float* position, float* rotation, float* velocity, float* omega) {
  World* w = W(world);
  if (!w) return fail(BB_E_INVALID, "null world");
  const uint32_t n = w->n;
  if (n == 0) return BB_OK;
  float* st = w->d.staging;
  k_pack_state<<<(n + 255) / 256, 256, 0, w->stream>>>(w->d, n, st);
  if (position) CU(cudaMemcpyAsync(position, st + 4ull * n, 12ull * n, cudaMemcpyDeviceToHost, w->stream));
  if (rotation) CU(cudaMemcpyAsync(rotation, st, 16ull * n, cudaMemcpyDeviceToHost, w->stream));
  if (velocity) CU(cudaMemcpyAsync(velocity, st + 7ull * n, 12ull * n, cudaMemcpyDeviceToHost, w->stream));
  if (omega) CU(cudaMemcpyAsync(omega, st + 10ull * n, 12ull * n, cudaMemcpyDeviceToHost, w->stream));
  CU(cudaStreamSynchronize(w->stream));
  return BB_OK;
}

bb_status bb_update_transforms(void* world) {
  World* w = W(world);
  if (!w) return fail(BB_E_INVALID, "null world");
  if (w->n) k_transforms<<<(w->n + 255) / 256, 256, 0, w->stream>>>(w->d, w->n, w->xforms);
  CU(cudaGetLastError());
  return BB_OK;
}

const float* bb_transforms_device(void* world) { return world ? W(world)->xforms : nullptr; }

bb_status bb_read_transforms(void* world, float* transforms) {
  World* w = W(world);
  if (!w || (!transforms && w->n)) return fail(BB_E_INVALID, "bb_read_transforms: bad arguments");
  bb_status st = bb_update_transforms(world);
  if (st != BB_OK) return st;
  if (w->n) CU(cudaMemcpyAsync(transforms, w->xforms, 48ull * w->n, cudaMemcpyDeviceToHost, w->stream));
  CU(cudaStreamSynchronize(w->stream));
  return BB_OK;
}

bb_status bb_read_contact_points(void* world, float* points, uint32_t max_points, uint32_t* count) {
  World* w = W(world);
  if (!w || !count || (!points && max_points)) return fail(BB_E_INVALID, "bb_read_contact_points: bad arguments");
  CU(cudaStreamSynchronize(w->stream));
  uint32_t M = 0;
  CU(cudaMemcpy(&M, &w->d.ctr->manifold_count, 4, cudaMemcpyDeviceToHost));
  *count = 0;
  if (!w->ran_any || M == 0) return BB_OK;
  const int cur = w->last_cur;
  k_contact_points<<<w->sms * 8, 256, 0, w->stream>>>(w->d, cur, w->d.c_r1);
  std::vector<float4> buf(size_t(M) * BB_MAX_CONTACTS);
  CU(cudaMemcpyAsync(buf.data(), w->d.c_r1, buf.size() * sizeof(float4), cudaMemcpyDeviceToHost, w->stream));
  CU(cudaStreamSynchronize(w->stream));
  uint32_t k = 0;
  for (const float4& c : buf) {
    if (c.w != c.w) continue;  // NaN: unused slot
    if (k < max_points) std::memcpy(points + 4 * size_t(k), &c, 16);
    ++k;
  }
  *count = k;
  return BB_OK;
}

bb_status bb_write_state(void* world, const float* position, const float* rotation, const float* velocity,
                         const float* omega) {
  World* w = W(world);
  if (!w) return fail(BB_E_INVALID, "null world");
  w->forget_snapshot();
  const uint32_t n = w->n;
  if (n == 0) return BB_OK;
  float* st = w->d.staging;
  uint32_t mask = 0;
  if (position) { CU(cudaMemcpyAsync(st + 4ull * n, position, 12ull * n, cudaMemcpyHostToDevice, w->stream)); mask |= 1; }
  if (rotation) { CU(cudaMemcpyAsync(st, rotation, 16ull * n, cudaMemcpyHostToDevice, w->stream)); mask |= 2; }
  if (velocity) { CU(cudaMemcpyAsync(st + 7ull * n, velocity, 12ull * n, cudaMemcpyHostToDevice, w->stream)); mask |= 4; }
  if (omega) { CU(cudaMemcpyAsync(st + 10ull * n, omega, 12ull * n, cudaMemcpyHostToDevice, w->stream)); mask |= 8; }
  k_unpack_state<<<(n + 255) / 256, 256, 0, w->stream>>>(w->d, n, st, mask);
  // moved poses: no body keeps last substep's manifolds as they were
  if (mask & 3u) {
    CU(cudaMemsetAsync(w->d.frozen, 0, 4ull * n, w->stream));
    CU(cudaMemsetAsync(&w->d.ctr->front_valid, 0, sizeof(uint32_t), w->stream));
  }
  // the caller may reuse its buffers as soon as this returns
  CU(cudaStreamSynchronize(w->stream));
  return BB_OK;
}

bb_status bb_read_flags(void* world, uint32_t* flags) {
  World* w = W(world);
  if (!w || !flags) return fail(BB_E_INVALID, "bad arguments");
  CU(cudaStreamSynchronize(w->stream));
  CU(cudaMemcpy(flags, w->d.flags, w->n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  return BB_OK;
}

bb_status bb_read_stats(void* world, bb_step_stats* s) {
  World* w = W(world);
  if (!w || !s) return fail(BB_E_INVALID, "bad arguments");
  CU(cudaStreamSynchronize(w->stream));
  DevCounters c;
  CU(cudaMemcpy(&c, w->d.ctr, sizeof(c), cudaMemcpyDeviceToHost));
  std::memset(s, 0, sizeof(*s));
  s->body_count = w->n;
  s->active_body_count = w->n_dyn;
  s->pair_count = c.pair_count;
  s->manifold_count = c.manifold_count;
  s->contact_count = c.contact_count;
  s->island_count = c.island_count;
  s->graph_color_count = c.gc_colors;
  s->graph_color_overflow = c.gc_overflow;
  s->graph_color_violations = c.gc_violations;
  s->avbd_color_count = c.avbd_colors;
  s->avbd_violations = c.avbd_violations;
  s->sleeping_count = c.sleeping;
  s->fresh_contacts = c.fresh;
  s->stick_count = c.stick;
  float mp;
  std::memcpy(&mp, &c.max_pen_bits, 4);
  s->max_penetration = mp;
  s->error_flags = c.error_flags;
  s->pair_capacity = w->cap_p;
  s->substeps_run = c.substeps;
  s->solved_manifolds = c.pgs_manifolds;
  s->solved_contacts = c.pgs_contacts;
  s->error_site = c.error_site;
  s->graph_color_rounds = c.gc_rounds_run;
  return BB_OK;
}

bb_status bb_debug_collide(void* world, uint32_t stage) {
  World* w = W(world);
  if (!w || stage < 1 || stage > 2) return fail(BB_E_INVALID, "bb_debug_collide: stage must be 1 or 2");
  if (w->n == 0) return BB_OK;
  bool warm = (w->params.flags & BB_SIM_WARM_STARTING) && !w->skip_warm_once;
  w->substep(0.0f, warm, stage, false);
  CU(cudaStreamSynchronize(w->stream));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(BB_E_CUDA, std::string("bb_debug_collide: ") + cudaGetErrorString(e));
  return BB_OK;
}

bb_status bb_debug_read(void* world, uint32_t which, void* dst, uint64_t max_bytes, uint64_t* count) {
  World* w = W(world);
  if (!w) return fail(BB_E_INVALID, "null world");
  CU(cudaStreamSynchronize(w->stream));
  DevCounters c;
  CU(cudaMemcpy(&c, w->d.ctr, sizeof(c), cudaMemcpyDeviceToHost));
  const uint32_t n = w->n;
  const int cur = w->last_cur;
  const uint32_t P = std::min(c.pair_count, w->cap_p), M = c.manifold_count;
  const uint32_t S = w->d.vox_on ? std::min(c.slot_count, w->cap_p) : P;  // manifold slots
  std::vector<uint8_t> out;
  uint64_t cnt = 0;
  auto grab = [&](const void* src, size_t bytes) -> bb_status {
    out.resize(bytes);
    if (bytes) CU(cudaMemcpy(out.data(), src, bytes, cudaMemcpyDeviceToHost));
    return BB_OK;
  };
  bb_status st = BB_OK;
  switch (which) {
    case BB_DBG_MORTON: {
      // keys[0] holds the sorted codes and vals[0] the ids: scatter back to id order
      std::vector<uint32_t> keys(n), ids(n);
      CU(cudaMemcpy(keys.data(), w->d.keys[0], n * 4, cudaMemcpyDeviceToHost));
      CU(cudaMemcpy(ids.data(), w->d.vals[0], n * 4, cudaMemcpyDeviceToHost));
      std::vector<uint32_t> by_id(n);
      for (uint32_t i = 0; i < n; ++i) by_id[ids[i]] = keys[i];
      out.resize(4 * n);
      std::memcpy(out.data(), by_id.data(), 4 * n);
      cnt = n;
      break;
    }
    case BB_DBG_SORTED_KEYS: st = grab(w->d.keys[0], 4 * n); cnt = n; break;
    case BB_DBG_SORTED_IDS: st = grab(w->d.vals[0], 4 * n); cnt = n; break;
    case BB_DBG_LBVH_CHILD: st = grab(w->d.child, n > 1 ? 8 * (n - 1) : 0); cnt = n > 1 ? 2 * (n - 1) : 0; break;
    case BB_DBG_LEAF_AABB:
    case BB_DBG_NODE_AABB: {
      uint32_t first = which == BB_DBG_LEAF_AABB ? n - 1 : 0, count_ = which == BB_DBG_LEAF_AABB ? n : (n > 0 ? n - 1 : 0);
      std::vector<float4> box(2 * count_);
      if (count_) CU(cudaMemcpy(box.data(), w->d.node_box + 2 * first, box.size() * sizeof(float4), cudaMemcpyDeviceToHost));
      out.resize(24 * count_);
      float* o = reinterpret_cast<float*>(out.data());
      for (uint32_t i = 0; i < count_; ++i) {
        o[6 * i] = box[2 * i].x; o[6 * i + 1] = box[2 * i].y; o[6 * i + 2] = box[2 * i].z;
        o[6 * i + 3] = box[2 * i + 1].x; o[6 * i + 4] = box[2 * i + 1].y; o[6 * i + 5] = box[2 * i + 1].z;
      }
      cnt = 6ull * count_;
      break;
    }
    case BB_DBG_PAIRS: st = grab(w->d.pairs, 8ull * P); cnt = 2ull * P; break;
    case BB_DBG_MANIFOLDS:
    case BB_DBG_CONTACTS:
    case BB_DBG_EDGE_COLORS: {
      std::vector<uint32_t> slot(M), color(M);
      if (M) CU(cudaMemcpy(slot.data(), w->d.man_slot[cur], 4 * M, cudaMemcpyDeviceToHost));
      if (which == BB_DBG_EDGE_COLORS) {
        if (M) CU(cudaMemcpy(color.data(), w->d.gc_color, 4 * M, cudaMemcpyDeviceToHost));
        out.resize(4 * M);
        std::memcpy(out.data(), color.data(), 4 * M);
        cnt = M;
        break;
      }
      if (which == BB_DBG_MANIFOLDS) {
        std::vector<uint2> bodies(S);
        std::vector<int2> kc(S);
        std::vector<float4> nrm(S), t0(S), t1(S);
        if (S) {
          CU(cudaMemcpy(bodies.data(), w->d.m_bodies[cur], 8 * S, cudaMemcpyDeviceToHost));
          CU(cudaMemcpy(kc.data(), w->d.m_keycc[cur], 8 * S, cudaMemcpyDeviceToHost));
          CU(cudaMemcpy(nrm.data(), w->d.m_normal[cur], 16 * S, cudaMemcpyDeviceToHost));
          CU(cudaMemcpy(t0.data(), w->d.m_t0[cur], 16 * S, cudaMemcpyDeviceToHost));
          CU(cudaMemcpy(t1.data(), w->d.m_t1[cur], 16 * S, cudaMemcpyDeviceToHost));
        }
        if (M) CU(cudaMemcpy(color.data(), w->d.gc_color, 4 * M, cudaMemcpyDeviceToHost));
        out.resize(sizeof(bb_manifold_info) * M);
        bb_manifold_info* mi = reinterpret_cast<bb_manifold_info*>(out.data());
        for (uint32_t m = 0; m < M; ++m) {
          uint32_t s = slot[m];
          mi[m].body_a = bodies[s].x;
          mi[m].body_b = bodies[s].y;
          mi[m].key = kc[s].x;
          mi[m].contact_count = kc[s].y;
          mi[m].normal[0] = nrm[s].x; mi[m].normal[1] = nrm[s].y; mi[m].normal[2] = nrm[s].z;
          mi[m].color = color[m];
          mi[m].tangent[0][0] = t0[s].x; mi[m].tangent[0][1] = t0[s].y; mi[m].tangent[0][2] = t0[s].z;
          mi[m].tangent[1][0] = t1[s].x; mi[m].tangent[1][1] = t1[s].y; mi[m].tangent[1][2] = t1[s].z;
        }
        cnt = M;
        break;
      }
      const size_t C = size_t(S) * BB_MAX_CONTACTS;
      std::vector<float4> cp(C), cl(C), ck(C), ca(C);
      std::vector<int2> kc(S);
      if (S) {
        CU(cudaMemcpy(cp.data(), w->d.c_pos[cur], 16 * C, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(cl.data(), w->d.c_lam[cur], 16 * C, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(ck.data(), w->d.c_kt[cur], 16 * C, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(ca.data(), w->d.c_anc_a[cur], 16 * C, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(kc.data(), w->d.m_keycc[cur], 8 * S, cudaMemcpyDeviceToHost));
      }
      out.assign(sizeof(bb_contact_info) * 8 * size_t(M), 0);
      bb_contact_info* ci = reinterpret_cast<bb_contact_info*>(out.data());
      for (uint32_t m = 0; m < M; ++m) {
        uint32_t s = slot[m];
        for (int j = 0; j < kc[s].y; ++j) {
          size_t k = size_t(s) * BB_MAX_CONTACTS + j;
          bb_contact_info& o = ci[8 * size_t(m) + j];
          o.position[0] = cp[k].x; o.position[1] = cp[k].y; o.position[2] = cp[k].z;
          o.penetration = cp[k].w;
          o.normal_impulse = cl[k].x;
          o.tangent_impulse[0] = cl[k].y;
          o.tangent_impulse[1] = cl[k].z;
          std::memcpy(&o.feature, &ca[k].w, 4);
          std::memcpy(&o.warm_start, &ck[k].w, 4);
          o.penalty = cl[k].w;
        }
      }
      cnt = 8ull * M;
      break;
    }
    case BB_DBG_BODY_COLORS: st = grab(w->d.body_color, 4 * n); cnt = n; break;
    case BB_DBG_ISLANDS: st = grab(w->d.island, 4 * n); cnt = n; break;
    case BB_DBG_SUPPORT_DEPTH: st = grab(w->d.a_depth, 4 * n); cnt = n; break;
    case BB_DBG_BODY_INERTIA: {
      std::vector<float4> ii(n), io(n);
      if (n) {
        CU(cudaMemcpy(ii.data(), w->d.iinv, 16ull * n, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(io.data(), w->d.iinv_off, 16ull * n, cudaMemcpyDeviceToHost));
      }
      out.resize(24ull * n);
      float* o = reinterpret_cast<float*>(out.data());
      for (uint32_t i = 0; i < n; ++i) {
        o[6 * i] = ii[i].x; o[6 * i + 1] = ii[i].y; o[6 * i + 2] = ii[i].z;
        o[6 * i + 3] = io[i].x; o[6 * i + 4] = io[i].y; o[6 * i + 5] = io[i].z;
      }
      cnt = 6ull * n;
      break;
    }
    default: return fail(BB_E_INVALID, "bb_debug_read: unknown buffer");
  }
  if (st != BB_OK) return st;
  if (dst) std::memcpy(dst, out.data(), std::min<uint64_t>(out.size(), max_bytes));
  if (count) *count = cnt;
  return BB_OK;
}

// ---- saved state ----------------------------------------------------------------------------
// Image of a world: a header with the host fields that steer the next step, the byte size of
// every device array in allocation order, then the arrays themselves (and the voxel slot buffer).
// Loading it into a world created with the same capacity and holding the same bodies (same
// shapes, same order, hence the same allocation sequence) restores every bit the step reads:
// poses, velocities, flags and sleep timers, both manifold buffers with their contacts,
// impulses and anchors, per-body lists, sort order, frozen bits, last island roots, counters.

bb_status bb_world_save_state(void* world, void* dst, uint64_t max_bytes, uint64_t* bytes) {
  World* w = W(world);
  if (!w || !bytes) return fail(BB_E_INVALID, "bb_world_save_state: bad arguments");
  const uint64_t total = state_bytes(w);
  *bytes = total;
  if (!dst) return BB_OK;
  if (max_bytes < total) return fail(BB_E_INVALID, "bb_world_save_state: buffer smaller than the state");
  CU(cudaStreamSynchronize(w->stream));
  StateHeader h{};
  h.magic = kStateMagic;
  h.version = kStateVersion;
  h.cap_n = w->cap_n;
  h.cap_p = w->cap_p;
  h.n = w->n;
  h.n_dyn = w->n_dyn;
  h.n_worlds = w->d.n_worlds;
  h.vox_on = w->d.vox_on;
  h.full_inertia = w->d.full_inertia;
  h.parity = w->parity;
  h.last_cur = w->last_cur;
  h.ran_any = w->ran_any ? 1u : 0u;
  h.skip_warm_once = w->skip_warm_once ? 1u : 0u;
  h.arrays = uint32_t(w->owned.size());
  h.slot_bytes = w->slot_buf ? 16ull * w->cap_p : 0ull;
  h.total = total;
  h.params = w->params;
  char* out = static_cast<char*>(dst);
  std::memcpy(out, &h, sizeof(h));
  uint64_t* sizes = reinterpret_cast<uint64_t*>(out + sizeof(h));
  char* p = out + sizeof(h) + 8ull * w->owned.size();
  for (size_t k = 0; k < w->owned.size(); ++k) {
    sizes[k] = w->owned[k].second;
    CU(cudaMemcpyAsync(p, w->owned[k].first, w->owned[k].second, cudaMemcpyDeviceToHost, w->stream));
    p += w->owned[k].second;
  }
  if (h.slot_bytes) CU(cudaMemcpyAsync(p, w->slot_buf, h.slot_bytes, cudaMemcpyDeviceToHost, w->stream));
  CU(cudaStreamSynchronize(w->stream));
  return BB_OK;
}

bb_status bb_world_load_state(void* world, const void* src, uint64_t bytes) {
  World* w = W(world);
  if (!w || !src || bytes < sizeof(StateHeader)) return fail(BB_E_INVALID, "bb_world_load_state: bad arguments");
  StateHeader h;
  std::memcpy(&h, src, sizeof(h));
  if (h.magic != kStateMagic || h.total != bytes)
    return fail(BB_E_INVALID, "bb_world_load_state: not a saved world state");
  if (h.version != kStateVersion)
    return fail(BB_E_INVALID, "bb_world_load_state: saved by another version of the library (different arrays)");
  if (h.cap_n != w->cap_n || h.cap_p != w->cap_p || h.n != w->n || h.n_dyn != w->n_dyn ||
      h.n_worlds != w->d.n_worlds || h.vox_on != w->d.vox_on || h.full_inertia != w->d.full_inertia ||
      h.arrays != w->owned.size() || h.slot_bytes != (w->slot_buf ? 16ull * w->cap_p : 0ull) ||
      state_bytes(w) != bytes)
    return fail(BB_E_INVALID,
                "bb_world_load_state: the world differs from the saved one (create it with the same capacity and "
                "add the same bodies first)");
  const char* in = static_cast<const char*>(src);
  const uint64_t* sizes = reinterpret_cast<const uint64_t*>(in + sizeof(h));
  for (size_t k = 0; k < w->owned.size(); ++k)
    if (sizes[k] != w->owned[k].second) return fail(BB_E_INVALID, "bb_world_load_state: array sizes differ");
  CU(cudaStreamSynchronize(w->stream));
  w->forget_snapshot();
  const char* p = in + sizeof(h) + 8ull * w->owned.size();
  for (auto& o : w->owned) {
    CU(cudaMemcpyAsync(o.first, p, o.second, cudaMemcpyHostToDevice, w->stream));
    p += o.second;
  }
  if (h.slot_bytes) CU(cudaMemcpyAsync(w->slot_buf, p, h.slot_bytes, cudaMemcpyHostToDevice, w->stream));
  CU(cudaStreamSynchronize(w->stream));
  w->parity = h.parity;
  w->last_cur = h.last_cur;
  w->ran_any = h.ran_any != 0;
  w->skip_warm_once = h.skip_warm_once != 0;
  w->params = h.params;
  w->invalidate_graphs();
  return BB_OK;
}

bb_status bb_world_set_auto_regrow(void* world, uint32_t max_pairs_per_body) {
  World* w = W(world);
  if (!w) return fail(BB_E_INVALID, "bb_world_set_auto_regrow: null world");
  if (max_pairs_per_body && max_pairs_per_body < w->ppb)
    return fail(BB_E_INVALID, "bb_world_set_auto_regrow: the limit is below the current pairs per body");
  CU(cudaStreamSynchronize(w->stream));
  w->regrow_max_ppb = max_pairs_per_body;
  w->forget_snapshot();
  if (!max_pairs_per_body && w->shadow) {
    cudaFree(w->shadow);
    w->shadow = nullptr;
    w->shadow_cap = 0;
  }
  return BB_OK;
}

bb_status bb_debug_wait_limit(void* world, uint32_t polls, uint32_t abandon_block) {
  World* w = W(world);
  if (!w) return fail(BB_E_INVALID, "null world");
  const uint32_t v[2] = {polls, abandon_block ? 1u : 0u};
  CU(cudaMemcpyAsync(&w->d.ctr->wait_limit, v, sizeof(v), cudaMemcpyHostToDevice, w->stream));
  CU(cudaStreamSynchronize(w->stream));
  return BB_OK;
}

bb_status bb_set_profiling(void* world, int32_t enabled) {
  World* w = W(world);
  if (!w) return fail(BB_E_INVALID, "null world");
  w->profiling = enabled != 0;
  w->stage_ms.assign(w->stage_ms.size(), 0.f);
  return BB_OK;
}

bb_status bb_read_stage_times(void* world, float* ms, uint32_t max_stages, uint32_t* n_stages, char* names,
                              uint32_t names_bytes) {
  World* w = W(world);
  if (!w) return fail(BB_E_INVALID, "null world");
  CU(cudaStreamSynchronize(w->stream));
  uint32_t ns = uint32_t(w->stage_ms.size());
  if (n_stages) *n_stages = ns;
  for (uint32_t k = 0; k < ns && k < max_stages && ms; ++k) ms[k] = w->stage_ms[k];
  if (names && names_bytes) {
    std::string all;
    for (auto& s : w->stage_names) {
      all += s;
      all.push_back('\0');
    }
    std::memcpy(names, all.data(), std::min<size_t>(all.size(), names_bytes));
  }
  return BB_OK;
}

uint64_t bb_kernel_launch_count(void* world) { return world ? W(world)->launches : 0; }

}  // extern "C"

// Serving: the first `count` bodies of world `src_widx` of batch `src` moved into slot `widx` of
// batch `dst` by device copies, with new Morton bounds -- the same bodies a bb_world_refill with
// their current state would write, without the round trip through host memory.  Both batches
// must step on one stream (the copy is ordered after the source's queued steps and before the
// destination's next).  The destination slot restarts as a refilled slot does; the source slot
// is left as it is (the caller reuses it).
bb_status bb_world_move_in(void* dst_world, uint32_t widx, const bb_batch_world_desc* desc, void* src_world,
                           uint32_t src_widx, uint32_t count) {
  World* w = W(dst_world);
  World* s = W(src_world);
  if (!w || !s || !desc || w == s) return fail(BB_E_INVALID, "bb_world_move_in: bad arguments");
  if (w->stream != s->stream) return fail(BB_E_INVALID, "bb_world_move_in: the batches step on different streams");
  if (w->d.n_worlds == 0 || widx >= w->wfirst.size() || s->d.n_worlds == 0 || src_widx >= s->wfirst.size())
    return fail(BB_E_INVALID, "bb_world_move_in: not a world of these batches");
  const uint32_t first = w->wfirst[widx], slot = w->wcount[widx], src_first = s->wfirst[src_widx];
  if (count > slot || count > s->wcount[src_widx])
    return fail(BB_E_CAPACITY, "bb_world_move_in: more bodies than the slot holds");
  w->forget_snapshot();
  const uint32_t tbits = BB_SHAPE_BOX;
  float tf;
  std::memcpy(&tf, &tbits, 4);
  k_move_bodies<<<(slot + 255) / 256, 256, 0, w->stream>>>(
      w->d, s->d, first, src_first, count, slot, make_float3(desc->world_min[0], desc->world_min[1], desc->world_min[2]),
      make_float4(0.001f, 0.001f, 0.001f, tf));
  for (uint32_t i = 0; i < slot; ++i) w->restitution[first + i] = i < count ? s->restitution[src_first + i] : 0.f;
  const uint32_t ndyn = s->wdyn[src_widx];
  w->n_dyn = w->n_dyn - w->wdyn[widx] + ndyn;
  w->wdyn[widx] = ndyn;
  if (s->d.full_inertia) w->d.full_inertia = 1;
  k_set_world<<<1, 1, 0, w->stream>>>(w->d, widx, first, slot,
                                      make_float4(desc->world_min[0], desc->world_min[1], desc->world_min[2], 0.f),
                                      make_float4(desc->world_extent[0], desc->world_extent[1], desc->world_extent[2], 0.f));
  k_refill_contacts<<<(slot + 255) / 256, 256, 0, w->stream>>>(w->d, first, slot);
  k_set_counts<<<1, 1, 0, w->stream>>>(w->d, w->n, w->n_dyn);
  CU(cudaGetLastError());
  return BB_OK;
}


// State of bodies [first, first + count) (the serving loop's view of one batch slot): xyz
// positions, xyzw rotations, velocities, angular velocities, flags (may each be null).
bb_status bb_world_read_range(void* world, uint32_t first, uint32_t count, float* position, float* rotation,
                              float* velocity, float* omega, uint32_t* flags) {
  World* w = W(world);
  if (!w || uint64_t(first) + count > w->n) return fail(BB_E_INVALID, "bb_world_read_range: bad range");
  if (count == 0) return BB_OK;
  float* st = w->d.staging;
  uint32_t* fl = reinterpret_cast<uint32_t*>(st + 13ull * count);
  k_pack_range<<<(count + 255) / 256, 256, 0, w->stream>>>(w->d, first, count, st, fl);
  if (position) CU(cudaMemcpyAsync(position, st + 4ull * count, 12ull * count, cudaMemcpyDeviceToHost, w->stream));
  if (rotation) CU(cudaMemcpyAsync(rotation, st, 16ull * count, cudaMemcpyDeviceToHost, w->stream));
  if (velocity) CU(cudaMemcpyAsync(velocity, st + 7ull * count, 12ull * count, cudaMemcpyDeviceToHost, w->stream));
  if (omega) CU(cudaMemcpyAsync(omega, st + 10ull * count, 12ull * count, cudaMemcpyDeviceToHost, w->stream));
  if (flags) CU(cudaMemcpyAsync(flags, fl, 4ull * count, cudaMemcpyDeviceToHost, w->stream));
  CU(cudaStreamSynchronize(w->stream));
  return BB_OK;
}

// device word of the world's sticky error bits (BB_ERRF_*)
const uint32_t* bb_world_error_word(void* world) { return world ? &W(world)->d.ctr->error_flags : nullptr; }
const uint32_t* bb_world_error_site_word(void* world) { return world ? &W(world)->d.ctr->error_site : nullptr; }


// ---- autotuner ------------------------------------------------------------------------------
// Coordinate descent over the launch-geometry fields and the colour-sweep schedule of
// bb_solver_params.  Every candidate computes bit-identical results, so the trial steps are
// ordinary steps of the world (they advance it; call this in place of warm-up steps).  Each
// candidate gets one untimed step (graph capture) and `trial_steps` steps timed with CUDA
// events on the world's stream.
bb_status bb_autotune(void* world, float dt, uint32_t substeps, uint32_t trial_steps, bb_solver_params* chosen) {
  World* w = W(world);
  if (!w || !(dt > 0) || substeps == 0 || trial_steps == 0) return fail(BB_E_INVALID, "bb_autotune: bad arguments");
  if (w->n == 0) {
    if (chosen) *chosen = w->params;
    return BB_OK;
  }
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  bb_solver_params best = w->params;
  auto trial = [&](const bb_solver_params& cand, float* ms) -> bb_status {
    bb_status st = bb_set_solver_params(world, &cand);
    if (st != BB_OK) return st;
    st = bb_step(world, dt, substeps);
    if (st != BB_OK) return st;
    CU(cudaEventRecord(e0, w->stream));
    for (uint32_t k = 0; k < trial_steps; ++k) {
      st = bb_step(world, dt, substeps);
      if (st != BB_OK) return st;
    }
    CU(cudaEventRecord(e1, w->stream));
    CU(cudaEventSynchronize(e1));
    CU(cudaEventElapsedTime(ms, e0, e1));
    return bb_sync(world);
  };
  bb_status st = BB_OK;
  struct Axis {
    uint32_t bb_solver_params::*field;
    std::vector<uint32_t> values;
    bool pgs_only, barrier_only;
  };
  const std::vector<Axis> axes = {
      {&bb_solver_params::schedule, {BB_SCHEDULE_DATAFLOW, BB_SCHEDULE_COLOUR_BARRIER}, true, false},
      {&bb_solver_params::broad_threads, {32, 64, 128}, false, false},
      {&bb_solver_params::narrow_blocks_per_sm, {4, 8, 16, 32}, false, false},
      {&bb_solver_params::pgs_stage_next, {0, 1}, true, true},
  };
  for (const Axis& ax : axes) {
    if (st != BB_OK) break;
    if (ax.pgs_only && best.solver != BB_SOLVER_PGS_SOFT) continue;
    if (ax.barrier_only && best.schedule != BB_SCHEDULE_COLOUR_BARRIER) continue;
    for (uint32_t v : ax.values) {
      if (best.*ax.field == v) continue;
      bb_solver_params cand = best;
      cand.*ax.field = v;
      // the world's step cost drifts as it evolves, so the candidate runs between two runs of
      // the incumbent and is compared with their mean
      float before = 0.f, ms = 0.f, after = 0.f;
      st = trial(best, &before);
      if (st == BB_OK) st = trial(cand, &ms);
      if (st == BB_OK) st = trial(best, &after);
      if (st != BB_OK) break;
      if (ms < 0.5f * (before + after)) best = cand;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != BB_OK) return st;
  st = bb_set_solver_params(world, &best);
  if (chosen) *chosen = best;
  return st;
}
