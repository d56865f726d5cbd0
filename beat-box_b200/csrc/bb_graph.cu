// bb_graph.cu -- advect, union-find islands, neighbourhood sleeping, edge colouring of the
// contact graph and the colour buckets the PGS sweeps run over.
//
// Reference: entry_rigid_body_sim / RigidBody::advect (src/shaders/simulation/RB_sim.slang:
// 518-554, src/shaders/extensions.slang:127-139); IslandBuilder (src/shaders/simulation/
// islands.slang:153-302); entry_sleep_reduce/veto/apply (RB_sim.slang:556-737); graph
// colouring (src/shaders/simulation/coloring.slang:25-292, rounds RBM:1332-1342).
//
// B200 design: the 32 bid/commit colouring rounds (96 dispatches in the reference) run in
// one persistent cooperative kernel with a grid barrier between phases and stop as soon as
// every manifold is coloured.  The per-(body, colour) owner cell holds (epoch << 32 | prio)
// in 64 bits, so it never needs the reference's per-round reset pass.  The colour buckets
// are one stable onesweep pass keyed by colour, so every colour sweep later reads a compact
// list instead of scanning all manifolds (RB_sim.slang:1416-1419).
#include "bb_common.cuh"
#include "bb_kernels.cuh"

// ---- advect (PGS family) ---------------------------------------------------------------------
__global__ void k_advect(const DevState d, Params p, uint32_t n, float h) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t f = d.flags[i];
  if (!(f & BB_BODY_DYNAMIC) || (f & BB_BODY_SLEEPING)) return;
  float4 v = d.vel[i];
  if (f & BB_BODY_GRAVITY) {
    float dv = p.gravity * h;
    if (p.quirks & BB_QUIRK_GRAVITY_IMPULSE) dv *= d.pos[i].w;  // impulse g*dt scaled by 1/m
    v.y += dv;
  }
  float lin = expf(-h * p.linear_damping), ang = expf(-h * p.angular_damping);
  d.vel[i] = make_float4(v.x * lin, v.y * lin, v.z * lin, v.w);
  float4 w = d.omega[i];
  d.omega[i] = make_float4(w.x * ang, w.y * ang, w.z * ang, w.w);
}

void bb_advect(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, float h, int sms) {
  (void)sms;
  if (p.solver == BB_SOLVER_AVBD || !(p.flags & BB_SIM_ADVECTION) || n == 0) return;
  k_advect<<<(n + BB_THREADS - 1) / BB_THREADS, BB_THREADS, 0, s>>>(d, p, n, h);
}

// ---- islands ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t ld_relaxed_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_gpu(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Connected components in synchronous rounds inside one persistent kernel (counter 7 of the
// substep's grid barriers): every round hooks, for each contact between two dynamic bodies,
// the larger of the two parents under the smaller (atomicMin, so parents only decrease and
// the forest stays acyclic), then lets every body jump one level (parent <- grandparent).  At
// the fixpoint every body points at the smallest id of its component -- the same roots as the
// reference's link-to-lower union-find (islands.slang:153-213) -- after O(log diameter)
// rounds, with no serial walk of a long chain by any one thread.
#define BB_CC_THREADS 512
#define BB_CC_MAX_ROUNDS 96u
__global__ void __launch_bounds__(BB_CC_THREADS, 1) k_components(const DevState d, int cur, uint32_t n) {
  DevCounters* c = d.ctr;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  const uint32_t M = c->manifold_count;
  uint32_t* sync = &c->sync_count[7];
  uint32_t* changed = c->round_flags;  // two alternating per-round flags (the AVBD colouring reuses them later)
  uint32_t ep = 0;
  uint32_t* parent = d.uf_parent;
  // Start from the last substep's roots where that is exact.  A last-substep component whose
  // bodies are all dynamic and were not awake at either narrow phase (frozen bit 1) keeps every
  // one of its manifolds (two such bodies keep their poses, so their pairs and manifolds
  // persist), so it lies inside one component now, and its root (its smallest id) is a valid
  // parent for its bodies: parents stay <= ids within the component, and the rounds below
  // converge to the same smallest ids.  Every other body starts alone, and any body that is not
  // such a body marks its old root, so its old component starts over.  Marks carry this
  // substep's number; a stale mark or a stray old parent can only make a component start over.
  const uint32_t mark = c->substeps;
  for (uint32_t i = tid; i < n; i += stride) {
    const bool keep = (d.flags[i] & BB_BODY_DYNAMIC) && (d.frozen[i] & 2u);
    const uint32_t old = parent[i];
    if (!keep && old < n) d.cc_mark[old] = mark;
  }
  if (tid == 0) {
    changed[0] = 0;
    changed[1] = 0;
  }
  grid_sync(c, sync, ep);
  for (uint32_t i = tid; i < n; i += stride) {  // each thread reads and writes only parent[i]
    const bool dyn = d.flags[i] & BB_BODY_DYNAMIC;
    const uint32_t old = parent[i];
    const bool keep = dyn && (d.frozen[i] & 2u) && old < n && d.cc_mark[old] != mark;
    parent[i] = !dyn ? BB_NONE : keep ? old : i;
  }
  grid_sync(c, sync, ep);
  uint32_t r = 0;
  for (; r < BB_CC_MAX_ROUNDS; ++r) {
    uint32_t any = 0;
    for (uint32_t m = tid; m < M; m += stride) {
      const uint2 b = d.m_bodies[cur][d.man_slot[cur][m]];
      const uint32_t pa = ld_relaxed_gpu(&parent[b.x]), pb = ld_relaxed_gpu(&parent[b.y]);
      if (pa == BB_NONE || pb == BB_NONE || pa == pb) continue;
      atomicMin(&parent[max(pa, pb)], min(pa, pb));
      any = 1;
    }
    grid_sync(c, sync, ep);
    for (uint32_t i = tid; i < n; i += stride) {
      const uint32_t p = parent[i];
      if (p == BB_NONE) continue;
      const uint32_t pp = ld_relaxed_gpu(&parent[p]);
      if (pp != p) {  // only this thread writes parent[i] in this pass
        st_relaxed_gpu(&parent[i], pp);
        any = 1;
      }
    }
    if (any) atomicOr(&changed[r & 1], 1u);
    grid_sync(c, sync, ep);
    const bool more = *(volatile uint32_t*)&changed[r & 1] != 0u;
    if (tid == 0) changed[(r + 1) & 1] = 0;
    if (!more) break;
    grid_sync(c, sync, ep);  // the reset above lands before anyone flags the next round
  }
  if (r == BB_CC_MAX_ROUNDS && tid == 0) raise_error(c, BB_ERRF_CAS_LIMIT);
  for (uint32_t i = tid; i < n; i += stride) {
    const uint32_t p = parent[i];
    d.island[i] = p;  // root; rank applied by k_island_ids
    d.is_root[i] = p == i ? 1u : 0u;
  }
}

__global__ void k_island_ids(const DevState d, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  d.island[i] = d.uf_parent[i] == BB_NONE ? BB_NONE : d.root_rank[d.island[i]];
}

int bb_components_blocks(int sms) { return bb_coop_blocks((const void*)k_components, BB_CC_THREADS, sms); }

void bb_islands(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, const StepScratch& sc, int sms,
                int cur, int coop_blocks) {
  (void)p;
  (void)sms;
  if (n == 0) return;
  const int T = BB_THREADS;
  uint32_t blocks = (n + T - 1) / T;
  DevState dd = d;
  int cc = cur;
  uint32_t nn = n;
  void* args[] = {&dd, &cc, &nn};
  bb_launch_coop((const void*)k_components, coop_blocks, BB_CC_THREADS, args, s);
  bb_launch_scan(s, d.is_root, d.root_rank, nullptr, n, &d.ctr->island_count, sc.scan_status + 3 * sc.scan_tiles,
                 sc.scan_tile_ctr + 3, d.ctr);
  k_island_ids<<<blocks, T, 0, s>>>(d, n);
}

// ---- sleeping (RB_sim.slang:556-737) --------------------------------------------------------
__global__ void k_sleep_reduce(const DevState d, Params p, uint32_t n, int cur) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t f = d.flags[i];
  if (!(f & BB_BODY_DYNAMIC) || (f & BB_BODY_PAUSED)) return;  // a paused world keeps its timers
  if (!(p.flags & BB_SIM_SLEEPING_ENABLED)) {
    d.sleep[i] = 0;
    d.flags[i] = f & ~BB_BODY_SLEEPING;
    return;
  }
  bool contactless = d.csr_start[cur][i] == d.csr_start[cur][i + 1];
  if (contactless && (f & BB_BODY_SLEEPING)) {
    uint32_t t = d.sleep[i] & BB_SLEEP_MASK;
    d.sleep[i] = t >= 10u ? t - 10u : 0u;
    return;
  }
  float3 v = f3(d.vel[i]), w = f3(d.omega[i]);
  float lin2 = dot3(v, v), ang2 = dot3(w, w);
  uint32_t timer = d.sleep[i] & BB_SLEEP_MASK;
  bool calm = lin2 < p.sleep_lin_vel2 && ang2 < p.sleep_ang_vel2;
  d.sleep[i] = calm ? min(timer + 1u, p.sleep_steps) : (timer >= 4u ? timer - 4u : 0u);
}
__global__ void k_sleep_veto(const DevState d, Params p, int cur) {
  const uint32_t M = d.ctr->manifold_count;
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    uint32_t slot = d.man_slot[cur][m];
    uint2 b = d.m_bodies[cur][slot];
    uint32_t fa = d.flags[b.x], fb = d.flags[b.y];
    if ((fa | fb) & BB_BODY_PAUSED) continue;
    bool ad = fa & BB_BODY_DYNAMIC, bd = fb & BB_BODY_DYNAMIC;
    bool a_loud = ad && (d.sleep[b.x] & BB_SLEEP_MASK) < p.sleep_steps;
    bool b_loud = bd && (d.sleep[b.y] & BB_SLEEP_MASK) < p.sleep_steps;
    int32_t err = __float_as_int(d.m_normal[cur][slot].w);
    bool stalled = err != 0x7FFFFFFF && abs(err) < 10;
    bool deep = false;
    if (!stalled) {
      int cc = d.m_keycc[cur][slot].y;
      for (int c = 0; c < cc; ++c)
        if (d.c_pos[cur][slot * BB_MAX_CONTACTS + c].w < -0.05f) {
          deep = true;
          break;
        }
    }
    if ((a_loud || deep) && bd) atomicOr(&d.sleep[b.y], BB_SLEEP_VETO);
    if ((b_loud || deep) && ad) atomicOr(&d.sleep[b.x], BB_SLEEP_VETO);
  }
}
__global__ void k_sleep_apply(const DevState d, uint32_t n, Params p) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) d.ctr->sleep_ran = 1u;  // with awake_after: the next substep may skip its front end
  if (i >= n) return;
  uint32_t f = d.flags[i];
  if (!(f & BB_BODY_DYNAMIC) || (f & BB_BODY_PAUSED)) return;
  uint32_t t = d.sleep[i];
  bool vetoed = (t & BB_SLEEP_VETO) != 0;
  bool quiet = (t & BB_SLEEP_MASK) >= p.sleep_steps;
  bool was = (f & BB_BODY_SLEEPING) != 0;
  if (quiet && !vetoed) {
    if (!was) {
      float4 v = d.vel[i];
      d.vel[i] = make_float4(0.f, 0.f, 0.f, v.w);
      d.omega[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      d.flags[i] = f | BB_BODY_SLEEPING;
    }
    atomicAdd(&d.ctr->sleeping, 1u);
  } else {
    if (was) d.flags[i] = f & ~BB_BODY_SLEEPING;
    if (d.ctr->awake_after == 0u) d.ctr->awake_after = 1u;  // this body is integrated: poses move
  }
}

void bb_sleep(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, int sms, int cur) {
  if (n == 0) return;
  const int T = BB_THREADS;
  uint32_t blocks = (n + T - 1) / T;
  k_sleep_reduce<<<blocks, T, 0, s>>>(d, p, n, cur);
  if (!(p.flags & BB_SIM_SLEEPING_ENABLED)) return;
  k_sleep_veto<<<sms * 8, T, 0, s>>>(d, p, cur);
  k_sleep_apply<<<blocks, T, 0, s>>>(d, n, p);
}

// ---- edge colouring ------------------------------------------------------------------------
__device__ __forceinline__ uint32_t gc_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ uint32_t gc_priority(uint32_t pid, uint32_t round) {
  uint32_t h = gc_hash(pid + round * 0x85ebca6bu) & 0xFFFu;
  if (h == 0u) h = 1u;
  return (h << 20) | (pid & 0xFFFFFu);
}

// Persistent cooperative kernel: init, then rounds r = 1..gc_rounds of
//   bid:    every uncoloured manifold takes the lowest colour free on both dynamic bodies
//           (gc_pick_color, coloring.slang:95-103) and atomically maxes its priority
//           (gc_priority, :130-138) into owner[body][colour];
//   commit: a manifold that won on both bodies takes the colour (:179-212).
// Finally writes the (colour, manifold) keys of the bucket sort.
// Persistent colouring kernel.  Each manifold's bodies, static bits and pair hash are packed
// into one record up front, so a round touches rec -> body masks -> owner words only; the
// grid barrier is the arrival-counter kind (counter 0 of the substep).
#define BB_GC_THREADS 1024
#define GC_UNROLL 3  // list entries a thread takes per trip of a round
// Owner word of (body, colour), colour-major: a round's bids go mostly to the lowest free colours,
// so the words in use (8 bytes per body for each colour bid) stay in L2, where a body-major
// table (256 bytes per body) spread every round's random atomics over the whole table in DRAM.
__device__ __forceinline__ size_t gc_owner_at(const DevState& d, uint32_t body, uint32_t col) {
  return size_t(col) * (size_t(d.body_capacity) + 1u) + body;
}
__global__ void __launch_bounds__(BB_GC_THREADS, 1) k_edge_color(const DevState d, Params p, int cur, uint32_t n) {
  DevCounters* c = d.ctr;
  const uint32_t M = c->manifold_count;
  const uint32_t epoch = c->gc_epoch;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  uint32_t* sync = &c->sync_count[0];
  uint32_t ep = 0;
  const int lane = threadIdx.x & 31;
  const uint32_t warp0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
  // Islands with an awake body get this launch's tag.  The rounds below are local to a
  // connected component of the conflict graph (manifolds sharing a dynamic body), and those
  // components are exactly the islands' manifold sets (k_components links every manifold).  So
  // leaving out the manifolds of islands with no awake body changes no other manifold's colour;
  // the solve skips those manifolds anyway (both bodies asleep or static), so they are marked
  // BB_RESTING and sorted behind the overflow bucket without being coloured.
  const uint32_t itag = epoch + 1u;  // never 0 (epochs step by 64), so zeroed tags never match
  // Colour reuse.  The colours of an island depend only on its set of manifolds (their bodies
  // and keys).  When every manifold of an island is one of last substep's (matched in the narrow
  // phase, gc_reuse) and none of last substep's manifolds on its bodies ended (gc_body_chg),
  // the set is last substep's and so are its colours: the island skips the rounds.  Islands
  // marked here (gc_island_chg) are coloured afresh.  Only right after a colouring.
  const uint32_t sub_tag = c->substeps;
  const bool reuse = c->gc_coloured + 1u == sub_tag;
  for (uint32_t i = tid; i < n; i += stride) {
    d.gc_mask[i] = 0;
    const uint32_t f = d.flags[i];
    const uint32_t isl = d.island[i];
    if ((f & BB_BODY_DYNAMIC) && !(f & BB_BODY_SLEEPING)) {
      if (isl != BB_NONE && d.gc_island_tag[isl] != itag) d.gc_island_tag[isl] = itag;
    }
    if (reuse && isl != BB_NONE && d.gc_body_chg[i] == sub_tag && d.gc_island_chg[isl] != itag)
      d.gc_island_chg[isl] = itag;
  }
  if (reuse) {  // manifolds that are not last substep's (or were not coloured then)
    for (uint32_t m = tid; m < M; m += stride) {
      const uint32_t slot = d.man_slot[cur][m];
      const uint32_t old = d.gc_reuse[slot];
      if (old != BB_NONE && old != BB_RESTING) continue;
      const uint2 b = d.m_bodies[cur][slot];
      const uint32_t isl = (d.flags[b.x] & BB_BODY_DYNAMIC) ? d.island[b.x] : d.island[b.y];
      if (isl != BB_NONE && d.gc_island_chg[isl] != itag) d.gc_island_chg[isl] = itag;
    }
  }
  if (tid == 0) {
    c->gc_colors = 0;
    c->gc_list_n[0] = 0;
    c->gc_list_n[1] = 0;
  }
  grid_sync(c, sync, ep);
  // round 1's list: the manifolds of islands with an awake body (a warp appends its lanes at once)
  uint32_t used0 = 0;  // colour + 1 of the reused colours
  for (uint32_t base = warp0; base < M; base += stride) {  // warp-uniform trips
    const uint32_t m = base + lane;
    bool colour = false;
    if (m < M) {
      const uint32_t slot = d.man_slot[cur][m];
      uint2 b = d.m_bodies[cur][slot];
      int key = d.m_keycc[cur][slot].x;
      const uint32_t fa = d.flags[b.x], fb = d.flags[b.y];
      const bool da = fa & BB_BODY_DYNAMIC, db = fb & BB_BODY_DYNAMIC;
      const uint32_t isl = da ? d.island[b.x] : db ? d.island[b.y] : BB_NONE;
      colour = isl != BB_NONE && d.gc_island_tag[isl] == itag;
      uint32_t kept = BB_NONE;  // a reused colour
      if (colour && reuse && d.gc_island_chg[isl] != itag) {
        kept = d.gc_reuse[slot];
        colour = false;
      }
      if (colour || kept != BB_NONE) {
        const uint32_t la = local_id(d, b.x), lb = local_id(d, b.y);
        uint32_t lo = min(la, lb), hi = max(la, lb);
        const uint32_t pid = gc_hash(lo * 0x9e3779b9u + hi * 0x85ebca6bu + uint32_t(key) * 0xc2b2ae35u);
        d.gc_pid[m] = pid;
        // bit 2: neither body awake (both asleep or static); the sweeps have nothing to do there
        const bool idle = !((fa & BB_BODY_DYNAMIC) && !(fa & BB_BODY_SLEEPING)) &&
                          !((fb & BB_BODY_DYNAMIC) && !(fb & BB_BODY_SLEEPING));
        d.gc_rec[m] = make_uint4(b.x, b.y, pid, (da ? 0u : 1u) | (db ? 0u : 2u) | (idle ? 4u : 0u));
      }
      d.gc_color[m] = kept != BB_NONE ? kept : colour ? BB_UNCOLORED : BB_RESTING;
      if (kept < BB_MAX_COLORS) used0 = max(used0, kept + 1u);
    }
    const unsigned mask = __ballot_sync(0xFFFFFFFFu, colour);
    if (mask) {
      uint32_t off = 0;
      if (lane == 0) off = atomicAdd(&c->gc_list_n[1], uint32_t(__popc(mask)));
      off = __shfl_sync(0xFFFFFFFFu, off, 0);
      if (colour) d.gc_list[1][off + __popc(mask & ((1u << lane) - 1u))] = m;
    }
  }
  used0 = __reduce_max_sync(0xFFFFFFFFu, used0);
  if (lane == 0 && used0) atomicMax(&c->gc_colors, used0);
  grid_sync(c, sync, ep);
  // Round r bids and commits over the manifolds still uncoloured when it starts: in round 1 all
  // manifolds of islands with an awake body (the identity list when that is all of them),
  // afterwards the list the previous round's commit left (in any order: a round's outcome
  // depends only on its set, since the highest priority wins every contested colour).
  const uint32_t n1 = *(volatile uint32_t*)&c->gc_list_n[1];
  // Once the uncoloured list fits in one block, block 0 runs the remaining rounds alone with
  // block barriers (the other blocks go straight to the final grid barrier): the same rounds
  // on the same sets, so the same colours, without two grid barriers per round.
  bool local = false;
  uint32_t ran = 0;
  for (uint32_t r = 1; r <= p.gc_rounds; ++r) {
    const uint32_t* L = r == 1 && n1 == M ? nullptr : d.gc_list[r & 1];
    const uint32_t nL = r == 1 ? n1 : *(volatile uint32_t*)&c->gc_list_n[r & 1];
    if (nL == 0) break;
    if (!local && nL <= blockDim.x) {
      local = true;
      if (blockIdx.x != 0) break;
    }
    ran = r;
    const uint32_t rtid = local ? threadIdx.x : tid, rstride = local ? blockDim.x : stride;
    if (rtid == 0) c->gc_list_n[(r + 1) & 1] = 0;  // the list this round fills (last read two rounds ago)
    const unsigned long long tag = (unsigned long long)(epoch + r) << 32;
    // A thread takes GC_UNROLL list entries per trip and issues each stage's loads (list entry,
    // record, body masks) for all of them before using any: the rounds are chains of dependent
    // loads, and this keeps several chains in flight per thread.  A round's outcome depends only
    // on its set of manifolds, not on the order in which they are taken.
    for (uint32_t i0 = rtid; i0 < nL; i0 += GC_UNROLL * rstride) {
      uint32_t m[GC_UNROLL];
      uint4 rec[GC_UNROLL];
      uint32_t ma[GC_UNROLL], mb[GC_UNROLL];
#pragma unroll
      for (int u = 0; u < GC_UNROLL; ++u) {
        const uint32_t i = i0 + uint32_t(u) * rstride;
        m[u] = i < nL ? (L ? L[i] : i) : BB_NONE;
      }
#pragma unroll
      for (int u = 0; u < GC_UNROLL; ++u) rec[u] = m[u] != BB_NONE ? d.gc_rec[m[u]] : make_uint4(0, 0, 0, 3u);
#pragma unroll
      for (int u = 0; u < GC_UNROLL; ++u) {
        ma[u] = (rec[u].w & 1u) ? 0u : d.gc_mask[rec[u].x];
        mb[u] = (rec[u].w & 2u) ? 0u : d.gc_mask[rec[u].y];
      }
#pragma unroll
      for (int u = 0; u < GC_UNROLL; ++u) {
        if (m[u] == BB_NONE) continue;
        const bool sa = rec[u].w & 1u, sb = rec[u].w & 2u;
        const uint32_t avail = ~(ma[u] | mb[u]);
        const uint32_t col = avail == 0u ? BB_MAX_COLORS : uint32_t(__ffs(avail) - 1);
        d.gc_choice[m[u]] = col;
        if (col >= BB_MAX_COLORS) continue;
        const unsigned long long v = tag | gc_priority(rec[u].z, r);
        if (!sa) atomicMax(&d.gc_owner[gc_owner_at(d, rec[u].x, col)], v);
        if (!sb) atomicMax(&d.gc_owner[gc_owner_at(d, rec[u].y, col)], v);
      }
    }
    if (local) __syncthreads();
    else grid_sync(c, sync, ep);
    uint32_t* next = d.gc_list[(r + 1) & 1];
    for (uint32_t base = local ? (threadIdx.x & ~31u) : warp0; base < nL; base += GC_UNROLL * rstride) {  // warp-uniform trips
      uint32_t m[GC_UNROLL], col[GC_UNROLL];
      uint4 rec[GC_UNROLL];
      unsigned long long oa[GC_UNROLL], ob[GC_UNROLL];
#pragma unroll
      for (int u = 0; u < GC_UNROLL; ++u) {
        const uint32_t i = base + uint32_t(u) * rstride + lane;
        m[u] = i < nL ? (L ? L[i] : i) : BB_NONE;
      }
#pragma unroll
      for (int u = 0; u < GC_UNROLL; ++u) {
        col[u] = m[u] != BB_NONE ? d.gc_choice[m[u]] : BB_MAX_COLORS;
        rec[u] = m[u] != BB_NONE ? d.gc_rec[m[u]] : make_uint4(0, 0, 0, 3u);
      }
#pragma unroll
      for (int u = 0; u < GC_UNROLL; ++u) {
        const bool live = col[u] < BB_MAX_COLORS;
        oa[u] = live && !(rec[u].w & 1u) ? d.gc_owner[gc_owner_at(d, rec[u].x, col[u])] : 0ull;
        ob[u] = live && !(rec[u].w & 2u) ? d.gc_owner[gc_owner_at(d, rec[u].y, col[u])] : 0ull;
      }
      uint32_t used = 0;  // colour + 1 of a committed manifold
#pragma unroll
      for (int u = 0; u < GC_UNROLL; ++u) {
        bool keep = m[u] != BB_NONE;
        if (keep && col[u] < BB_MAX_COLORS) {
          const bool sa = rec[u].w & 1u, sb = rec[u].w & 2u;
          const unsigned long long v = tag | gc_priority(rec[u].z, r);
          const bool wa = sa || oa[u] == v, wb = sb || ob[u] == v;
          if (wa && wb) {
            d.gc_color[m[u]] = col[u];
            if (!sa) atomicOr(&d.gc_mask[rec[u].x], 1u << col[u]);
            if (!sb) atomicOr(&d.gc_mask[rec[u].y], 1u << col[u]);
            used = max(used, col[u] + 1u);
            keep = false;
          }
        }
        const unsigned mask = __ballot_sync(0xFFFFFFFFu, keep);
        if (mask) {
          uint32_t off = 0;
          if (lane == 0) off = atomicAdd(&c->gc_list_n[(r + 1) & 1], uint32_t(__popc(mask)));
          off = __shfl_sync(0xFFFFFFFFu, off, 0);
          if (keep) next[off + __popc(mask & ((1u << lane) - 1u))] = m[u];
        }
      }
      used = __reduce_max_sync(0xFFFFFFFFu, used);  // one colour-count update per warp
      if (lane == 0 && used) atomicMax(&c->gc_colors, used);
    }
    if (local) __syncthreads();
    else grid_sync(c, sync, ep);
  }
  if (local) grid_sync(c, sync, ep);  // block 0's rounds are done before anyone reads the colours
  if (blockIdx.x == 0 && threadIdx.x == 0) c->gc_rounds_run = ran;
  // Keys: colour, 32 = overflow, 33 = not swept.  Under the colour-barrier schedule a coloured
  // manifold whose two bodies are both asleep or static is also keyed 33: its sweep items would
  // do nothing (both bodies are frozen this substep), and leaving them out of the colour lists
  // saves the sweeps from walking them.  Its colour (gc_color) is kept.  The dataflow schedule
  // ranks every manifold on a body's list, so there every coloured manifold stays in its colour.
  const bool drop_idle = p.schedule == BB_SCHEDULE_COLOUR_BARRIER;
  uint32_t over = 0;
  for (uint32_t m = tid; m < M; m += stride) {
    uint32_t col = d.gc_color[m];
    if (col == BB_UNCOLORED) ++over;
    uint32_t key = col == BB_UNCOLORED ? BB_MAX_COLORS : col == BB_RESTING ? BB_MAX_COLORS + 1 : col;
    if (drop_idle && key <= BB_MAX_COLORS && (reinterpret_cast<const uint32_t*>(d.gc_rec + m)[3] & 4u))
      key = BB_MAX_COLORS + 1;
    d.bucket_keys[0][m] = key;
    d.bucket_vals[0][m] = m;
    d.gc_slot_color[cur][d.man_slot[cur][m]] = col;  // for the next substep's colour reuse
  }
  if (over) atomicAdd(&c->gc_overflow, over);
  if (tid == 0) {
    c->gc_epoch = epoch + 64u;
    c->gc_coloured = sub_tag;
  }
}

// bucket_start[0..34]: start of colour c (32 = overflow, 33 = resting manifolds), [34] = M
__global__ void k_bucket_starts(const uint32_t* hist_scan, const uint32_t* n_ptr, uint32_t* starts, int nb) {
  int t = threadIdx.x;
  if (t < nb) starts[t] = hist_scan[t];
  if (t == nb) starts[t] = *n_ptr;
}

// Colour reuse: the bodies of last substep's manifolds that no manifold of this substep took
// over (their pair ended, or its key changed) mark their islands for a fresh colouring.
__global__ void k_gc_ended(const DevState d, int cur) {
  const int prv = cur ^ 1;
  const uint32_t tag = d.ctr->substeps;
  if (d.ctr->gc_coloured + 1u != tag) return;  // no reuse this substep
  const uint32_t Mp = min(d.ctr->prev_manifolds, d.pair_capacity);
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < Mp; m += gridDim.x * blockDim.x) {
    const uint32_t os = d.man_slot[prv][m];
    if (d.gc_survived[os] == tag) continue;
    const uint2 b = d.m_bodies[prv][os];
    if (b.x != BB_NONE) d.gc_body_chg[b.x] = tag;
    if (b.y != BB_NONE) d.gc_body_chg[b.y] = tag;
  }
}

int bb_edge_coloring_blocks(int sms) { return bb_coop_blocks((const void*)k_edge_color, BB_GC_THREADS, sms); }

void bb_edge_coloring(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, const StepScratch& sc,
                      int sms, int cur, int coop_blocks) {
  Params pp = p;
  int cc = cur;
  uint32_t nn = n;
  DevState dd = d;
  void* args[] = {&dd, &pp, &cc, &nn};
  k_gc_ended<<<sms * 8, BB_THREADS, 0, s>>>(d, cur);
  bb_launch_coop((const void*)k_edge_color, coop_blocks, BB_GC_THREADS, args, s);
  // stable bucket sort of manifold ids by colour (one 8-bit digit)
  uint32_t* keys[2] = {d.bucket_keys[0], d.bucket_keys[1]};
  uint32_t* vals[2] = {d.bucket_vals[0], d.bucket_vals[1]};
  // scratch: histogram region 1, status / tile-counter slot 6 (the front-end sort uses 0..5)
  uint32_t* hist = sc.sort_hist + 1 * BB_HIST_REGION;
  bb_launch_sort(s, keys, vals, &d.ctr->manifold_count, d.pair_capacity, 1, 0, hist,
                 sc.sort_status + 6 * size_t(sc.sort_tiles) * 256, sc.sort_tile_ctr + 6, d.ctr, sms);
  k_bucket_starts<<<1, 64, 0, s>>>(hist + 8 * 256, &d.ctr->manifold_count, d.bucket_start, BB_MAX_COLORS + 2);
}
