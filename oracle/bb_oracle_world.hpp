// bb_oracle_world.hpp -- TEST INFRASTRUCTURE ONLY: the oracle's world and step.
//
// The per-substep task order follows RigidBodyManager::create's task graph
// (src/rigid_body_manager.cpp:1284-1427).  One substep here = one reference simulate() at
// h = dt / substeps.
#pragma once
#include "bb_oracle.hpp"
#include "bb_oracle_voxel.hpp"

namespace bbo {

template <class R> class World {
 public:
  std::vector<Body<R>> bodies;
  bb_solver_params p;
  Pool pool;

  // persistent across substeps
  std::vector<uint32_t> order;  // body ids in the previous substep's sorted order
  std::vector<Manifold<R>> prev_manifolds;
  std::unordered_map<uint64_t, uint32_t> prev_pair_index;  // (min id, max id) -> prev manifold
  std::map<std::tuple<uint32_t, uint32_t, int>, uint32_t> prev_voxel_index;  // (a, b, key) -> prev manifold
  VoxelPool voxels;
  // frozen[i]: body i was asleep or static at the last narrow phase (its pose has not changed
  // since); carry_frozen: pairs of frozen, non-awake bodies carry their manifolds over
  std::vector<uint8_t> frozen;
  bool carry_frozen = true;
  bool skip_warm_once = false;
  // Test hook: the next narrow phase takes these manifolds' geometry (identity, key, normal,
  // contact points, depths, features) instead of computing it, so two implementations whose
  // near-degenerate contact decisions could differ solve the same contact set.  Warm-start
  // matching, anchors and tangent bases are still the oracle's own.
  std::vector<bb_manifold_info> inj_m;
  std::vector<bb_contact_info> inj_c;
  bool inj = false;

  // products of the last substep (debug readback)
  std::vector<uint32_t> morton;       // code of body order[i]
  std::vector<uint32_t> sorted_keys, sorted_ids, rank;
  std::vector<int32_t> child;         // 2(N-1)
  std::vector<Aabb> leaf, node;
  std::vector<uint32_t> pair_a, pair_b;
  std::vector<Manifold<R>> manifolds;
  std::vector<std::vector<uint32_t>> lists;  // per body id: manifold indices, ascending
  std::vector<uint32_t> island, body_color;
  std::vector<AvbdState<R>> avbd;
  bb_step_stats stats{};

  World(int threads) : pool(threads) { default_params(&p); }

  size_t n() const { return bodies.size(); }
  static bool is_dyn(const Body<R>& b) { return (b.flags & BB_BODY_DYNAMIC) != 0; }
  static bool awake(const Body<R>& b) { return is_dyn(b) && (b.flags & BB_BODY_SLEEPING) == 0; }

  // RigidBody::get_transformed_inertia (extensions.slang:184-188): M * D * M^T with
  // M = get_rotation_matrix() = to_matrix()^T  (i.e. R^T D R).  Physical: R D R^T.
  // A body with a non-zero off-diagonal (voxel bodies) uses its full symmetric matrix.
  Mat3<R> world_inv_inertia(const Body<R>& b) const {
    Mat3<R> Rm = to_matrix(b.rot);
    Mat3<R> D = diag(b.inv_inertia);
    const Vec3<R>& o = b.inv_inertia_off;
    if (o.x != R(0) || o.y != R(0) || o.z != R(0)) {
      D = Mat3<R>::rows(Vec3<R>(b.inv_inertia.x, o.x, o.y), Vec3<R>(o.x, b.inv_inertia.y, o.z),
                        Vec3<R>(o.y, o.z, b.inv_inertia.z));
    }
    if (p.quirks & BB_QUIRK_INERTIA_TRANSPOSE) return mul_mm(transpose(Rm), mul_mm(D, Rm));
    return mul_mm(Rm, mul_mm(D, transpose(Rm)));
  }

  // ------------------------------------------------------------------------------------
  // Front end: Morton -> sort -> LBVH -> pairs (RBM:1287-1304).
  void bounds(float wmin[3], float wext[3]) const {
    if (p.bounds_mode == BB_BOUNDS_AUTO && n() > 0) {
      float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      for (auto& b : bodies) {
        float pp[3] = {float(b.pos.x), float(b.pos.y), float(b.pos.z)};
        for (int k = 0; k < 3; ++k) {
          mn[k] = fminx(mn[k], pp[k]);
          mx[k] = fmaxx(mx[k], pp[k]);
        }
      }
      for (int k = 0; k < 3; ++k) {
        wmin[k] = mn[k];
        float e = mx[k] - mn[k];
        wext[k] = e > 0.0f ? e : 1.0f;
      }
      return;
    }
    for (int k = 0; k < 3; ++k) {
      wmin[k] = p.world_min[k];
      wext[k] = p.world_extent[k];
    }
  }

  void front_end() {
    const size_t N = n();
    if (order.size() != N) {
      order.resize(N);
      for (size_t i = 0; i < N; ++i) order[i] = uint32_t(i);
    }
    float wmin[3], wext[3];
    bounds(wmin, wext);
    morton.assign(N, 0);
    pool.parallel_for(N, [&](size_t i) {
      const Body<R>& b = bodies[order[i]];
      float pp[3] = {float(b.pos.x), float(b.pos.y), float(b.pos.z)};
      morton[i] = morton_of(pp, wmin, wext);
    }, 1024);
    // stable LSD radix sort == stable sort by key (LBVH.slang:34-152)
    std::vector<uint32_t> idx(N);
    for (size_t i = 0; i < N; ++i) idx[i] = uint32_t(i);
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) { return morton[x] < morton[y]; });
    sorted_keys.resize(N);
    sorted_ids.resize(N);
    rank.assign(N, 0);
    for (size_t i = 0; i < N; ++i) {
      sorted_keys[i] = morton[idx[i]];
      sorted_ids[i] = order[idx[i]];
      rank[sorted_ids[i]] = uint32_t(i);
    }
    // leaves (entry_generate_hierarchy_linear_bvh, RB_sim.slang:206-278)
    leaf.resize(N);
    pool.parallel_for(N, [&](size_t i) {
      const Body<R>& b = bodies[sorted_ids[i]];
      float pp[3] = {float(b.pos.x), float(b.pos.y), float(b.pos.z)};
      float qq[4] = {float(b.rot.v.x), float(b.rot.v.y), float(b.rot.v.z), float(b.rot.w)};
      leaf[i] = b.shape == BB_SHAPE_VOXEL ? leaf_aabb_box(b.lo, b.hi, pp, qq) : leaf_aabb(b.shape, b.half, pp, qq);
    }, 1024);
    const int n_ = int(N);
    child.assign(N > 1 ? 2 * (N - 1) : 0, 0);
    node.assign(N > 1 ? N - 1 : 0, Aabb());
    if (N > 1) {
      pool.parallel_for(N - 1, [&](size_t i) {
        int first, last;
        lbvh_range(sorted_keys, n_, int(i), first, last);
        int split = lbvh_split(sorted_keys, n_, first, last);
        int ca = (split == first) ? (n_ - 1 + split) : split;
        int cb = (split + 1 == last) ? (n_ - 1 + split + 1) : split + 1;
        child[2 * i] = ca;
        child[2 * i + 1] = cb;
      }, 1024);
      // refit (RB_sim.slang:282-349): union of descendant leaf AABBs; exact min/max
      std::vector<int> parent(2 * N - 1, -1);
      for (size_t i = 0; i + 1 < N; ++i) {
        parent[child[2 * i]] = int(i);
        parent[child[2 * i + 1]] = int(i);
      }
      std::vector<Aabb> all(2 * N - 1);
      std::vector<uint8_t> done(2 * N - 1, 0);
      for (size_t i = 0; i < N; ++i) all[N - 1 + i] = leaf[i];
      // post-order via explicit stack
      std::vector<std::pair<int, int>> st;
      st.push_back({0, 0});
      while (!st.empty()) {
        auto& top = st.back();
        int nd = top.first;
        if (nd >= n_ - 1) {
          st.pop_back();
          continue;
        }
        if (top.second == 0) {
          top.second = 1;
          st.push_back({child[2 * nd], 0});
        } else if (top.second == 1) {
          top.second = 2;
          st.push_back({child[2 * nd + 1], 0});
        } else {
          const Aabb& l = all[child[2 * nd]];
          const Aabb& r = all[child[2 * nd + 1]];
          Aabb u;
          for (int k = 0; k < 3; ++k) {
            u.mn[k] = fminx(l.mn[k], r.mn[k]);
            u.mx[k] = fmaxx(l.mx[k], r.mx[k]);
          }
          all[nd] = u;
          st.pop_back();
        }
      }
      for (size_t i = 0; i + 1 < N; ++i) node[i] = all[i];
    }
    // pairs: every (i, j), i < j, with overlapping leaf AABBs (LBVH.slang:223-286).  Found
    // by sweep-and-prune along the axis of largest spread, independent of the tree.
    int ax = 0;
    if (N > 0) {
      float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      for (size_t i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) {
          lo[k] = std::min(lo[k], leaf[i].mn[k]);
          hi[k] = std::max(hi[k], leaf[i].mn[k]);
        }
      for (int k = 1; k < 3; ++k)
        if (hi[k] - lo[k] > hi[ax] - lo[ax]) ax = k;
    }
    std::vector<uint32_t> byx(N);
    for (size_t i = 0; i < N; ++i) byx[i] = uint32_t(i);
    std::sort(byx.begin(), byx.end(), [&](uint32_t x, uint32_t y) {
      return leaf[x].mn[ax] < leaf[y].mn[ax] || (leaf[x].mn[ax] == leaf[y].mn[ax] && x < y);
    });
    std::vector<std::vector<uint32_t>> found(N);
    pool.parallel_for(N, [&](size_t s) {
      uint32_t i = byx[s];
      for (size_t t = s + 1; t < N; ++t) {
        uint32_t j = byx[t];
        if (leaf[j].mn[ax] > leaf[i].mx[ax]) break;
        if (overlap(leaf[i], leaf[j])) {
          uint32_t a = std::min(i, j), b = std::max(i, j);
          found[s].push_back((uint32_t(a)));
          found[s].push_back((uint32_t(b)));
        }
      }
    }, 256);
    std::vector<uint64_t> keys;
    for (auto& f : found)
      for (size_t k = 0; k < f.size(); k += 2) keys.push_back((uint64_t(f[k]) << 32) | f[k + 1]);
    std::sort(keys.begin(), keys.end());
    pair_a.resize(keys.size());
    pair_b.resize(keys.size());
    for (size_t k = 0; k < keys.size(); ++k) {
      pair_a[k] = uint32_t(keys[k] >> 32);
      pair_b[k] = uint32_t(keys[k] & 0xFFFFFFFFu);
    }
    stats.pair_count = uint32_t(keys.size());
  }

  // ------------------------------------------------------------------------------------
  // Carry-over of a frozen pair (neither body awake, both asleep or static at the last narrow
  // phase as well, so both poses are bit for bit those of the previous substep): instead of
  // recomputing its contacts and matching them against last substep's, the previous
  // manifold(s) of the pair in the same body order are kept as they were -- contacts, features,
  // impulses, penalties -- with warm-start counts + 1 and the extraction trend 0, as a
  // recomputation whose contacts all match by feature gives.  Returns false (recompute) when
  // the pair had no manifold last substep.
  bool carry_pair(size_t k, uint32_t ida, uint32_t idb, bool vox, std::array<Manifold<R>, 6>& out, uint8_t& have) {
    auto carry = [&](const Manifold<R>& old, Manifold<R>& m) {
      m = old;
      m.sa = pair_a[k];
      m.sb = pair_b[k];
      m.anchor_a = bodies[ida].pos;
      m.anchor_b = bodies[idb].pos;
      m.error = 0;
      m.color = MAX_U32;
      for (int c = 0; c < m.cc; ++c) {
        m.c[c].warm = std::min(255u, m.c[c].warm + 1u);
        if (m.c[c].stick == 0) {
          m.c[c].anchor_a = Vec3<R>();
          m.c[c].anchor_b = Vec3<R>();
        }
      }
    };
    if (vox) {
      bool any = false;
      for (uint32_t code = 0; code < 6; ++code) {
        auto it = prev_voxel_index.find(std::make_tuple(ida, idb, VOXEL_KEY0 + int(code)));
        if (it == prev_voxel_index.end()) continue;
        carry(prev_manifolds[it->second], out[code]);
        have |= uint8_t(1u << code);
        any = true;
      }
      return any;
    }
    auto it = prev_pair_index.find((uint64_t(std::min(ida, idb)) << 32) | std::max(ida, idb));
    if (it == prev_pair_index.end() || prev_manifolds[it->second].a != ida) return false;
    carry(prev_manifolds[it->second], out[0]);
    have = 1;
    return true;
  }

  // ------------------------------------------------------------------------------------
  // Narrow phase + warm start (collision_detection.slang:1514-1755).
  void narrow_from_injected() {
    const bool warm = (p.flags & BB_SIM_WARM_STARTING) && !skip_warm_once;
    manifolds.clear();
    for (size_t k = 0; k < inj_m.size(); ++k) {
      const bb_manifold_info& mi = inj_m[k];
      Manifold<R> m;
      m.a = mi.body_a;
      m.b = mi.body_b;
      m.sa = rank[m.a];
      m.sb = rank[m.b];
      m.key = mi.key;
      m.cc = mi.contact_count;
      m.normal = Vec3<R>(R(mi.normal[0]), R(mi.normal[1]), R(mi.normal[2]));
      for (int c = 0; c < m.cc; ++c) {
        const bb_contact_info& ci = inj_c[k * MAX_CONTACTS + c];
        Contact<R> ct;
        ct.pos = Vec3<R>(R(ci.position[0]), R(ci.position[1]), R(ci.position[2]));
        ct.pen = R(ci.penetration);
        ct.fp.in_ref = ci.feature & 0xFF;
        ct.fp.out_ref = (ci.feature >> 8) & 0xFF;
        ct.fp.in_inc = (ci.feature >> 16) & 0xFF;
        ct.fp.out_inc = ci.feature >> 24;
        m.c[c] = ct;
      }
      m.anchor_a = bodies[m.a].pos;
      m.anchor_b = bodies[m.b].pos;
      m.error = 0x7FFFFFFF;
      compute_basis(m);
      if (warm) {
        uint64_t key = (uint64_t(std::min(m.a, m.b)) << 32) | std::max(m.a, m.b);
        auto it = prev_pair_index.find(key);
        if (it != prev_pair_index.end()) {
          const Manifold<R>& old = prev_manifolds[it->second];
          update_from_old(m, old, old.a != m.a);
        }
      }
      manifolds.push_back(m);
    }
    inj = false;
  }

  void narrow_phase() {
    if (inj) narrow_from_injected();
    else narrow_manifolds();
    frozen.assign(n(), 0);
    for (size_t i = 0; i < n(); ++i) frozen[i] = awake(bodies[i]) ? 0 : 1;
    skip_warm_once = false;
    // per-body manifold lists in ascending manifold order (body_link_manifold :881-905)
    lists.assign(n(), {});
    uint32_t fresh = 0;
    float maxpen = 0;
    uint32_t contacts = 0;
    for (uint32_t m = 0; m < manifolds.size(); ++m) {
      lists[manifolds[m].a].push_back(m);
      lists[manifolds[m].b].push_back(m);
      for (int c = 0; c < manifolds[m].cc; ++c) {
        if (manifolds[m].c[c].warm == 0) ++fresh;
        maxpen = std::max(maxpen, float(-manifolds[m].c[c].pen));
        ++contacts;
      }
    }
    stats.manifold_count = uint32_t(manifolds.size());
    stats.contact_count = contacts;
    stats.fresh_contacts = fresh;
    stats.max_penetration = maxpen;
  }

  void narrow_manifolds() {
    const size_t P = pair_a.size();
    // up to six manifolds per pair (voxel pairs, one per face direction); one otherwise
    std::vector<std::array<Manifold<R>, 6>> per(P);
    std::vector<uint8_t> have(P, 0);
    bool warm = (p.flags & BB_SIM_WARM_STARTING) && !skip_warm_once;
    bool quirk = (p.quirks & BB_QUIRK_SAT_FRAME) != 0;
    pool.parallel_for(P, [&](size_t k) {
      uint32_t ida = sorted_ids[pair_a[k]], idb = sorted_ids[pair_b[k]];
      const Body<R>& A = bodies[ida];
      const Body<R>& B = bodies[idb];
      if (!is_dyn(A) && !is_dyn(B)) return;  // static-static skip (:1525)
      const bool vox = A.shape == BB_SHAPE_VOXEL || B.shape == BB_SHAPE_VOXEL;
      if (warm && carry_frozen && !awake(A) && !awake(B) && frozen.size() == n() && frozen[ida] && frozen[idb] &&
          carry_pair(k, ida, idb, vox, per[k], have[k]))
        return;
      for (uint32_t code = 0; code < (vox ? 6u : 1u); ++code) {
        SatResult<R> s;
        bool hit;
        if (vox) hit = voxel_collide(A, B, code, voxels, s);
        else if (A.shape == BB_SHAPE_BOX && B.shape == BB_SHAPE_BOX) hit = box_box(A, B, quirk, s);
        else if (A.shape == BB_SHAPE_SPHERE && B.shape == BB_SHAPE_SPHERE) hit = sphere_sphere(A, B, s);
        else hit = box_sphere(A, B, s);
        if (!hit) continue;
        Manifold<R>& m = per[k][code];
        m.a = ida;
        m.b = idb;
        m.sa = pair_a[k];
        m.sb = pair_b[k];
        m.key = s.key;
        m.cc = s.cc;
        m.normal = s.normal;
        for (int c = 0; c < s.cc; ++c) {
          Contact<R> ct;
          ct.pos = s.pos[c];
          // extraction cap of the SAT path (:1575-1578); the voxel path caps its own depths
          ct.pen = vox ? s.pen[c] : std::max(s.pen[c], R(p.penetration_cap));
          ct.fp = s.fp[c];
          m.c[c] = ct;
        }
        m.anchor_a = A.pos;
        m.anchor_b = B.pos;
        m.error = 0x7FFFFFFF;
        compute_basis(m);
        if (warm) {
          // find_old_collision (collision_detection.slang:914-963): voxel manifolds match their
          // own key in the same body order only; others any key, either order
          if (vox) {
            auto it = prev_voxel_index.find(std::make_tuple(ida, idb, m.key));
            if (it != prev_voxel_index.end()) update_from_old(m, prev_manifolds[it->second], false);
          } else {
            uint64_t key = (uint64_t(std::min(ida, idb)) << 32) | std::max(ida, idb);
            auto it = prev_pair_index.find(key);
            if (it != prev_pair_index.end()) {
              const Manifold<R>& old = prev_manifolds[it->second];
              update_from_old(m, old, old.a != ida);
            }
          }
        }
        have[k] |= uint8_t(1u << code);
      }
    }, 64);
    manifolds.clear();
    for (size_t k = 0; k < P; ++k)
      for (uint32_t code = 0; code < 6; ++code)
        if (have[k] & (1u << code)) manifolds.push_back(per[k][code]);
  }

  // ------------------------------------------------------------------------------------
  // Active list (entry_reset_body_links, RB_sim.slang:388-411) and islands
  // (islands.slang:153-302): union-find over dynamic bodies; island id = rank of the root
  // (lowest active index) among roots.
  void islands() {
    uint32_t na = 0;
    for (auto& b : bodies) b.active_index = is_dyn(b) ? na++ : MAX_U32;
    std::vector<uint32_t> parent(na);
    for (uint32_t i = 0; i < na; ++i) parent[i] = i;
    std::function<uint32_t(uint32_t)> find = [&](uint32_t x) {
      while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
      }
      return x;
    };
    for (auto& m : manifolds) {
      uint32_t x = bodies[m.a].active_index, y = bodies[m.b].active_index;
      if (x == MAX_U32 || y == MAX_U32) continue;
      uint32_t rx = find(x), ry = find(y);
      if (rx == ry) continue;
      if (rx < ry) parent[ry] = rx;
      else parent[rx] = ry;
    }
    std::vector<uint32_t> root_id(na, MAX_U32);
    uint32_t count = 0;
    for (uint32_t i = 0; i < na; ++i)
      if (find(i) == i) root_id[i] = count++;
    island.assign(n(), MAX_U32);
    for (auto& b : bodies)
      if (b.active_index != MAX_U32) island[b.id] = root_id[find(b.active_index)];
    stats.island_count = count;
    stats.active_body_count = na;
  }

  // ------------------------------------------------------------------------------------
  // Neighbourhood sleeping (RB_sim.slang:556-737).
  void sleep() {
    const uint32_t steps = p.sleep_steps;
    bool enabled = (p.flags & BB_SIM_SLEEPING_ENABLED) != 0;
    for (auto& r : bodies) {
      if (!is_dyn(r)) continue;
      if (!enabled) {
        r.sleep_timer = 0;
        r.flags &= ~BB_BODY_SLEEPING;
        continue;
      }
      if (lists[r.id].empty() && (r.flags & BB_BODY_SLEEPING)) {
        uint32_t t = r.sleep_timer & SLEEP_TIMER_MASK;
        r.sleep_timer = t >= 10u ? t - 10u : 0u;
        continue;
      }
      R lin2 = dot(r.vel, r.vel), ang2 = dot(r.omega, r.omega);
      uint32_t timer = r.sleep_timer & SLEEP_TIMER_MASK;
      bool calm = lin2 < R(p.sleep_lin_vel2) && ang2 < R(p.sleep_ang_vel2);
      r.sleep_timer = calm ? std::min(timer + 1u, steps) : (timer >= 4u ? timer - 4u : 0u);
    }
    if (!enabled) {
      stats.sleeping_count = 0;
      return;
    }
    for (auto& m : manifolds) {
      Body<R>& ra = bodies[m.a];
      Body<R>& rb = bodies[m.b];
      bool ad = is_dyn(ra), bd = is_dyn(rb);
      bool a_loud = ad && (ra.sleep_timer & SLEEP_TIMER_MASK) < steps;
      bool b_loud = bd && (rb.sleep_timer & SLEEP_TIMER_MASK) < steps;
      bool stalled = m.error != 0x7FFFFFFF && std::abs(m.error) < 10;
      bool deep = false;
      if (!stalled)
        for (int c = 0; c < m.cc; ++c)
          if (m.c[c].pen < R(-0.05)) { deep = true; break; }
      if ((a_loud || deep) && bd) rb.sleep_timer |= SLEEP_VETO_BIT;
      if ((b_loud || deep) && ad) ra.sleep_timer |= SLEEP_VETO_BIT;
    }
    uint32_t sleeping = 0;
    for (auto& r : bodies) {
      if (!is_dyn(r)) continue;
      bool vetoed = (r.sleep_timer & SLEEP_VETO_BIT) != 0;
      bool quiet = (r.sleep_timer & SLEEP_TIMER_MASK) >= steps;
      bool was = (r.flags & BB_BODY_SLEEPING) != 0;
      if (quiet && !vetoed) {
        if (!was) {
          r.vel = Vec3<R>();
          r.omega = Vec3<R>();
          r.flags |= BB_BODY_SLEEPING;
        }
        ++sleeping;
      } else if (was) {
        r.flags &= ~BB_BODY_SLEEPING;
      }
    }
    stats.sleeping_count = sleeping;
  }

  // ------------------------------------------------------------------------------------
  // Edge colouring (coloring.slang:45-292): rounds r = 1..gc_rounds of bid (InterlockedMax
  // of the priority on (body, lowest free colour)) and commit (won on both bodies).
  void edge_coloring() {
    const size_t M = manifolds.size();
    std::vector<uint32_t> mask(n(), 0);
    std::vector<uint32_t> pid(M);
    for (size_t m = 0; m < M; ++m) {
      manifolds[m].color = MAX_U32;
      pid[m] = gc_pair_id(manifolds[m].a, manifolds[m].b, manifolds[m].key);
    }
    std::unordered_map<uint64_t, uint32_t> owner;
    auto pick = [&](const Manifold<R>& mf, bool sa, bool sb) -> uint32_t {
      uint32_t ma = sa ? 0u : mask[mf.a], mb = sb ? 0u : mask[mf.b];
      uint32_t avail = ~(ma | mb);
      if (avail == 0) return MAX_COLORS;
      uint32_t c = uint32_t(__builtin_ctz(avail));
      return c < MAX_COLORS ? c : MAX_COLORS;
    };
    for (uint32_t r = 1; r <= p.gc_rounds; ++r) {
      owner.clear();
      bool any = false;
      std::vector<uint32_t> choice(M, MAX_COLORS);
      for (size_t m = 0; m < M; ++m) {
        Manifold<R>& mf = manifolds[m];
        if (mf.color != MAX_U32) continue;
        any = true;
        bool sa = !is_dyn(bodies[mf.a]), sb = !is_dyn(bodies[mf.b]);
        uint32_t c = pick(mf, sa, sb);
        choice[m] = c;
        if (c >= MAX_COLORS) continue;
        uint32_t pr = gc_priority(pid[m], r);
        if (!sa) {
          auto& o = owner[(uint64_t(mf.a) << 8) | c];
          o = std::max(o, pr);
        }
        if (!sb) {
          auto& o = owner[(uint64_t(mf.b) << 8) | c];
          o = std::max(o, pr);
        }
      }
      if (!any) break;
      std::vector<uint32_t> commit;
      for (size_t m = 0; m < M; ++m) {
        Manifold<R>& mf = manifolds[m];
        uint32_t c = choice[m];
        if (mf.color != MAX_U32 || c >= MAX_COLORS) continue;
        bool sa = !is_dyn(bodies[mf.a]), sb = !is_dyn(bodies[mf.b]);
        uint32_t pr = gc_priority(pid[m], r);
        bool wa = sa || owner[(uint64_t(mf.a) << 8) | c] == pr;
        bool wb = sb || owner[(uint64_t(mf.b) << 8) | c] == pr;
        if (wa && wb) commit.push_back(uint32_t(m));
      }
      for (uint32_t m : commit) {
        Manifold<R>& mf = manifolds[m];
        mf.color = choice[m];
        if (is_dyn(bodies[mf.a])) mask[mf.a] |= 1u << mf.color;
        if (is_dyn(bodies[mf.b])) mask[mf.b] |= 1u << mf.color;
      }
    }
    uint32_t used = 0, overflow = 0, viol = 0;
    std::unordered_map<uint64_t, uint32_t> seen;
    for (auto& mf : manifolds) {
      if (mf.color == MAX_U32) { ++overflow; continue; }
      used = std::max(used, mf.color + 1);
      if (is_dyn(bodies[mf.a]) && seen[(uint64_t(mf.a) << 8) | mf.color]++ > 0) ++viol;
      if (is_dyn(bodies[mf.b]) && seen[(uint64_t(mf.b) << 8) | mf.color]++ > 0) ++viol;
    }
    stats.graph_color_count = used;
    stats.graph_color_overflow = overflow;
    stats.graph_color_violations = viol;
  }

  // manifolds of each colour (ascending m) + the overflow list
  void color_buckets(std::vector<std::vector<uint32_t>>& buckets, std::vector<uint32_t>& overflow) const {
    buckets.assign(MAX_COLORS, {});
    overflow.clear();
    for (uint32_t m = 0; m < manifolds.size(); ++m) {
      uint32_t c = manifolds[m].color;
      if (c < MAX_COLORS) buckets[c].push_back(m);
      else overflow.push_back(m);
    }
  }

  // ------------------------------------------------------------------------------------
  // PGS_SOFT (solvers.slang:142-279) on graph colours (RB_sim.slang:1408-1578).
  void pgs_pre_step(Manifold<R>& m, R h, R hertz) {
    Body<R>& A = bodies[m.a];
    Body<R>& B = bodies[m.b];
    bool accum = (p.flags & BB_SIM_ACCUM_IMPULSE) != 0, fric = (p.flags & BB_SIM_FRICTION) != 0;
    Mat3<R> IA = world_inv_inertia(A), IB = world_inv_inertia(B);
    // velocities are staged locally and written back only to dynamic bodies: statics carry
    // zero inverse mass and inertia, so the reference's writes to them are no-ops
    Vec3<R> va = A.vel, wa = A.omega, vb = B.vel, wb = B.omega;
    for (int i = 0; i < m.cc; ++i) {
      Contact<R>& c = m.c[i];
      Vec3<R> r1 = c.pos - m.anchor_a, r2 = c.pos - m.anchor_b;
      Vec3<R> rn1 = cross(r1, m.normal), rn2 = cross(r2, m.normal);
      R kn = A.inv_mass + B.inv_mass + dot(rn1, mul_mv(IA, rn1)) + dot(rn2, mul_mv(IB, rn2));
      c.nmass = kn == 0 ? R(0) : R(1) / kn;
      for (int j = 0; j < 2; ++j) {
        Vec3<R> rt1 = cross(r1, m.t[j]), rt2 = cross(r2, m.t[j]);
        R kt = A.inv_mass + B.inv_mass + dot(rt1, mul_mv(IA, rt1)) + dot(rt2, mul_mv(IB, rt2));
        c.tmass[j] = kt == 0 ? R(0) : R(1) / kt;
      }
      R ch = (A.inv_mass == 0 || B.inv_mass == 0) ? R(2) * hertz : hertz;
      const R zeta = 10;
      const R omega = R(2) * R(PI_F) * ch;
      const R cc = h * omega * (R(2) * zeta + h * omega);
      c.bias = omega / (R(2) * zeta + h * omega);
      c.icoef = R(1) / (R(1) + cc);
      c.mcoef = cc * c.icoef;
      if (accum) {
        Vec3<R> P = m.normal * c.ni;
        if (fric)
          for (int j = 0; j < 2; ++j) P = P + m.t[j] * c.ti[j];
        va = va - P * A.inv_mass;
        wa = wa - mul_mv(IA, cross(r1, P));
        vb = vb + P * B.inv_mass;
        wb = wb + mul_mv(IB, cross(r2, P));
      }
    }
    if (is_dyn(A)) { A.vel = va; A.omega = wa; }
    if (is_dyn(B)) { B.vel = vb; B.omega = wb; }
  }
  void pgs_solve(Manifold<R>& m, bool use_bias, R inv_h) {
    Body<R>& A = bodies[m.a];
    Body<R>& B = bodies[m.b];
    bool accum = (p.flags & BB_SIM_ACCUM_IMPULSE) != 0, fric = (p.flags & BB_SIM_FRICTION) != 0;
    Mat3<R> IA = world_inv_inertia(A), IB = world_inv_inertia(B);
    R mu = std::sqrt(A.friction * B.friction);
    Vec3<R> va = A.vel, wa = A.omega, vb = B.vel, wb = B.omega;
    for (int i = 0; i < m.cc; ++i) {
      Contact<R>& c = m.c[i];
      Vec3<R> r1 = c.pos - m.anchor_a, r2 = c.pos - m.anchor_b;
      Vec3<R> rv = vb + cross(wb, r2) - va - cross(wa, r1);
      if (fric) {
        for (int j = 0; j < 2; ++j) {
          R tv = dot(rv, m.t[j]);
          R ti = c.tmass[j] * -tv;
          R maxf = mu * c.ni;
          if (accum) {
            R old = c.ti[j];
            c.ti[j] = std::min(std::max(old + ti, -maxf), maxf);
            ti = c.ti[j] - old;
          } else {
            ti = std::min(std::max(ti, -maxf), maxf);
          }
          Vec3<R> P = m.t[j] * ti;
          va = va - P * A.inv_mass;
          wa = wa - mul_mv(IA, cross(r1, P));
          vb = vb + P * B.inv_mass;
          wb = wb + mul_mv(IB, cross(r2, P));
        }
      }
      rv = vb + cross(wb, r2) - va - cross(wa, r1);
      R vn = dot(rv, m.normal);
      R bias = 0, ms = 1, is = 0;
      if (c.pen > 0) bias = c.pen * inv_h;
      else if (use_bias) {
        bias = std::max(c.bias * c.pen, R(-4));
        ms = c.mcoef;
        is = c.icoef;
      }
      R imp = -c.nmass * ms * (vn + bias) - is * c.ni;
      if (accum) {
        R old = c.ni;
        c.ni = std::max(old + imp, R(0));
        imp = c.ni - old;
      } else {
        imp = std::max(imp, R(0));
      }
      Vec3<R> P = m.normal * imp;
      va = va - P * A.inv_mass;
      wa = wa - mul_mv(IA, cross(r1, P));
      vb = vb + P * B.inv_mass;
      wb = wb + mul_mv(IB, cross(r2, P));
    }
    if (is_dyn(A)) { A.vel = va; A.omega = wa; }
    if (is_dyn(B)) { B.vel = vb; B.omega = wb; }
  }
  bool pair_active(const Manifold<R>& m) const { return awake(bodies[m.a]) || awake(bodies[m.b]); }

  // Quaternion integration (extensions.slang:148-166).
  static Quat<R> apply_angular_velocity(const Quat<R>& rot, Vec3<R> w, R dt) {
    R angle = length(w) * dt;
    if (angle > R(0.0001)) {
      Vec3<R> axis = normalize(w);
      R half = angle / R(2);
      Quat<R> q(axis * std::sin(half), std::cos(half));
      return (q * rot).normalize();
    }
    Vec3<R> dr = w * dt * R(0.5);
    Quat<R> q(dr, R(1));
    return (q * rot).normalize();
  }

  void solve_pgs_soft(R h) {
    std::vector<std::vector<uint32_t>> buckets;
    std::vector<uint32_t> overflow;
    color_buckets(buckets, overflow);
    R inv_h = h > 0 ? R(1) / h : R(0);
    R hertz = std::min(R(p.contact_hertz), inv_h * R(0.3333333333333333));
    auto sweep = [&](auto&& fn) {
      for (uint32_t c = 0; c < MAX_COLORS; ++c) {
        auto& bk = buckets[c];
        pool.parallel_for(bk.size(), [&](size_t k) {
          Manifold<R>& m = manifolds[bk[k]];
          if (pair_active(m)) fn(m);
        }, 32);
      }
      for (uint32_t mi : overflow)
        if (pair_active(manifolds[mi])) fn(manifolds[mi]);
    };
    sweep([&](Manifold<R>& m) { pgs_pre_step(m, h, hertz); });
    for (uint32_t it = 0; it < p.iterations; ++it) sweep([&](Manifold<R>& m) { pgs_solve(m, true, inv_h); });
    // entry_integrate_positions_rigid_bodies (RB_sim.slang:1287-1326)
    if (p.flags & BB_SIM_ADVECTION) {
      pool.parallel_for(n(), [&](size_t i) {
        Body<R>& r = bodies[i];
        if (!awake(r)) return;
        r.pos = r.pos + r.vel * h;
        r.rot = apply_angular_velocity(r.rot, r.omega, h);
      }, 1024);
    }
    for (uint32_t it = 0; it < p.relax_iterations; ++it) sweep([&](Manifold<R>& m) { pgs_solve(m, false, inv_h); });
  }

  // ---- per-island path (USE_GRAPH_COLORING off): RBM:1390-1399 ----------------------------
  // PGS::pre_step (solvers.slang:3-66): rows from the arms at pre-step time, Baumgarte bias
  // -BIAS_FACTOR / h * min(depth + PENETRATION_FACTOR, 0), warm start.
  void baum_pre_step(Manifold<R>& m, R inv_h) {
    Body<R>& A = bodies[m.a];
    Body<R>& B = bodies[m.b];
    bool accum = (p.flags & BB_SIM_ACCUM_IMPULSE) != 0, fric = (p.flags & BB_SIM_FRICTION) != 0;
    Mat3<R> IA = world_inv_inertia(A), IB = world_inv_inertia(B);
    Vec3<R> va = A.vel, wa = A.omega, vb = B.vel, wb = B.omega;
    for (int i = 0; i < m.cc; ++i) {
      Contact<R>& c = m.c[i];
      Vec3<R> r1 = c.pos - A.pos, r2 = c.pos - B.pos;
      Vec3<R> rn1 = cross(r1, m.normal), rn2 = cross(r2, m.normal);
      R kn = A.inv_mass + B.inv_mass + dot(rn1, mul_mv(IA, rn1)) + dot(rn2, mul_mv(IB, rn2));
      c.nmass = kn == 0 ? R(0) : R(1) / kn;
      for (int j = 0; j < 2; ++j) {
        Vec3<R> rt1 = cross(r1, m.t[j]), rt2 = cross(r2, m.t[j]);
        R kt = A.inv_mass + B.inv_mass + dot(rt1, mul_mv(IA, rt1)) + dot(rt2, mul_mv(IB, rt2));
        c.tmass[j] = kt == 0 ? R(0) : R(1) / kt;
      }
      c.bias = -R(0.2) * inv_h * std::min(c.pen + R(0.01), R(0));
      if (accum) {
        Vec3<R> P = m.normal * c.ni;
        if (fric)
          for (int j = 0; j < 2; ++j) P = P + m.t[j] * c.ti[j];
        va = va - P * A.inv_mass;
        wa = wa - mul_mv(IA, cross(r1, P));
        vb = vb + P * B.inv_mass;
        wb = wb + mul_mv(IB, cross(r2, P));
      }
    }
    if (is_dyn(A)) { A.vel = va; A.omega = wa; }
    if (is_dyn(B)) { B.vel = vb; B.omega = wb; }
  }
  // PGS::solve (solvers.slang:68-136): friction rows, then the normal row with the Baumgarte bias
  void baum_solve(Manifold<R>& m) {
    Body<R>& A = bodies[m.a];
    Body<R>& B = bodies[m.b];
    bool accum = (p.flags & BB_SIM_ACCUM_IMPULSE) != 0, fric = (p.flags & BB_SIM_FRICTION) != 0;
    Mat3<R> IA = world_inv_inertia(A), IB = world_inv_inertia(B);
    R mu = std::sqrt(A.friction * B.friction);
    Vec3<R> va = A.vel, wa = A.omega, vb = B.vel, wb = B.omega;
    for (int i = 0; i < m.cc; ++i) {
      Contact<R>& c = m.c[i];
      Vec3<R> r1 = c.pos - A.pos, r2 = c.pos - B.pos;
      Vec3<R> rv = vb + cross(wb, r2) - va - cross(wa, r1);
      if (fric) {
        for (int j = 0; j < 2; ++j) {
          R ti = c.tmass[j] * -dot(rv, m.t[j]);
          R maxf = mu * c.ni;
          if (accum) {
            R old = c.ti[j];
            c.ti[j] = std::min(std::max(old + ti, -maxf), maxf);
            ti = c.ti[j] - old;
          } else {
            ti = std::min(std::max(ti, -maxf), maxf);
          }
          Vec3<R> P = m.t[j] * ti;
          va = va - P * A.inv_mass;
          wa = wa - mul_mv(IA, cross(r1, P));
          vb = vb + P * B.inv_mass;
          wb = wb + mul_mv(IB, cross(r2, P));
        }
      }
      rv = vb + cross(wb, r2) - va - cross(wa, r1);
      R imp = c.nmass * (-dot(rv, m.normal) + c.bias);
      if (accum) {
        R old = c.ni;
        c.ni = std::max(old + imp, R(0));
        imp = c.ni - old;
      } else {
        imp = std::max(imp, R(0));
      }
      Vec3<R> P = m.normal * imp;
      va = va - P * A.inv_mass;
      wa = wa - mul_mv(IA, cross(r1, P));
      vb = vb + P * B.inv_mass;
      wb = wb + mul_mv(IB, cross(r2, P));
    }
    if (is_dyn(A)) { A.vel = va; A.omega = wa; }
    if (is_dyn(B)) { B.vel = vb; B.omega = wb; }
  }
  // entry_collision_pre_solver / solver / integrate / solver_relaxation (RB_sim.slang:1122-1406):
  // each contact island's manifolds serially, islands independent.  A manifold belongs to the
  // island of its dynamic body; within an island the manifolds run in manifold (pair) order.
  void solve_islands(R h) {
    const R inv_h = h > 0 ? R(1) / h : R(0);
    const R hertz = std::min(R(p.contact_hertz), inv_h * R(0.3333333333333333));
    const bool soft = p.solver == BB_SOLVER_PGS_SOFT;
    std::vector<std::vector<uint32_t>> lists(stats.island_count);
    for (uint32_t mi = 0; mi < manifolds.size(); ++mi) {
      const Manifold<R>& m = manifolds[mi];
      uint32_t isl = island[m.a] != MAX_U32 ? island[m.a] : island[m.b];
      if (isl != MAX_U32) lists[isl].push_back(mi);
    }
    auto per_island = [&](auto&& fn) {
      pool.parallel_for(lists.size(), [&](size_t k) {
        for (uint32_t mi : lists[k])
          if (pair_active(manifolds[mi])) fn(manifolds[mi]);
      }, 16);
    };
    per_island([&](Manifold<R>& m) {
      if (soft) pgs_pre_step(m, h, hertz);
      else baum_pre_step(m, inv_h);
    });
    for (uint32_t it = 0; it < p.iterations; ++it)
      per_island([&](Manifold<R>& m) {
        if (soft) pgs_solve(m, true, inv_h);
        else baum_solve(m);
      });
    if (p.flags & BB_SIM_ADVECTION) {
      pool.parallel_for(n(), [&](size_t i) {
        Body<R>& r = bodies[i];
        if (!awake(r)) return;
        r.pos = r.pos + r.vel * h;
        r.rot = apply_angular_velocity(r.rot, r.omega, h);
      }, 1024);
    }
    if (soft)
      for (uint32_t it = 0; it < p.relax_iterations; ++it) per_island([&](Manifold<R>& m) { pgs_solve(m, false, inv_h); });
  }

  // entry_rigid_body_sim / RigidBody::advect (RB_sim.slang:518-554, extensions.slang:127-139)
  void advect(R h) {
    if (p.solver == BB_SOLVER_AVBD || !(p.flags & BB_SIM_ADVECTION)) return;
    bool impulse = (p.quirks & BB_QUIRK_GRAVITY_IMPULSE) != 0;
    pool.parallel_for(n(), [&](size_t i) {
      Body<R>& r = bodies[i];
      if (!awake(r)) return;
      if (r.flags & BB_BODY_GRAVITY) {
        R dv = R(p.gravity) * h;
        if (impulse) dv = dv * r.inv_mass;
        r.vel.y = r.vel.y + dv;
      }
      r.vel = r.vel * R(std::exp(-h * R(p.linear_damping)));
      r.omega = r.omega * R(std::exp(-h * R(p.angular_damping)));
    }, 1024);
  }

  // ------------------------------------------------------------------------------------
  // AVBD (avbd.slang).
  static Vec3<R> small_angle_delta(const Quat<R>& now, const Quat<R>& start) {
    Quat<R> dq = now * start.conjugate();
    R sg = dq.w < 0 ? R(-1) : R(1);
    return dq.v * (R(2) * sg);
  }
  static Vec3<R> q_rotate(const Quat<R>& q, Vec3<R> u) { return u + R(2) * cross(q.v, cross(q.v, u) + q.w * u); }

  void avbd_coloring() {
    const uint32_t N = uint32_t(n());
    body_color.assign(N, MAX_U32);
    for (uint32_t rd = 0; rd < p.avbd_color_rounds; ++rd) {
      std::vector<uint32_t> next = body_color;
      pool.parallel_for(N, [&](size_t i) {
        const Body<R>& r = bodies[i];
        if (body_color[i] != MAX_U32 || !is_dyn(r)) return;
        uint32_t mine = avbd_priority(r.id, rd);
        uint32_t used = 0;
        for (uint32_t mi : lists[i]) {
          const Manifold<R>& m = manifolds[mi];
          uint32_t pp = m.a == i ? m.b : m.a;
          if (pp == i || !is_dyn(bodies[pp])) continue;
          uint32_t pc = body_color[pp];
          if (pc == MAX_U32) {
            if (avbd_priority(bodies[pp].id, rd) > mine) return;
          } else if (pc < MAX_COLORS) {
            used |= 1u << pc;
          }
        }
        uint32_t avail = ~used;
        if (avail == 0) return;
        uint32_t c = uint32_t(__builtin_ctz(avail));
        if (c >= MAX_COLORS) return;
        next[i] = c;
      }, 256);
      body_color.swap(next);
    }
    uint32_t used = 0, viol = 0;
    for (uint32_t i = 0; i < N; ++i) {
      if (!is_dyn(bodies[i])) continue;
      bool has = false;
      for (uint32_t mi : lists[i]) {
        const Manifold<R>& m = manifolds[mi];
        uint32_t pp = m.a == i ? m.b : m.a;
        if (pp == i || !is_dyn(bodies[pp])) continue;
        has = true;
        if (body_color[i] != MAX_U32 && body_color[pp] == body_color[i] && pp > i) ++viol;
      }
      if (body_color[i] == MAX_U32) {
        if (has) ++viol;
        continue;
      }
      used = std::max(used, body_color[i] + 1);
    }
    stats.avbd_color_count = used;
    stats.avbd_violations = viol;
  }

  void avbd_prepare(R dt) {
    avbd.resize(n());
    pool.parallel_for(n(), [&](size_t i) {
      Body<R>& r = bodies[i];
      if (!awake(r)) return;
      AvbdState<R>& s = avbd[i];
      R om = length(r.omega);
      if (om > R(50)) r.omega = r.omega * (R(50) / om);
      R grav = (r.flags & BB_BODY_GRAVITY) ? R(p.gravity) : R(0);
      s.pos_start = r.pos;
      s.rot_start = r.rot;
      s.pos_tilde = r.pos + r.vel * dt + Vec3<R>(0, grav, 0) * (dt * dt);
      Quat<R> qt = apply_angular_velocity(r.rot, r.omega, dt);
      s.rot_tilde = qt;
      R aw = 0;
      if (std::fabs(grav) > R(1e-6)) {
        R ay = (r.vel.y - r.prev_vel.y) / dt;
        R sg = grav > 0 ? R(1) : (grav < 0 ? R(-1) : R(0));
        aw = std::min(std::max(ay * sg / std::fabs(grav), R(0)), R(1));
      }
      r.pos = r.pos + r.vel * dt + Vec3<R>(0, grav, 0) * (aw * dt * dt);
      r.rot = qt;
    }, 1024);
  }

  void avbd_warmstart() {
    bool warm = (p.flags & BB_SIM_WARM_STARTING) != 0;
    std::atomic<uint32_t> sticks{0};
    pool.parallel_for(manifolds.size(), [&](size_t mi) {
      Manifold<R>& m = manifolds[mi];
      const Body<R>& r1 = bodies[m.a];
      const Body<R>& r2 = bodies[m.b];
      bool d1 = awake(r1), d2 = awake(r2);
      Vec3<R> c1 = d1 ? avbd[m.a].pos_start : r1.pos;
      Vec3<R> c2 = d2 ? avbd[m.b].pos_start : r2.pos;
      Quat<R> q1c = (d1 ? avbd[m.a].rot_start : r1.rot).conjugate();
      Quat<R> q2c = (d2 ? avbd[m.b].rot_start : r2.rot).conjugate();
      for (int j = 0; j < m.cc; ++j) {
        Contact<R>& c = m.c[j];
        bool matched = c.warm != 0 && warm;
        if (!matched) {
          c.ni = 0;
          c.mcoef = R(p.avbd_k_min);
          c.ti[0] = c.ti[1] = 0;
          c.tmass[0] = c.tmass[1] = R(p.avbd_k_min);
          c.stick = 0;
        } else {
          c.mcoef = std::min(std::max(c.mcoef * R(p.avbd_gamma), R(p.avbd_k_min)), R(p.avbd_k_max));
          c.ni = std::min(c.ni, R(0));
          for (int t = 0; t < 2; ++t)
            c.tmass[t] = std::min(std::max(c.tmass[t] * R(p.avbd_gamma), R(p.avbd_k_min)), R(p.avbd_k_max));
        }
        bool sticking = matched && c.stick != 0;
        if (!sticking) {
          c.anchor_a = q_rotate(q1c, c.pos - c1);
          c.anchor_b = q_rotate(q2c, c.pos - c2);
        } else {
          sticks.fetch_add(1);
        }
      }
    }, 64);
    stats.stick_count = sticks.load();
  }

  void avbd_depth() {
    const uint32_t N = uint32_t(n());
    for (uint32_t i = 0; i < N; ++i) avbd[i].depth = awake(bodies[i]) ? MAX_U32 : 0u;
    for (uint32_t pass = 0; pass < p.avbd_shock_layers; ++pass) {
      std::vector<uint32_t> d(N);
      for (uint32_t i = 0; i < N; ++i) d[i] = avbd[i].depth;
      for (auto& m : manifolds) {
        if (m.cc <= 0) continue;
        uint32_t d1 = d[m.a], d2 = d[m.b];
        if (d2 != MAX_U32 && d2 + 1 < d1) avbd[m.a].depth = std::min(avbd[m.a].depth, d2 + 1);
        if (d1 != MAX_U32 && d1 + 1 < d2) avbd[m.b].depth = std::min(avbd[m.b].depth, d1 + 1);
      }
    }
  }

  R contact_C(const Manifold<R>& m, int j, bool d1, bool d2, R alpha, Vec3<R>& rr1, Vec3<R>& rr2) const {
    const Body<R>& r1 = bodies[m.a];
    const Body<R>& r2 = bodies[m.b];
    Vec3<R> n = m.normal, pp = m.c[j].pos;
    Vec3<R> c1 = d1 ? avbd[m.a].pos_start : r1.pos;
    Vec3<R> c2 = d2 ? avbd[m.b].pos_start : r2.pos;
    rr1 = pp - c1;
    rr2 = pp - c2;
    R C0 = m.c[j].pen + R(p.avbd_margin);
    R C = C0 * (R(1) - alpha);
    if (d1) {
      Vec3<R> dp = r1.pos - avbd[m.a].pos_start;
      Vec3<R> dth = small_angle_delta(r1.rot, avbd[m.a].rot_start);
      C = C - dot(n, dp + cross(dth, rr1));
    }
    if (d2) {
      Vec3<R> dp = r2.pos - avbd[m.b].pos_start;
      Vec3<R> dth = small_angle_delta(r2.rot, avbd[m.b].rot_start);
      C = C + dot(n, dp + cross(dth, rr2));
    }
    return C;
  }
  R dir_C(Vec3<R> d, const Manifold<R>& m, int j, bool d1, bool d2, R alpha, Vec3<R>& ar1, Vec3<R>& ar2,
          R& C0t) const {
    const Body<R>& r1 = bodies[m.a];
    const Body<R>& r2 = bodies[m.b];
    Vec3<R> c1 = d1 ? avbd[m.a].pos_start : r1.pos;
    Vec3<R> c2 = d2 ? avbd[m.b].pos_start : r2.pos;
    Quat<R> q1 = d1 ? avbd[m.a].rot_start : r1.rot;
    Quat<R> q2 = d2 ? avbd[m.b].rot_start : r2.rot;
    ar1 = q_rotate(q1, m.c[j].anchor_a);
    ar2 = q_rotate(q2, m.c[j].anchor_b);
    C0t = dot(d, (c2 + ar2) - (c1 + ar1));
    R sg = C0t > 0 ? R(1) : (C0t < 0 ? R(-1) : R(0));
    R c0e = sg * std::max(R(0), std::fabs(C0t) - R(p.avbd_stick_slop));
    R C = c0e * (R(1) - alpha);
    if (d1) {
      Vec3<R> dp = r1.pos - avbd[m.a].pos_start;
      Vec3<R> dth = small_angle_delta(r1.rot, avbd[m.a].rot_start);
      C = C - dot(d, dp + cross(dth, ar1));
    }
    if (d2) {
      Vec3<R> dp = r2.pos - avbd[m.b].pos_start;
      Vec3<R> dth = small_angle_delta(r2.rot, avbd[m.b].rot_start);
      C = C + dot(d, dp + cross(dth, ar2));
    }
    return C;
  }

  // avbd_inverse3 (avbd.slang:309-326)
  static Mat3<R> inverse3(const Mat3<R>& a) {
    Vec3<R> c0 = a.col(0), c1 = a.col(1), c2 = a.col(2);
    Vec3<R> r0 = cross(c1, c2), r1 = cross(c2, c0), r2 = cross(c0, c1);
    R det = dot(c0, r0);
    R inv = std::fabs(det) > R(1e-12) ? R(1) / det : R(0);
    return Mat3<R>::rows(r0 * inv, r1 * inv, r2 * inv);
  }
  // avbd_solve6 (avbd.slang:329-387): in-place LDL^T with diagonal floor 1e-8.
  static void solve6(R H[6][6], R b[6], R x[6]) {
    for (int jj = 0; jj < 6; ++jj) {
      R d = H[jj][jj];
      for (int kk = 0; kk < jj; ++kk) d -= H[jj][kk] * H[jj][kk] * H[kk][kk];
      d = std::max(d, R(1e-8));
      H[jj][jj] = d;
      for (int ii = jj + 1; ii < 6; ++ii) {
        R s = H[ii][jj];
        for (int kk = 0; kk < jj; ++kk) s -= H[ii][kk] * H[jj][kk] * H[kk][kk];
        H[ii][jj] = s / d;
      }
    }
    for (int ii = 0; ii < 6; ++ii) {
      R s = b[ii];
      for (int kk = 0; kk < ii; ++kk) s -= H[ii][kk] * b[kk];
      b[ii] = s;
    }
    for (int ii = 0; ii < 6; ++ii) b[ii] /= H[ii][ii];
    for (int ii = 5; ii >= 0; --ii) {
      R s = b[ii];
      for (int kk = ii + 1; kk < 6; ++kk) s -= H[kk][ii] * x[kk];
      x[ii] = s;
    }
  }

  // entry_avbd_primal (avbd.slang:478-658)
  void avbd_primal(uint32_t i, R dt, R alpha) {
    Body<R>& r = bodies[i];
    AvbdState<R>& s = avbd[i];
    R inv_dt2 = dt > 0 ? R(1) / (dt * dt) : R(0);
    R m_lin = r.mass * inv_dt2;
    Mat3<R> Iw = inverse3(world_inv_inertia(r));
    R H[6][6] = {};
    R g[6] = {};
    H[0][0] = H[1][1] = H[2][2] = m_lin;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) H[3 + a][3 + b] = Iw.m[a][b] * inv_dt2;
    Vec3<R> dpos = r.pos - s.pos_tilde;
    Vec3<R> dth = small_angle_delta(r.rot, s.rot_tilde);
    g[0] = m_lin * dpos.x;
    g[1] = m_lin * dpos.y;
    g[2] = m_lin * dpos.z;
    Vec3<R> ga = mul_mv(Iw, dth) * inv_dt2;
    g[3] = ga.x;
    g[4] = ga.y;
    g[5] = ga.z;
    for (uint32_t mi : lists[i]) {
      const Manifold<R>& m = manifolds[mi];
      bool i1 = m.a == i;
      bool d1 = awake(bodies[m.a]), d2 = awake(bodies[m.b]);
      R mu = std::sqrt(std::max(bodies[m.a].friction, R(0)) * std::max(bodies[m.b].friction, R(0)));
      for (int j = 0; j < m.cc; ++j) {
        Vec3<R> rr1, rr2;
        R C = contact_C(m, j, d1, d2, alpha, rr1, rr2);
        R lam = m.c[j].ni, k = m.c[j].mcoef;
        R f = std::min(k * C + lam, R(0));
        Vec3<R> n = m.normal;
        Vec3<R> Jl = i1 ? -n : n;
        Vec3<R> Ja = i1 ? -cross(rr1, n) : cross(rr2, n);
        R J[6] = {Jl.x, Jl.y, Jl.z, Ja.x, Ja.y, Ja.z};
        for (int a = 0; a < 6; ++a) g[a] += f * J[a];
        for (int a = 0; a < 6; ++a)
          for (int b = 0; b < 6; ++b) H[a][b] += k * J[a] * J[b];
        R bound = mu * std::fabs(lam);
        for (int t = 0; t < 2; ++t) {
          Vec3<R> td = m.t[t], ar1, ar2;
          R C0t;
          R Ct = dir_C(td, m, j, d1, d2, alpha, ar1, ar2, C0t);
          R kt = m.c[j].tmass[t];
          R ft = std::min(std::max(kt * Ct + m.c[j].ti[t], -bound), bound);
          Vec3<R> Jlt = i1 ? -td : td;
          Vec3<R> Jat = i1 ? -cross(ar1, td) : cross(ar2, td);
          R Jt[6] = {Jlt.x, Jlt.y, Jlt.z, Jat.x, Jat.y, Jat.z};
          for (int a = 0; a < 6; ++a) g[a] += ft * Jt[a];
          for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b) H[a][b] += kt * Jt[a] * Jt[b];
        }
      }
    }
    R rhs[6], dx[6] = {};
    for (int a = 0; a < 6; ++a) rhs[a] = -g[a];
    solve6(H, rhs, dx);
    r.pos = r.pos + Vec3<R>(dx[0], dx[1], dx[2]);
    Vec3<R> half = Vec3<R>(dx[3], dx[4], dx[5]) * R(0.5);
    r.rot = (Quat<R>(half, R(1)) * r.rot).normalize();
  }

  // entry_avbd_dual (avbd.slang:728-808)
  void avbd_dual(Manifold<R>& m) {
    bool d1 = awake(bodies[m.a]), d2 = awake(bodies[m.b]);
    if (!d1 && !d2) return;
    R mu = std::sqrt(std::max(bodies[m.a].friction, R(0)) * std::max(bodies[m.b].friction, R(0)));
    for (int j = 0; j < m.cc; ++j) {
      Contact<R>& c = m.c[j];
      Vec3<R> rr1, rr2;
      R C = contact_C(m, j, d1, d2, R(1), rr1, rr2);
      R lam = c.ni, k = c.mcoef;
      R nl = std::min(k * C + lam, R(0));
      c.ni = nl;
      if (nl < 0) c.mcoef = std::min(k + R(p.avbd_beta) * std::fabs(C), R(p.avbd_k_max));
      R bound = mu * std::fabs(lam);
      bool stick_ok = true;
      R drift2 = 0;
      for (int t = 0; t < 2; ++t) {
        Vec3<R> ar1, ar2;
        R C0t;
        R Ct = dir_C(m.t[t], m, j, d1, d2, R(1), ar1, ar2, C0t);
        R lt = c.ti[t], kt = c.tmass[t];
        R nlt = std::min(std::max(kt * Ct + lt, -bound), bound);
        c.ti[t] = nlt;
        if (nlt > -bound && nlt < bound) c.tmass[t] = std::min(kt + R(p.avbd_beta) * std::fabs(Ct), R(p.avbd_k_max));
        else stick_ok = false;
        drift2 += C0t * C0t;
      }
      R th = R(p.avbd_stick_thresh);
      c.stick = (stick_ok && drift2 < th * th) ? 1u : 0u;
    }
  }

  void avbd_finalize(R dt) {
    R inv_dt = dt > 0 ? R(1) / dt : R(0);
    pool.parallel_for(n(), [&](size_t i) {
      Body<R>& r = bodies[i];
      if (!awake(r)) return;
      AvbdState<R>& s = avbd[i];
      r.prev_vel = r.vel;
      r.vel = (r.pos - s.pos_start) * inv_dt;
      Quat<R> dq = r.rot * s.rot_start.conjugate();
      R sg = dq.w < 0 ? R(-1) : R(1);
      r.omega = dq.v * (R(2) * sg * inv_dt);
      R v2 = dot(r.vel, r.vel), w2 = dot(r.omega, r.omega);
      if (v2 < R(0.09) && w2 < R(0.16) && lists[i].size() >= 3) {
        r.vel = r.vel * R(0.9);
        r.omega = r.omega * R(0.9);
      }
    }, 1024);
  }

  void solve_avbd(R h) {
    avbd_coloring();
    avbd_prepare(h);
    avbd_warmstart();
    avbd_depth();
    std::vector<std::vector<uint32_t>> by_color(MAX_COLORS);
    for (uint32_t i = 0; i < n(); ++i)
      if (body_color[i] < MAX_COLORS && awake(bodies[i])) by_color[body_color[i]].push_back(i);
    auto primal_sweep = [&](R alpha, uint32_t layer) {
      for (uint32_t c = 0; c < MAX_COLORS; ++c) {
        auto& bk = by_color[c];
        pool.parallel_for(bk.size(), [&](size_t k) {
          uint32_t i = bk[k];
          if (layer != MAX_U32) {
            uint32_t my = std::min(avbd[i].depth, p.avbd_shock_layers - 1);
            if (my != layer) return;
          }
          avbd_primal(i, h, alpha);
        }, 16);
      }
    };
    for (uint32_t it = 0; it < p.avbd_iterations; ++it) {
      primal_sweep(R(1), MAX_U32);
      pool.parallel_for(manifolds.size(), [&](size_t mi) { avbd_dual(manifolds[mi]); }, 64);
    }
    avbd_finalize(h);
    for (uint32_t d = 0; d < p.avbd_shock_layers; ++d) primal_sweep(R(0), d);
    for (uint32_t ps = 1; ps < p.avbd_post_stab_sweeps; ++ps) primal_sweep(R(0), MAX_U32);
  }

  // ------------------------------------------------------------------------------------
  // Collision front end only (stage 1: broad phase, 2: + narrow phase).
  void collide(uint32_t stage) {
    front_end();
    if (stage >= 2) narrow_phase();
    order = sorted_ids;  // the sorted order seeds the next sort's tie order, as in a substep
  }

  void publish() {
    order = sorted_ids;
    prev_manifolds = manifolds;
    prev_pair_index.clear();
    prev_voxel_index.clear();
    for (uint32_t m = 0; m < prev_manifolds.size(); ++m) {
      const auto& mf = prev_manifolds[m];
      if (mf.key >= VOXEL_KEY0 && mf.key < VOXEL_KEY0 + 6) prev_voxel_index[std::make_tuple(mf.a, mf.b, mf.key)] = m;
      else prev_pair_index[(uint64_t(std::min(mf.a, mf.b)) << 32) | std::max(mf.a, mf.b)] = m;
    }
  }

  void substep(R h) {
    stats = bb_step_stats{};
    stats.body_count = uint32_t(n());
    front_end();
    narrow_phase();
    advect(h);
    islands();
    sleep();
    const bool coloured = (p.flags & BB_SIM_USE_GRAPH_COLORING) != 0;
    if (coloured || p.solver == BB_SOLVER_AVBD) edge_coloring();
    if (p.solver == BB_SOLVER_AVBD) solve_avbd(h);
    else if (!coloured) solve_islands(h);
    else if (p.solver == BB_SOLVER_PGS_SOFT) solve_pgs_soft(h);
    publish();
  }

  void step(R dt, uint32_t substeps) {
    if (substeps == 0) substeps = 1;
    R h = dt / R(substeps);
    for (uint32_t s = 0; s < substeps; ++s) substep(h);
    stats.substeps_run = substeps;
  }
};

}  // namespace bbo
