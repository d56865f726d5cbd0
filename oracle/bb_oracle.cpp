// bb_oracle.cpp -- TEST INFRASTRUCTURE ONLY: extern "C" surface of the oracle for ctypes.
// Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg; never by the
// product library.  The debug-read layouts are the product's BB_DBG_* layouts
// (include/beatbox.h) so tests can compare buffers directly.
#include <cstring>
#include <memory>

#include "bb_oracle_world.hpp"

using namespace bbo;

namespace {
struct Handle {
  bool dbl;
  std::unique_ptr<World<double>> d;
  std::unique_ptr<World<float>> f;
};

template <class R>
void load(World<R>& w, uint32_t n, const float* pos, const float* quat, const float* vel, const float* omega,
          const uint32_t* shape, const float* half, const uint32_t* flags, const float* mass, const float* inv_mass,
          const float* inv_inertia, const float* friction, const float* restitution) {
  w.bodies.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    Body<R>& b = w.bodies[i];
    b.id = i;
    b.flags = flags[i];
    b.shape = shape[i];
    for (int k = 0; k < 3; ++k) b.half[k] = half[3 * i + k];
    b.pos = Vec3<R>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    b.rot = Quat<R>(Vec3<R>(quat[4 * i], quat[4 * i + 1], quat[4 * i + 2]), quat[4 * i + 3]);
    b.vel = vel ? Vec3<R>(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]) : Vec3<R>();
    b.omega = omega ? Vec3<R>(omega[3 * i], omega[3 * i + 1], omega[3 * i + 2]) : Vec3<R>();
    b.prev_vel = b.vel;
    bool dyn = (b.flags & BB_BODY_DYNAMIC) != 0;
    b.mass = dyn ? R(mass[i]) : R(0);
    b.inv_mass = dyn ? R(inv_mass[i]) : R(0);
    b.inv_inertia = dyn ? Vec3<R>(inv_inertia[3 * i], inv_inertia[3 * i + 1], inv_inertia[3 * i + 2]) : Vec3<R>();
    b.friction = friction[i];
    b.restitution = restitution[i];
  }
  w.order.clear();
  w.frozen.clear();
  w.prev_manifolds.clear();
  w.prev_pair_index.clear();
}

template <class R> uint64_t debug_read(World<R>& w, uint32_t which, void* dst, uint64_t max_bytes) {
  auto put = [&](const void* src, uint64_t bytes) { std::memcpy(dst, src, std::min(bytes, max_bytes)); };
  const uint64_t N = w.n();
  switch (which) {
    case BB_DBG_MORTON: {
      std::vector<uint32_t> by_id(w.sorted_keys.size());
      for (size_t i = 0; i < w.sorted_keys.size(); ++i) by_id[w.sorted_ids[i]] = w.sorted_keys[i];
      put(by_id.data(), 4 * by_id.size());
      return by_id.size();
    }
    case BB_DBG_SORTED_KEYS: put(w.sorted_keys.data(), 4 * w.sorted_keys.size()); return w.sorted_keys.size();
    case BB_DBG_SORTED_IDS: put(w.sorted_ids.data(), 4 * w.sorted_ids.size()); return w.sorted_ids.size();
    case BB_DBG_LBVH_CHILD: put(w.child.data(), 4 * w.child.size()); return w.child.size();
    case BB_DBG_LEAF_AABB: put(w.leaf.data(), 24 * w.leaf.size()); return w.leaf.size() * 6;
    case BB_DBG_NODE_AABB: put(w.node.data(), 24 * w.node.size()); return w.node.size() * 6;
    case BB_DBG_PAIRS: {
      std::vector<uint32_t> pr(2 * w.pair_a.size());
      for (size_t k = 0; k < w.pair_a.size(); ++k) {
        pr[2 * k] = w.pair_a[k];
        pr[2 * k + 1] = w.pair_b[k];
      }
      put(pr.data(), 4 * pr.size());
      return pr.size();
    }
    case BB_DBG_MANIFOLDS: {
      std::vector<bb_manifold_info> mi(w.manifolds.size());
      for (size_t m = 0; m < mi.size(); ++m) {
        const auto& mf = w.manifolds[m];
        mi[m].body_a = mf.a;
        mi[m].body_b = mf.b;
        mi[m].key = mf.key;
        mi[m].contact_count = mf.cc;
        mi[m].normal[0] = float(mf.normal.x);
        mi[m].normal[1] = float(mf.normal.y);
        mi[m].normal[2] = float(mf.normal.z);
        mi[m].color = mf.color;
        for (int t = 0; t < 2; ++t) {
          mi[m].tangent[t][0] = float(mf.t[t].x);
          mi[m].tangent[t][1] = float(mf.t[t].y);
          mi[m].tangent[t][2] = float(mf.t[t].z);
        }
      }
      put(mi.data(), sizeof(bb_manifold_info) * mi.size());
      return mi.size();
    }
    case BB_DBG_CONTACTS: {
      std::vector<bb_contact_info> ci(8 * w.manifolds.size());
      std::memset(ci.data(), 0, ci.size() * sizeof(bb_contact_info));
      for (size_t m = 0; m < w.manifolds.size(); ++m) {
        const auto& mf = w.manifolds[m];
        for (int j = 0; j < mf.cc; ++j) {
          bb_contact_info& c = ci[8 * m + j];
          const auto& s = mf.c[j];
          c.position[0] = float(s.pos.x);
          c.position[1] = float(s.pos.y);
          c.position[2] = float(s.pos.z);
          c.penetration = float(s.pen);
          c.normal_impulse = float(s.ni);
          c.tangent_impulse[0] = float(s.ti[0]);
          c.tangent_impulse[1] = float(s.ti[1]);
          // voxel manifolds: the sampled voxel and corner (in_inc); else four 8-bit ids
          c.feature = (mf.key >= VOXEL_KEY0 && mf.key < VOXEL_KEY0 + 6)
                          ? s.fp.in_inc
                          : (s.fp.in_ref & 0xFF) | ((s.fp.out_ref & 0xFF) << 8) | ((s.fp.in_inc & 0xFF) << 16) |
                                ((s.fp.out_inc & 0xFF) << 24);
          c.warm_start = s.warm;
          c.penalty = float(s.mcoef);
        }
      }
      put(ci.data(), sizeof(bb_contact_info) * ci.size());
      return ci.size();
    }
    case BB_DBG_EDGE_COLORS: {
      std::vector<uint32_t> c(w.manifolds.size());
      for (size_t m = 0; m < c.size(); ++m) c[m] = w.manifolds[m].color;
      put(c.data(), 4 * c.size());
      return c.size();
    }
    case BB_DBG_BODY_COLORS: put(w.body_color.data(), 4 * w.body_color.size()); return w.body_color.size();
    case BB_DBG_ISLANDS: put(w.island.data(), 4 * w.island.size()); return w.island.size();
    case BB_DBG_SUPPORT_DEPTH: {
      std::vector<uint32_t> d(N, 0);
      for (size_t i = 0; i < w.avbd.size() && i < N; ++i) d[i] = w.avbd[i].depth;
      put(d.data(), 4 * d.size());
      return d.size();
    }
    default: return 0;
  }
}
}  // namespace

extern "C" {

// real_is_double: 1 = FP64 checker, 0 = FP32.  threads: worker threads (1 = serial).
void* orc_create(uint32_t n, const float* pos, const float* quat, const float* vel, const float* omega,
                 const uint32_t* shape, const float* half, const uint32_t* flags, const float* mass,
                 const float* inv_mass, const float* inv_inertia, const float* friction, const float* restitution,
                 int real_is_double, int threads) {
  Handle* h = new Handle();
  h->dbl = real_is_double != 0;
  if (h->dbl) {
    h->d.reset(new World<double>(threads));
    load(*h->d, n, pos, quat, vel, omega, shape, half, flags, mass, inv_mass, inv_inertia, friction, restitution);
  } else {
    h->f.reset(new World<float>(threads));
    load(*h->f, n, pos, quat, vel, omega, shape, half, flags, mass, inv_mass, inv_inertia, friction, restitution);
  }
  return h;
}

void orc_destroy(void* hp) { delete static_cast<Handle*>(hp); }

// Voxel shapes (build_voxel_shape, src/scene_manager.hpp:488-560): returns the shape index.
uint32_t orc_add_voxel_shape(void* hp, uint32_t nx, uint32_t ny, uint32_t nz, float vs, const uint8_t* solid) {
  Handle* h = static_cast<Handle*>(hp);
  uint32_t a = h->dbl ? h->d->voxels.add(nx, ny, nz, vs, solid) : h->f->voxels.add(nx, ny, nz, vs, solid);
  return a;
}

// Binds voxel bodies (shape BB_SHAPE_VOXEL) to their shapes and sets the off-diagonal inverse
// inertia (xy, xz, yz per body; NULL = zero) of dynamic bodies.
void orc_set_voxel_bodies(void* hp, const uint32_t* voxel_index, const float* inv_inertia_off) {
  Handle* h = static_cast<Handle*>(hp);
  auto set = [&](auto& w) {
    using R = typename std::remove_reference<decltype(w.bodies[0].pos.x)>::type;
    for (size_t i = 0; i < w.n(); ++i) {
      auto& b = w.bodies[i];
      if (b.shape == BB_SHAPE_VOXEL) {
        b.voxel = voxel_index[i];
        const VoxelShape& s = w.voxels.shapes[b.voxel];
        for (int k = 0; k < 3; ++k) {
          b.lo[k] = s.lo[k];
          b.hi[k] = s.hi[k];
        }
      }
      if (inv_inertia_off && (b.flags & BB_BODY_DYNAMIC))
        b.inv_inertia_off = Vec3<R>(inv_inertia_off[3 * i], inv_inertia_off[3 * i + 1], inv_inertia_off[3 * i + 2]);
    }
  };
  if (h->dbl) set(*h->d);
  else set(*h->f);
}

// The oracle's build of voxel shape `index`: origin[3], lo[3], hi[3] into f9; solid and
// surface counts into u2; the surface list into surf (surface-count entries) when not NULL.
void orc_voxel_shape(void* hp, uint32_t index, float* f9, uint32_t* u2, uint32_t* surf) {
  Handle* h = static_cast<Handle*>(hp);
  const VoxelPool& vp = h->dbl ? h->d->voxels : h->f->voxels;
  const VoxelShape& s = vp.shapes[index];
  for (int k = 0; k < 3; ++k) {
    f9[k] = s.origin[k];
    f9[3 + k] = s.lo[k];
    f9[6 + k] = s.hi[k];
  }
  u2[0] = s.solid;
  u2[1] = s.surf_count;
  if (surf)
    for (uint32_t i = 0; i < s.surf_count; ++i) surf[i] = vp.surf[s.surf_off + i];
}

void orc_default_params(bb_solver_params* p) { default_params(p); }

void orc_set_params(void* hp, const bb_solver_params* p) {
  Handle* h = static_cast<Handle*>(hp);
  auto set = [&](auto& w) {
    // contact geometry depends on these: no pair keeps last substep's manifolds as they were
    if (p->quirks != w.p.quirks || p->penetration_cap != w.p.penetration_cap) w.frozen.clear();
    w.p = *p;
  };
  if (h->dbl) set(*h->d);
  else set(*h->f);
}

void orc_step(void* hp, float dt, uint32_t substeps) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->dbl) h->d->step(double(dt), substeps);
  else h->f->step(dt, substeps);
}

void orc_collide(void* hp, uint32_t stage) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->dbl) h->d->collide(stage);
  else h->f->collide(stage);
}

// 0: frozen pairs recompute their contacts like every other pair (for tests of the carry-over)
void orc_set_carry_frozen(void* hp, int on) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->dbl) h->d->carry_frozen = on != 0;
  else h->f->carry_frozen = on != 0;
}

// The next substep's narrow phase uses these n manifolds (bb_manifold_info, pair order) and
// their contacts (bb_contact_info, MAX_CONTACTS per manifold) as its geometry (no voxel keys).
void orc_inject_manifolds(void* hp, const bb_manifold_info* m, const bb_contact_info* c, uint32_t n) {
  Handle* h = static_cast<Handle*>(hp);
  auto set = [&](auto& w) {
    w.inj_m.assign(m, m + n);
    w.inj_c.assign(c, c + size_t(n) * MAX_CONTACTS);
    w.inj = true;
  };
  if (h->dbl) set(*h->d);
  else set(*h->f);
}

void orc_skip_warm_starting_once(void* hp) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->dbl) h->d->skip_warm_once = true;
  else h->f->skip_warm_once = true;
}

// State by id in double precision (any pointer may be NULL).
void orc_read_state(void* hp, double* pos, double* quat, double* vel, double* omega, uint32_t* flags) {
  Handle* h = static_cast<Handle*>(hp);
  auto rd = [&](auto& w) {
    for (size_t i = 0; i < w.n(); ++i) {
      auto& b = w.bodies[i];
      if (pos) { pos[3 * i] = b.pos.x; pos[3 * i + 1] = b.pos.y; pos[3 * i + 2] = b.pos.z; }
      if (quat) { quat[4 * i] = b.rot.v.x; quat[4 * i + 1] = b.rot.v.y; quat[4 * i + 2] = b.rot.v.z; quat[4 * i + 3] = b.rot.w; }
      if (vel) { vel[3 * i] = b.vel.x; vel[3 * i + 1] = b.vel.y; vel[3 * i + 2] = b.vel.z; }
      if (omega) { omega[3 * i] = b.omega.x; omega[3 * i + 1] = b.omega.y; omega[3 * i + 2] = b.omega.z; }
      if (flags) flags[i] = b.flags;
    }
  };
  if (h->dbl) rd(*h->d);
  else rd(*h->f);
}

void orc_read_stats(void* hp, bb_step_stats* s) {
  Handle* h = static_cast<Handle*>(hp);
  *s = h->dbl ? h->d->stats : h->f->stats;
}

uint64_t orc_debug_read(void* hp, uint32_t which, void* dst, uint64_t max_bytes) {
  Handle* h = static_cast<Handle*>(hp);
  return h->dbl ? debug_read(*h->d, which, dst, max_bytes) : debug_read(*h->f, which, dst, max_bytes);
}

// Stand-alone FP32 geometry used by the bit-exact tests.
uint32_t orc_morton(const float* p, const float* wmin, const float* wext) { return morton_of(p, wmin, wext); }
void orc_leaf_aabb(uint32_t shape, const float* half, const float* p, const float* q, float* out6) {
  Aabb a = leaf_aabb(shape, half, p, q);
  for (int k = 0; k < 3; ++k) {
    out6[k] = a.mn[k];
    out6[3 + k] = a.mx[k];
  }
}

// One narrow-phase query on two bodies given as (shape, half, pos, quat); returns the
// contact count and fills normal[3], key, positions[3*8], depths[8].
int orc_collide_pair(uint32_t shape_a, const float* half_a, const double* pos_a, const double* quat_a,
                     uint32_t shape_b, const float* half_b, const double* pos_b, const double* quat_b,
                     int sat_frame_quirk, double* normal, int* key, double* positions, double* depths) {
  Body<double> A, B;
  A.shape = shape_a;
  B.shape = shape_b;
  for (int k = 0; k < 3; ++k) {
    A.half[k] = half_a[k];
    B.half[k] = half_b[k];
  }
  A.pos = Vec3<double>(pos_a[0], pos_a[1], pos_a[2]);
  B.pos = Vec3<double>(pos_b[0], pos_b[1], pos_b[2]);
  A.rot = Quat<double>(Vec3<double>(quat_a[0], quat_a[1], quat_a[2]), quat_a[3]);
  B.rot = Quat<double>(Vec3<double>(quat_b[0], quat_b[1], quat_b[2]), quat_b[3]);
  SatResult<double> s;
  bool hit;
  if (shape_a == BB_SHAPE_BOX && shape_b == BB_SHAPE_BOX) hit = box_box(A, B, sat_frame_quirk != 0, s);
  else if (shape_a == BB_SHAPE_SPHERE && shape_b == BB_SHAPE_SPHERE) hit = sphere_sphere(A, B, s);
  else hit = box_sphere(A, B, s);
  if (!hit) return 0;
  normal[0] = s.normal.x;
  normal[1] = s.normal.y;
  normal[2] = s.normal.z;
  *key = s.key;
  for (int c = 0; c < s.cc; ++c) {
    positions[3 * c] = s.pos[c].x;
    positions[3 * c + 1] = s.pos[c].y;
    positions[3 * c + 2] = s.pos[c].z;
    depths[c] = s.pen[c];
  }
  return s.cc;
}

}  // extern "C"
