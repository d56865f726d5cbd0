// bb_oracle.hpp -- TEST INFRASTRUCTURE ONLY: the oracle.
//
// A single-threaded (optionally thread-pooled) CPU restatement of beat-box's per-step
// rigid-body pipeline, written from the reference's Slang compute passes.  It is the
// checker for the CUDA product library and the timed CPU baseline; it is never linked into
// the product.  Instantiated with R = double (the FP64 checker) and R = float (the
// multithreaded CPU baseline).
//
// Reference files (paths inside the reference project):
//   LBVH.slang                 src/shaders/simulation/LBVH.slang
//   RB_sim.slang               src/shaders/simulation/RB_sim.slang
//   collision_detection.slang  src/shaders/simulation/collision_detection.slang
//   extensions.slang           src/shaders/extensions.slang
//   solvers.slang              src/shaders/simulation/solvers.slang
//   islands.slang              src/shaders/simulation/islands.slang
//   coloring.slang             src/shaders/simulation/coloring.slang
//   avbd.slang                 src/shaders/simulation/avbd.slang
//   RBM                        src/rigid_body_manager.cpp (per-step task order 1284-1427)
//
// Determinism contract (where the reference orders work by atomics, the oracle uses a
// canonical order that the CUDA library reproduces):
//   * sort keys are emitted in the previous step's sorted order, so the stable radix sort
//     breaks Morton ties exactly as RB_sim.slang:75-111 + LBVH.slang:34-152 do;
//   * broad-phase pairs are sorted by (sorted index a, sorted index b), a < b;
//   * manifolds are stored in pair order (the reference appends them with an atomic);
//   * a body's manifold list is in ascending manifold order (reference: atomic list heads);
//   * the AVBD body colouring and the support-depth BFS read start-of-round state (the
//     reference reads racy in-round state, avbd.slang:880-891 / 690-724);
//   * serial overflow manifolds are solved in manifold order.
// Bit-exact stages (Morton codes, leaf AABBs, sort, LBVH topology, pair set) are computed
// in FP32 with the reference's operation order; build with -ffp-contract=off.
#pragma once
#include <algorithm>
#include <array>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../include/beatbox.h"
#include "bb_oracle_math.hpp"

namespace bbo {

static const uint32_t MAX_U32 = 0xFFFFFFFFu;
static const int MAX_CONTACTS = 8;  // MAX_CONTACT_POINT_COUNT, include/math.hpp:260
static const uint32_t MAX_COLORS = 32;
static const float PI_F = 3.14159265359f;
static const uint32_t SLEEP_VETO_BIT = 0x80000000u;
static const uint32_t SLEEP_TIMER_MASK = 0x7FFFFFFFu;

// ---------------------------------------------------------------------------------------
// Small thread pool: parallel_for over [0, n) with dynamic chunks.  Results never depend on
// the thread count (every parallel loop writes disjoint items).
class Pool {
 public:
  explicit Pool(int threads) : nthreads_(std::max(1, threads)) {
    for (int t = 1; t < nthreads_; ++t) workers_.emplace_back([this] { worker(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
  }
  int threads() const { return nthreads_; }
  template <class F> void parallel_for(size_t n, F&& f, size_t grain = 64) {
    if (nthreads_ == 1 || n <= grain) {
      for (size_t i = 0; i < n; ++i) f(i);
      return;
    }
    std::function<void(size_t)> fn = f;
    {
      std::lock_guard<std::mutex> lk(m_);
      job_ = &fn;
      n_ = n;
      grain_ = grain;
      next_.store(0);
      active_ = nthreads_ - 1;
      ++gen_;
    }
    cv_.notify_all();
    run_chunks(fn);
    std::unique_lock<std::mutex> lk(m_);
    done_cv_.wait(lk, [this] { return active_ == 0; });
    job_ = nullptr;
  }

 private:
  void run_chunks(std::function<void(size_t)>& fn) {
    for (;;) {
      size_t s = next_.fetch_add(grain_);
      if (s >= n_) break;
      size_t e = std::min(n_, s + grain_);
      for (size_t i = s; i < e; ++i) fn(i);
    }
  }
  void worker() {
    uint64_t seen = 0;
    for (;;) {
      std::function<void(size_t)>* job;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
        job = job_;
      }
      if (job) run_chunks(*job);
      {
        std::lock_guard<std::mutex> lk(m_);
        if (--active_ == 0) done_cv_.notify_one();
      }
    }
  }
  int nthreads_;
  std::vector<std::thread> workers_;
  std::mutex m_;
  std::condition_variable cv_, done_cv_;
  std::function<void(size_t)>* job_ = nullptr;
  size_t n_ = 0, grain_ = 64;
  std::atomic<size_t> next_{0};
  int active_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

// ---------------------------------------------------------------------------------------
// Data model.  Body fields follow RigidBody (include/shared.inl:335-475); the box extents
// are kept as float half extents (min = -half, max = +half).
template <class R> struct Body {
  uint32_t id = 0, flags = 0, shape = BB_SHAPE_BOX;
  float half[3] = {0.5f, 0.5f, 0.5f};  // box half extents; sphere radius in half[0]
  uint32_t voxel = 0;                  // voxel shape index (BB_SHAPE_VOXEL)
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};  // voxel bodies: body-frame box [minimum, maximum]
  Vec3<R> pos, vel, omega, prev_vel;
  Quat<R> rot;
  R mass = 0, inv_mass = 0;
  Vec3<R> inv_inertia;      // body-frame diagonal
  Vec3<R> inv_inertia_off;  // body-frame off-diagonal (xy, xz, yz); zero for boxes and spheres
  R friction = 0.5, restitution = 0;
  uint32_t sleep_timer = 0;
  uint32_t active_index = MAX_U32;
};

struct FeaturePair {
  uint32_t in_ref = 0, out_ref = 0, in_inc = 0, out_inc = 0;
};

// Contact (include/math.hpp:430-452).
template <class R> struct Contact {
  Vec3<R> pos;
  R pen = 0, ni = 0, ti[2] = {0, 0};
  R bias = 0, icoef = 0, mcoef = 0, nmass = 0, tmass[2] = {0, 0};
  Vec3<R> anchor_a, anchor_b;
  uint32_t stick = 0;
  FeaturePair fp;
  uint32_t warm = 0;
};

// Manifold (include/math.hpp:454-478).  a/b are body ids; sa/sb their sorted positions.
template <class R> struct Manifold {
  uint32_t a = 0, b = 0, sa = 0, sb = 0;
  Vec3<R> anchor_a, anchor_b;
  int key = -1;
  int32_t error = 0;
  Vec3<R> normal, t[2];
  int cc = 0;
  Contact<R> c[MAX_CONTACTS];
  uint32_t color = MAX_U32;
};

template <class R> struct AvbdState {
  Vec3<R> pos_start, pos_tilde;
  Quat<R> rot_start, rot_tilde;
  uint32_t depth = 0;
};

inline void default_params(bb_solver_params* p) {
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
  p->schedule = BB_SCHEDULE_COLOUR_BARRIER;  // execution details of the CUDA library; ignored here
  p->broad_threads = 128;
  p->narrow_blocks_per_sm = 16;
  p->pgs_stage_next = 0;
  p->bounds_mode = BB_BOUNDS_FIXED;
  for (int i = 0; i < 3; ++i) {
    p->world_min[i] = -64.0f;
    p->world_extent[i] = 128.0f;
  }
}

// ---------------------------------------------------------------------------------------
// FP32-exact geometry shared by Morton, LBVH leaves and the broad phase.

// MortonCodeGenerator::expand_bits / morton3D (LBVH.slang:8-31).
inline uint32_t expand_bits(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}
inline uint32_t morton3d(float x, float y, float z) {
  x = std::min(std::max(x * 1024.0f, 0.0f), 1023.0f);
  y = std::min(std::max(y * 1024.0f, 0.0f), 1023.0f);
  z = std::min(std::max(z * 1024.0f, 0.0f), 1023.0f);
  uint32_t xx = expand_bits(uint32_t(x)), yy = expand_bits(uint32_t(y)), zz = expand_bits(uint32_t(z));
  return xx * 4 + yy * 2 + zz;
}
// entry_generate_morton_codes (RB_sim.slang:75-111): (p - min) / extent, then morton3D.
inline uint32_t morton_of(const float p[3], const float wmin[3], const float wext[3]) {
  float n[3];
  for (int k = 0; k < 3; ++k) n[k] = (p[k] - wmin[k]) / wext[k];
  return morton3d(n[0], n[1], n[2]);
}

struct Aabb {
  float mn[3], mx[3];
};
inline float fminx(float a, float b) { return b < a ? b : a; }
inline float fmaxx(float a, float b) { return b > a ? b : a; }

// RigidBody::get_AABB_from_OBB (extensions.slang:195-210): the 8 corners of [min, max]
// pushed through object_to_world (quaternion sandwich, shared.inl:455-475).  Boxes have
// [min, max] = [-half, half]; voxel bodies their grid box [lo, hi] (off-centre: the body origin
// is the centre of mass).  Spheres: centre +- radius.
inline Aabb leaf_aabb_box(const float lo[3], const float hi[3], const float p[3], const float q[4]) {
  Aabb a;
  Quat<float> qq(Vec3<float>(q[0], q[1], q[2]), q[3]);
  for (int k = 0; k < 3; ++k) {
    a.mn[k] = FLT_MAX;
    a.mx[k] = -FLT_MAX;
  }
  for (uint32_t i = 0; i < 8; ++i) {
    Vec3<float> c((i & 1) == 0 ? lo[0] : hi[0], (i & 2) == 0 ? lo[1] : hi[1], (i & 4) == 0 ? lo[2] : hi[2]);
    Vec3<float> w = rotate_vector(qq, c);
    float wv[3] = {w.x + p[0], w.y + p[1], w.z + p[2]};
    for (int k = 0; k < 3; ++k) {
      a.mn[k] = fminx(a.mn[k], wv[k]);
      a.mx[k] = fmaxx(a.mx[k], wv[k]);
    }
  }
  return a;
}
inline Aabb leaf_aabb(uint32_t shape, const float half[3], const float p[3], const float q[4]) {
  Aabb a;
  if (shape == BB_SHAPE_SPHERE) {
    for (int k = 0; k < 3; ++k) {
      a.mn[k] = p[k] - half[0];
      a.mx[k] = p[k] + half[0];
    }
    return a;
  }
  const float lo[3] = {-half[0], -half[1], -half[2]};
  return leaf_aabb_box(lo, half, p, q);
}
// Aabb::overlap (include/math.hpp:213-217), closed intervals.
inline bool overlap(const Aabb& a, const Aabb& b) {
  return a.mn[0] <= b.mx[0] && a.mx[0] >= b.mn[0] && a.mn[1] <= b.mx[1] && a.mx[1] >= b.mn[1] &&
         a.mn[2] <= b.mx[2] && a.mx[2] >= b.mn[2];
}

// LBVH::delta / determine_range / find_split (LBVH.slang:155-221).
inline int clz32(uint32_t x) { return x == 0 ? 32 : __builtin_clz(x); }
inline int lbvh_delta(const std::vector<uint32_t>& codes, int n, int i, uint32_t code_i, int j) {
  if (j < 0 || j > n - 1) return -1;
  uint32_t code_j = codes[j];
  if (code_i == code_j) return 32 + clz32(uint32_t(i ^ j));
  return clz32(code_i ^ code_j);
}
inline void lbvh_range(const std::vector<uint32_t>& codes, int n, int index, int& first, int& last) {
  uint32_t code = codes[index];
  int dl = lbvh_delta(codes, n, index, code, index - 1);
  int dr = lbvh_delta(codes, n, index, code, index + 1);
  int d = (dr >= dl) ? 1 : -1;
  int dmin = std::min(dl, dr);
  int lmax = 2;
  while (lbvh_delta(codes, n, index, code, index + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t > 0; t >>= 1)
    if (lbvh_delta(codes, n, index, code, index + (l + t) * d) > dmin) l += t;
  int j = index + l * d;
  first = std::min(index, j);
  last = std::max(index, j);
}
inline int lbvh_split(const std::vector<uint32_t>& codes, int n, int first, int last) {
  uint32_t fc = codes[first];
  int common = lbvh_delta(codes, n, first, fc, last);
  int split = first, step = last - first;
  do {
    step = (step + 1) >> 1;
    int ns = split + step;
    if (ns < last) {
      if (lbvh_delta(codes, n, first, fc, ns) > common) split = ns;
    }
  } while (step > 1);
  return split;
}

// ---------------------------------------------------------------------------------------
// Narrow phase: OBBvsOBBCollision (collision_detection.slang:5-877), the qu3e-derived SAT
// with Sutherland-Hodgman clipping, transliterated with the reference's matrix layout.
enum Edge : uint32_t {
  POS_X_POS_Y = 0, POS_X_NEG_Y = 1, POS_X_POS_Z = 2, POS_X_NEG_Z = 3, NEG_X_POS_Y = 4, NEG_X_NEG_Y = 5,
  NEG_X_POS_Z = 6, NEG_X_NEG_Z = 7, POS_Y_POS_Z = 8, POS_Y_NEG_Z = 9, NEG_Y_POS_Z = 10, NEG_Y_NEG_Z = 11
};

template <class R> struct ClipVertex {
  Vec3<R> v;
  FeaturePair f;
};

template <class R> struct SatResult {
  int cc = 0;
  int key = -1;
  Vec3<R> normal;
  Vec3<R> pos[MAX_CONTACTS];
  R pen[MAX_CONTACTS];
  FeaturePair fp[MAX_CONTACTS];
};

// compute_incident_face (collision_detection.slang:123-243).
template <class R>
void incident_face(const Transform<R>& itx, Vec3<R> e, Vec3<R> n, ClipVertex<R> out[4]) {
  n = -itx.rotate_transpose(n);
  Vec3<R> an = vabs(n);
  Vec3<R> v[4];
  uint32_t fi[4][2];
  if (an.x > an.y && an.x > an.z) {
    if (n.x > 0) {
      v[0] = {e.x, e.y, -e.z}; v[1] = {e.x, e.y, e.z}; v[2] = {e.x, -e.y, e.z}; v[3] = {e.x, -e.y, -e.z};
      uint32_t t[4][2] = {{POS_Y_NEG_Z, POS_X_NEG_Y}, {POS_X_NEG_Y, POS_Y_POS_Z}, {POS_Y_POS_Z, NEG_X_NEG_Z}, {NEG_X_NEG_Z, POS_Y_NEG_Z}};
      std::memcpy(fi, t, sizeof(t));
    } else {
      v[0] = {-e.x, -e.y, e.z}; v[1] = {-e.x, e.y, e.z}; v[2] = {-e.x, e.y, -e.z}; v[3] = {-e.x, -e.y, -e.z};
      uint32_t t[4][2] = {{NEG_X_NEG_Y, NEG_Y_NEG_Z}, {NEG_Y_NEG_Z, POS_X_NEG_Z}, {POS_X_NEG_Z, NEG_Y_POS_Z}, {NEG_Y_POS_Z, NEG_X_NEG_Y}};
      std::memcpy(fi, t, sizeof(t));
    }
  } else if (an.y > an.x && an.y > an.z) {
    if (n.y > 0) {
      v[0] = {-e.x, e.y, e.z}; v[1] = {e.x, e.y, e.z}; v[2] = {e.x, e.y, -e.z}; v[3] = {-e.x, e.y, -e.z};
      uint32_t t[4][2] = {{POS_X_NEG_Z, POS_X_POS_Y}, {POS_X_POS_Y, POS_X_NEG_Y}, {POS_X_NEG_Y, POS_X_POS_Z}, {POS_X_POS_Z, POS_X_NEG_Z}};
      std::memcpy(fi, t, sizeof(t));
    } else {
      v[0] = {e.x, -e.y, e.z}; v[1] = {-e.x, -e.y, e.z}; v[2] = {-e.x, -e.y, -e.z}; v[3] = {e.x, -e.y, -e.z};
      uint32_t t[4][2] = {{NEG_X_NEG_Z, NEG_X_POS_Y}, {NEG_X_POS_Y, NEG_X_NEG_Y}, {NEG_X_NEG_Y, NEG_X_POS_Z}, {NEG_X_POS_Z, NEG_X_NEG_Z}};
      std::memcpy(fi, t, sizeof(t));
    }
  } else {
    if (n.z > 0) {
      v[0] = {-e.x, e.y, e.z}; v[1] = {-e.x, -e.y, e.z}; v[2] = {e.x, -e.y, e.z}; v[3] = {e.x, e.y, e.z};
      uint32_t t[4][2] = {{POS_X_POS_Y, NEG_Y_NEG_Z}, {NEG_Y_NEG_Z, NEG_X_POS_Y}, {NEG_X_POS_Y, POS_Y_POS_Z}, {POS_Y_POS_Z, POS_X_POS_Y}};
      std::memcpy(fi, t, sizeof(t));
    } else {
      v[0] = {e.x, -e.y, -e.z}; v[1] = {-e.x, -e.y, -e.z}; v[2] = {-e.x, e.y, -e.z}; v[3] = {e.x, e.y, -e.z};
      uint32_t t[4][2] = {{POS_Y_NEG_Z, NEG_X_POS_Z}, {NEG_X_POS_Z, NEG_Y_POS_Z}, {NEG_Y_POS_Z, POS_X_POS_Z}, {POS_X_POS_Z, POS_Y_NEG_Z}};
      std::memcpy(fi, t, sizeof(t));
    }
  }
  for (int i = 0; i < 4; ++i) {
    out[i].v = itx.transform(v[i]);
    out[i].f = FeaturePair();  // in/out_reference are not written by the reference: taken as 0
    out[i].f.in_inc = fi[i][0];
    out[i].f.out_inc = fi[i][1];
  }
}

// compute_reference_edges_and_basis (collision_detection.slang:245-336).
template <class R>
void reference_edges(Vec3<R> er, const Transform<R>& rtx, Vec3<R> n, int axis, uint32_t clip[4], Mat3<R>& basis,
                     Vec3<R>& e) {
  n = rtx.rotate_transpose(n);
  if (axis > 2) axis -= 3;
  const Mat3<R>& r = rtx.rot;
  Vec3<R> r0 = r.row(0), r1 = r.row(1), r2 = r.row(2);
  auto set = [&](uint32_t a, uint32_t b, uint32_t c, uint32_t d) { clip[0] = a; clip[1] = b; clip[2] = c; clip[3] = d; };
  if (axis == 0) {
    if (n.x > 0) { set(POS_X_NEG_Y, POS_Y_POS_Z, NEG_X_NEG_Z, POS_Y_NEG_Z); e = {er.y, er.z, er.x}; basis = Mat3<R>::rows(r1, r2, r0); }
    else { set(NEG_Y_NEG_Z, POS_X_NEG_Z, NEG_Y_POS_Z, NEG_X_NEG_Y); e = {er.z, er.y, er.x}; basis = Mat3<R>::rows(r2, r1, -r0); }
  } else if (axis == 1) {
    if (n.y > 0) { set(POS_X_POS_Y, POS_X_NEG_Y, POS_X_POS_Z, POS_X_NEG_Z); e = {er.z, er.x, er.y}; basis = Mat3<R>::rows(r2, r0, r1); }
    else { set(NEG_X_POS_Y, NEG_X_NEG_Y, NEG_X_POS_Z, NEG_X_NEG_Z); e = {er.z, er.x, er.y}; basis = Mat3<R>::rows(r2, -r0, -r1); }
  } else {
    if (n.z > 0) { set(NEG_Y_NEG_Z, NEG_X_POS_Y, POS_Y_POS_Z, POS_X_POS_Y); e = {er.y, er.x, er.z}; basis = Mat3<R>::rows(-r1, r0, r2); }
    else { set(NEG_X_POS_Z, NEG_Y_POS_Z, POS_X_POS_Z, POS_Y_NEG_Z); e = {er.y, er.x, er.z}; basis = Mat3<R>::rows(-r1, -r0, -r2); }
  }
}

// ortographic_clip (collision_detection.slang:352-387).  Output capped at 8 vertices.
template <class R>
int ortho_clip(R sign, R e, int axis, uint32_t clip_edge, const ClipVertex<R>* in, int in_count, ClipVertex<R>* out) {
  const R TH = R(0.005);
  auto on = [&](R v) { return v < TH && v > -TH; };
  int oc = 0;
  auto push = [&](const ClipVertex<R>& c) { if (oc < MAX_CONTACTS) out[oc++] = c; };
  ClipVertex<R> a = in[in_count - 1];
  for (int i = 0; i < in_count; ++i) {
    ClipVertex<R> b = in[i];
    R da = sign * a.v[axis] - e;
    R db = sign * b.v[axis] - e;
    if ((da < 0 && db < 0) || on(da) || on(db)) {
      push(b);
    } else if (da < 0 && db >= 0) {
      ClipVertex<R> cv;
      cv.f = b.f;
      cv.v = a.v + (b.v - a.v) * (da / (da - db));
      cv.f.out_ref = clip_edge;
      push(cv);
    } else if (da >= 0 && db < 0) {
      ClipVertex<R> cv;
      cv.f = a.f;
      cv.v = a.v + (b.v - a.v) * (da / (da - db));
      cv.f.in_ref = clip_edge;
      push(cv);
      push(b);
    }
    a = b;
  }
  return oc;
}

// clip (collision_detection.slang:391-449).  Returns -1 on a clip error (10..13).
template <class R>
int clip_face(const Transform<R>& tx, Vec3<R> e, const uint32_t clip[4], const ClipVertex<R> inc[4],
              ClipVertex<R> outv[MAX_CONTACTS], R depths[MAX_CONTACTS]) {
  ClipVertex<R> in[MAX_CONTACTS], out[MAX_CONTACTS];
  for (int i = 0; i < 4; ++i) {
    in[i].v = tx.transform_transpose(inc[i].v);
    in[i].f = inc[i].f;
  }
  int oc = ortho_clip(R(1), e.x, 0, clip[0], in, 4, out);
  if (oc == 0) return -1;
  int ic = ortho_clip(R(1), e.y, 1, clip[1], out, oc, in);
  if (ic == 0) return -1;
  oc = ortho_clip(R(-1), e.x, 0, clip[2], in, ic, out);
  if (oc == 0) return -1;
  ic = ortho_clip(R(-1), e.y, 1, clip[3], out, oc, in);
  if (ic == 0) return -1;
  int n = 0;
  for (int i = 0; i < ic; ++i) {
    R d = in[i].v.z - e.z;
    if (d <= 0) {
      outv[n].v = tx.transform(in[i].v);
      outv[n].f = in[i].f;
      depths[n] = d;
      ++n;
    }
  }
  return n;
}

template <class R> inline R c_sign(R x) { return x < 0 ? R(-1) : R(1); }

// support_edge (collision_detection.slang:456-497).
template <class R> void support_edge(const Transform<R>& tx, Vec3<R> e, Vec3<R> n, Vec3<R>& ca, Vec3<R>& cb) {
  n = tx.rotate_transpose(n);
  Vec3<R> an = vabs(n);
  int axis;
  if (an.x <= an.y && an.x <= an.z) axis = 0;
  else if (an.y <= an.x && an.y <= an.z) axis = 1;
  else axis = 2;
  Vec3<R> v0(c_sign(n.x) * e.x, c_sign(n.y) * e.y, c_sign(n.z) * e.z), v1 = v0;
  v0[axis] = e[axis];
  v1[axis] = -e[axis];
  ca = tx.transform(v0);
  cb = tx.transform(v1);
}

// edges_contact (collision_detection.slang:499-548), segment-segment closest points.
template <class R> void edges_contact(Vec3<R> pa, Vec3<R> qa, Vec3<R> pb, Vec3<R> qb, Vec3<R>& ca, Vec3<R>& cb) {
  Vec3<R> da = qa - pa, db = qb - pb, r = pa - pb;
  R a = dot(da, da), e = dot(db, db), f = dot(db, r), c = dot(da, r), b = dot(da, db);
  R denom = a * e - b * b;
  auto clamp01 = [](R x) { return std::min(std::max(x, R(0)), R(1)); };
  if (denom == 0) {
    R t = clamp01(dot(r, da) / a);
    ca = pa + da * t;
    Vec3<R> s = ca - pb;
    R u = clamp01(dot(s, db) / e);
    cb = pb + db * u;
    return;
  }
  R ta = clamp01((b * f - c * e) / denom);
  R tb = (b * ta + f) / e;
  if (tb < 0) {
    tb = 0;
    ta = clamp01(-c / a);
  } else if (tb > 1) {
    tb = 1;
    ta = clamp01((b - c) / a);
  }
  ca = pa + da * ta;
  cb = pb + db * tb;
}

// Slang RigidBody::get_rotation_matrix (shared.inl:367-375): transpose(to_matrix()), the
// matrix whose rows are the body axes.
template <class R> inline Mat3<R> body_axes(const Quat<R>& q) { return transpose(to_matrix(q)); }

// OBBvsOBBCollision::collision_detection (collision_detection.slang:562-876).
// sat_frame_quirk selects the reference's relative rotation C = mul(transpose(A), B) with
// A, B the axis-row matrices; otherwise C = mul(B, transpose(A)) (rows = B axes in A's
// frame), which the formulas below assume.
template <class R>
bool box_box(const Body<R>& A, const Body<R>& B, bool sat_frame_quirk, SatResult<R>& out) {
  out.cc = 0;
  out.key = -1;
  Transform<R> txa{body_axes(A.rot), A.pos}, txb{body_axes(B.rot), B.pos};
  Vec3<R> ea(A.half[0], A.half[1], A.half[2]), eb(B.half[0], B.half[1], B.half[2]);
  Mat3<R> C = sat_frame_quirk ? mul_mm(transpose(txa.rot), txb.rot) : mul_mm(txb.rot, transpose(txa.rot));
  Mat3<R> absC = mabs(C);
  const R THRESH = R(0.9998);
  bool parallel = false;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      if (absC.m[i][j] > THRESH) parallel = true;
  Transform<R> txc{C, Vec3<R>()}, txac{absC, Vec3<R>()};
  Vec3<R> t = rotate_vector_inverse(A.rot, B.pos - A.pos);
  R a_max = -FLT_MAX, b_max = -FLT_MAX, e_max = -FLT_MAX;
  int a_axis = -1, b_axis = -1, e_axis = -1;
  Vec3<R> n_a, n_b, n_e;
  for (int i = 0; i < 3; ++i) {
    R s = std::fabs(t[i]) - (ea[i] + dot(txac.get_inverse_axis(i), eb));
    if (s > 0) return false;
    if (s > a_max) { a_max = s; a_axis = i; n_a = txa.get_axis(i); }
  }
  for (int i = 0; i < 3; ++i) {
    R proj = dot(t, txc.get_axis(i));
    R s = std::fabs(proj) - (eb[i] + dot(txac.get_axis(i), ea));
    if (s > 0) return false;
    if (s > b_max) { b_max = s; b_axis = 3 + i; n_b = txb.get_axis(i); }
  }
  if (!parallel) {
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j) {
        int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        R rA = ea[i1] * absC.m[j][i2] + ea[i2] * absC.m[j][i1];
        R rB = eb[j1] * absC.m[j2][i] + eb[j2] * absC.m[j1][i];
        R s = std::fabs(t[i2] * C.m[j][i1] - t[i1] * C.m[j][i2]) - (rA + rB);
        Vec3<R> axis;
        axis[i1] = -C.m[j][i2];
        axis[i2] = C.m[j][i1];
        if (s > 0) return false;
        R l = R(1) / length(axis);
        s *= l;
        if (s > e_max) { e_max = s; e_axis = 6 + i * 3 + j; n_e = axis * l; }
      }
    }
  }
  const R rel = R(0.95), abs_t = R(0.01);
  int axis;
  R s_max;
  Vec3<R> normal;
  R face_max = std::max(a_max, b_max);
  if (rel * e_max > face_max + abs_t) { axis = e_axis; s_max = e_max; normal = n_e; }
  else if (rel * b_max > a_max + abs_t) { axis = b_axis; s_max = b_max; normal = n_b; }
  else { axis = a_axis; s_max = a_max; normal = n_a; }
  if (dot(normal, B.pos - A.pos) < 0) normal = -normal;
  if (axis == -1) return false;
  if (axis <= 5) {
    Transform<R> rtx, itx;
    Vec3<R> er, ei;
    bool flip = false;
    if (axis <= 2) { rtx = txa; itx = txb; er = ea; ei = eb; }
    else { rtx = txb; itx = txa; er = eb; ei = ea; flip = true; normal = -normal; }
    ClipVertex<R> inc[4];
    incident_face(itx, ei, normal, inc);
    uint32_t clip[4];
    Mat3<R> basis;
    Vec3<R> e;
    reference_edges(er, rtx, normal, axis, clip, basis, e);
    Transform<R> tx{basis, rtx.pos};
    ClipVertex<R> outv[MAX_CONTACTS];
    R depths[MAX_CONTACTS];
    int n = clip_face(tx, e, clip, inc, outv, depths);
    if (n < 0) return false;  // clip error: no manifold (collision_detection.slang:791-807)
    if (n > 0) {
      out.cc = n;
      out.normal = flip ? -normal : normal;
      for (int i = 0; i < n; ++i) {
        FeaturePair f = outv[i].f;
        if (flip) {
          std::swap(f.in_ref, f.in_inc);
          std::swap(f.out_ref, f.out_inc);
        }
        out.fp[i] = f;
        out.pos[i] = outv[i].v;
        out.pen[i] = depths[i];
      }
    }
  } else {
    normal = txa.rotate(normal);
    if (dot(normal, B.pos - A.pos) < 0) normal = -normal;
    Vec3<R> pa, qa, pb, qb, ca, cb;
    support_edge(txa, ea, normal, pa, qa);
    support_edge(txb, eb, -normal, pb, qb);
    edges_contact(pa, qa, pb, qb, ca, cb);
    out.cc = 1;
    out.normal = normal;
    out.pos[0] = (ca + cb) * R(0.5);
    out.pen[0] = s_max;
    FeaturePair f;
    f.in_ref = f.out_ref = f.in_inc = f.out_inc = uint32_t(axis);
    out.fp[0] = f;
  }
  out.key = axis;
  return out.cc > 0;
}

// Sphere contacts (no reference counterpart; first principles).  One contact at the
// midpoint between the two surface points, normal from A to B, depth <= 0 on overlap.
static const int KEY_SPHERE_SPHERE = 20;
static const int KEY_BOX_SPHERE = 21;  // A box, B sphere
static const int KEY_SPHERE_BOX = 22;  // A sphere, B box
template <class R> bool sphere_sphere(const Body<R>& A, const Body<R>& B, SatResult<R>& out) {
  Vec3<R> d = B.pos - A.pos;
  R ra = A.half[0], rb = B.half[0];
  R dist = length(d);
  if (dist > ra + rb) return false;
  Vec3<R> n = dist > R(1e-9) ? d / dist : Vec3<R>(0, 1, 0);
  R pen = dist - (ra + rb);
  out.cc = 1;
  out.key = KEY_SPHERE_SPHERE;
  out.normal = n;
  out.pen[0] = pen;
  out.pos[0] = A.pos + n * (ra + pen * R(0.5));
  FeaturePair f;
  f.in_ref = f.out_ref = f.in_inc = f.out_inc = KEY_SPHERE_SPHERE;
  out.fp[0] = f;
  return true;
}
// box (X) against sphere (S); normal returned from the box towards the sphere.
template <class R>
bool box_sphere_core(const Body<R>& X, const Body<R>& S, Vec3<R>& n, R& pen, Vec3<R>& pos) {
  R r = S.half[0];
  Vec3<R> e(X.half[0], X.half[1], X.half[2]);
  Vec3<R> c = rotate_vector_inverse(X.rot, S.pos - X.pos);
  Vec3<R> q(std::min(std::max(c.x, -e.x), e.x), std::min(std::max(c.y, -e.y), e.y), std::min(std::max(c.z, -e.z), e.z));
  bool inside = std::fabs(c.x) < e.x && std::fabs(c.y) < e.y && std::fabs(c.z) < e.z;
  if (!inside) {
    Vec3<R> dl = c - q;
    R dist = length(dl);
    if (dist > r) return false;
    Vec3<R> nl = dist > R(1e-9) ? dl / dist : Vec3<R>(0, 1, 0);
    n = rotate_vector(X.rot, nl);
    pen = dist - r;
    Vec3<R> box_pt = X.pos + rotate_vector(X.rot, q);
    Vec3<R> sph_pt = S.pos - n * r;
    pos = (box_pt + sph_pt) * R(0.5);
    return true;
  }
  int ax = 0;
  R best = e.x - std::fabs(c.x);
  for (int k = 1; k < 3; ++k) {
    R gap = e[k] - std::fabs(c[k]);
    if (gap < best) { best = gap; ax = k; }
  }
  Vec3<R> nl;
  nl[ax] = c[ax] < 0 ? R(-1) : R(1);
  n = rotate_vector(X.rot, nl);
  pen = -best - r;
  Vec3<R> face = c;
  face[ax] = nl[ax] * e[ax];
  Vec3<R> box_pt = X.pos + rotate_vector(X.rot, face);
  Vec3<R> sph_pt = S.pos - n * r;
  pos = (box_pt + sph_pt) * R(0.5);
  return true;
}
template <class R> bool box_sphere(const Body<R>& A, const Body<R>& B, SatResult<R>& out) {
  Vec3<R> n, pos;
  R pen;
  int key;
  if (A.shape == BB_SHAPE_BOX) {
    if (!box_sphere_core(A, B, n, pen, pos)) return false;
    key = KEY_BOX_SPHERE;
  } else {
    if (!box_sphere_core(B, A, n, pen, pos)) return false;
    n = -n;
    key = KEY_SPHERE_BOX;
  }
  out.cc = 1;
  out.key = key;
  out.normal = n;
  out.pen[0] = pen;
  out.pos[0] = pos;
  FeaturePair f;
  f.in_ref = f.out_ref = f.in_inc = f.out_inc = uint32_t(key);
  out.fp[0] = f;
  return true;
}

// Manifold::compute_basis (extensions.slang:262-272).
template <class R> void compute_basis(Manifold<R>& m) {
  Vec3<R> n = m.normal, t0;
  if (std::fabs(n.x) > std::fabs(n.y)) t0 = Vec3<R>(n.z, 0, -n.x);
  else t0 = Vec3<R>(0, -n.z, n.y);
  t0 = normalize(t0);
  m.t[0] = t0;
  m.t[1] = cross(t0, n);
}

// Manifold::update_from_old (extensions.slang:306-473).
template <class R> void update_from_old(Manifold<R>& m, const Manifold<R>& old, bool swapped) {
  R sgn = swapped ? R(-1) : R(1);
  bool cross_key = m.key != old.key || swapped;
  if (cross_key) {
    if (dot(m.normal, old.normal * sgn) <= R(0.7)) return;
  }
  uint32_t used_old = 0, matched_new = 0;
  for (int i = 0; !cross_key && i < m.cc; ++i) {
    for (int j = 0; j < old.cc; ++j) {
      if (used_old & (1u << j)) continue;
      const Contact<R>& oc = old.c[j];
      Contact<R>& nc = m.c[i];
      bool feat = oc.fp.in_inc == nc.fp.in_inc && oc.fp.out_inc == nc.fp.out_inc;
      Vec3<R> dp = oc.pos - nc.pos;
      bool close = dot(dp, dp) < R(0.1) * R(0.1);
      if (feat && close) {
        nc.ni = oc.ni;
        nc.ti[0] = oc.ti[0];
        nc.ti[1] = oc.ti[1];
        nc.mcoef = oc.mcoef;
        nc.tmass[0] = oc.tmass[0];
        nc.tmass[1] = oc.tmass[1];
        nc.stick = oc.stick;
        if (oc.stick != 0) {
          nc.anchor_a = oc.anchor_a;
          nc.anchor_b = oc.anchor_b;
        }
        Vec3<R> d2 = nc.pos - oc.pos;
        if (dot(d2, d2) < R(0.01)) nc.pos = oc.pos;
        nc.warm = std::min(255u, oc.warm + 1u);
        used_old |= 1u << j;
        matched_new |= 1u << i;
        break;
      }
    }
  }
  const R radius2 = R(0.1225);
  for (int round = 0; round < std::max(m.cc, 0); ++round) {
    R best_d2 = radius2;
    int bi = -1, bj = -1;
    for (int i = 0; i < m.cc; ++i) {
      if (matched_new & (1u << i)) continue;
      for (int j = 0; j < old.cc; ++j) {
        if (used_old & (1u << j)) continue;
        Vec3<R> dp = m.c[i].pos - old.c[j].pos;
        R d2 = dot(dp, dp);
        if (d2 < best_d2) { best_d2 = d2; bi = i; bj = j; }
      }
    }
    if (bi < 0) break;
    const Contact<R>& oc = old.c[bj];
    Contact<R>& nc = m.c[bi];
    nc.ni = oc.ni;
    nc.ti[0] = oc.ti[0] * sgn;
    nc.ti[1] = oc.ti[1];
    nc.mcoef = oc.mcoef;
    nc.tmass[0] = oc.tmass[0];
    nc.tmass[1] = oc.tmass[1];
    nc.stick = oc.stick;
    if (oc.stick != 0) {
      nc.anchor_a = swapped ? oc.anchor_b : oc.anchor_a;
      nc.anchor_b = swapped ? oc.anchor_a : oc.anchor_b;
    }
    nc.fp = oc.fp;
    nc.warm = std::min(255u, oc.warm + 1u);
    matched_new |= 1u << bi;
    used_old |= 1u << bj;
  }
  R deep_new = 0, deep_old = 0;
  for (int i = 0; i < m.cc; ++i) deep_new = std::min(deep_new, m.c[i].pen);
  for (int j = 0; j < old.cc; ++j) deep_old = std::min(deep_old, old.c[j].pen);
  R v = std::min(std::max((deep_new - deep_old) * R(10000), R(-32000)), R(32000));
  m.error = int32_t(v);
}

// gc_hash / gc_pair_id / gc_priority (coloring.slang:114-138) and avbd_priority
// (avbd.slang:58-63).
inline uint32_t gc_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
inline uint32_t gc_pair_id(uint32_t ida, uint32_t idb, int key) {
  uint32_t lo = std::min(ida, idb), hi = std::max(ida, idb);
  return gc_hash(lo * 0x9e3779b9u + hi * 0x85ebca6bu + uint32_t(key) * 0xc2b2ae35u);
}
inline uint32_t gc_priority(uint32_t pair_id, uint32_t round) {
  uint32_t h = gc_hash(pair_id + round * 0x85ebca6bu) & 0xFFFu;
  if (h == 0u) h = 1u;
  return (h << 20) | (pair_id & 0xFFFFFu);
}
inline uint32_t avbd_priority(uint32_t body, uint32_t round) {
  uint32_t x = body * 0x9e3779b9u + round * 0x85ebca6bu;
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return ((x & 0xFFFu) << 20) | (body & 0xFFFFFu);
}

}  // namespace bbo
