// bb_oracle_voxel.hpp -- TEST INFRASTRUCTURE ONLY: voxel (concave) bodies in the oracle.
//
// Restates the reference's voxel-bitmask narrow phase (src/shaders/simulation/
// collision_detection.slang:1001-1512), its shape pool (VoxelShape, include/shared.inl:938-951)
// and the scene builder that fills the pool (build_voxel_shape, src/scene_manager.hpp:488-560).
// A voxel body is an occupancy bitmask over a small grid plus the list of its surface cells.
// A pair with a voxel body emits up to six manifolds, one per contact-face direction of the
// non-sampled body (keys 90..95); every other stage consumes them as ordinary manifolds.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

#include "bb_oracle.hpp"

namespace bbo {

static const int VOXEL_KEY0 = 90;  // key of the code-0 manifold (-x face); code c has key 90 + c

// VoxelShape with the body-frame box RigidBody::minimum/maximum precomputed as the builder
// writes it (scene_manager.hpp:553-554): lo = grid_origin, hi = grid_origin + dims * vs.
struct VoxelShape {
  uint32_t dims[3] = {0, 0, 0};
  float vs = 0;
  float origin[3] = {0, 0, 0};  // body-frame corner of cell (0,0,0) = minus the centre of mass
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  uint32_t occ_off = 0, surf_off = 0, surf_count = 0, solid = 0;
};

struct VoxelPool {
  std::vector<VoxelShape> shapes;
  std::vector<uint32_t> occ, surf;

  // build_voxel_shape (scene_manager.hpp:488-560): centre of mass in double, occupancy bits
  // x-major, surface cells in z, y, x order tagged with their first empty neighbour direction
  // (-x, +x, -y, +y, -z, +z).  solid[x + y*nx + z*nx*ny] != 0 marks a solid cell.
  uint32_t add(uint32_t nx, uint32_t ny, uint32_t nz, float vs, const uint8_t* solid) {
    VoxelShape s;
    s.dims[0] = nx;
    s.dims[1] = ny;
    s.dims[2] = nz;
    s.vs = vs;
    auto at = [&](int x, int y, int z) -> bool {
      if (x < 0 || y < 0 || z < 0 || x >= int(nx) || y >= int(ny) || z >= int(nz)) return false;
      return solid[size_t(x) + size_t(y) * nx + size_t(z) * nx * ny] != 0;
    };
    double cx = 0, cy = 0, cz = 0;
    uint32_t count = 0;
    for (uint32_t z = 0; z < nz; ++z)
      for (uint32_t y = 0; y < ny; ++y)
        for (uint32_t x = 0; x < nx; ++x)
          if (at(int(x), int(y), int(z))) {
            cx += x + 0.5;
            cy += y + 0.5;
            cz += z + 0.5;
            ++count;
          }
    s.solid = count;
    if (count) {
      cx = cx / double(count) * double(vs);
      cy = cy / double(count) * double(vs);
      cz = cz / double(count) * double(vs);
    }
    s.origin[0] = -float(cx);
    s.origin[1] = -float(cy);
    s.origin[2] = -float(cz);
    for (int k = 0; k < 3; ++k) {
      s.lo[k] = s.origin[k];
      s.hi[k] = s.origin[k] + float(s.dims[k]) * vs;
    }
    const uint64_t bits = uint64_t(nx) * ny * nz;
    s.occ_off = uint32_t(occ.size());
    occ.resize(occ.size() + size_t((bits + 31) / 32), 0u);
    s.surf_off = uint32_t(surf.size());
    static const int nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (uint32_t z = 0; z < nz; ++z)
      for (uint32_t y = 0; y < ny; ++y)
        for (uint32_t x = 0; x < nx; ++x) {
          if (!at(int(x), int(y), int(z))) continue;
          const uint64_t b = uint64_t(x) + uint64_t(y) * nx + uint64_t(z) * nx * ny;
          occ[s.occ_off + size_t(b / 32)] |= 1u << (b % 32);
          for (uint32_t dd = 0; dd < 6; ++dd)
            if (!at(int(x) + nb[dd][0], int(y) + nb[dd][1], int(z) + nb[dd][2])) {
              surf.push_back(x | (y << 8) | (z << 16) | (dd << 24));
              break;
            }
        }
    s.surf_count = uint32_t(surf.size()) - s.surf_off;
    shapes.push_back(s);
    return uint32_t(shapes.size() - 1);
  }

  // voxel_occ_bit (collision_detection.slang:1009-1018): out-of-grid cells are empty
  bool bit(const VoxelShape& s, int x, int y, int z) const {
    if (x < 0 || y < 0 || z < 0 || x >= int(s.dims[0]) || y >= int(s.dims[1]) || z >= int(s.dims[2])) return false;
    const uint32_t b = uint32_t(x) + uint32_t(y) * s.dims[0] + uint32_t(z) * s.dims[0] * s.dims[1];
    return ((occ[s.occ_off + b / 32u] >> (b % 32u)) & 1u) != 0u;
  }
};

template <class R> inline R vget(const Vec3<R>& v, uint32_t k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
template <class R> inline Vec3<R> unit_axis(uint32_t k, R s) {
  return Vec3<R>(k == 0 ? s : R(0), k == 1 ? s : R(0), k == 2 ? s : R(0));
}
inline uint32_t pack_cell(int x, int y, int z) {
  return uint32_t(x & 0xFF) | (uint32_t(y & 0xFF) << 8) | (uint32_t(z & 0xFF) << 16);
}

// The body's box [minimum, maximum] in its own frame: the voxel grid box, else +-half (a sphere
// is read as its bounding cube, as the reference's voxel path reads any non-voxel body).
template <class R> void body_box(const Body<R>& b, const VoxelPool& vp, Vec3<R>& lo, Vec3<R>& hi) {
  if (b.shape == BB_SHAPE_VOXEL) {
    const VoxelShape& s = vp.shapes[b.voxel];
    lo = Vec3<R>(s.lo[0], s.lo[1], s.lo[2]);
    hi = Vec3<R>(s.hi[0], s.hi[1], s.hi[2]);
  } else {
    const float h1 = b.shape == BB_SHAPE_SPHERE ? b.half[0] : b.half[1];
    const float h2 = b.shape == BB_SHAPE_SPHERE ? b.half[0] : b.half[2];
    lo = Vec3<R>(-b.half[0], -h1, -h2);
    hi = Vec3<R>(b.half[0], h1, h2);
  }
}

// VoxelManifoldReducer (collision_detection.slang:1032-1093): per extreme direction of the
// contact face (the four diagonals of the two tangent coordinates) the winning sample, ranked
// by half-voxel score bucket (higher wins), then depth bucket (deeper wins), then the lower
// voxel id.  The ranking is a strict total order (voxel ids are unique within a surface list),
// so the winners do not depend on the order the samples arrive in.  The normal sums of the
// reference reducer feed nothing downstream and are not kept.
template <class R> struct VoxelReducer {
  Vec3<R> pos[4], nrm[4];
  R pen[4], score[4];
  uint32_t fa[4], fb[4];
  uint32_t samples = 0, interior = 0;
  VoxelReducer() {
    for (int o = 0; o < 4; ++o) {
      pen[o] = R(1.0e9);
      score[o] = R(-1.0e30);
      fa[o] = 0;
      fb[o] = 0;
    }
  }
  void add(Vec3<R> p, R pe, Vec3<R> n, uint32_t a, uint32_t b, R su, R sv, R quant) {
    const R sc4[4] = {su + sv, su - sv, -su + sv, -su - sv};
    const int nbk = int(std::floor(pe / quant));
    for (int o = 0; o < 4; ++o) {
      const bool empty = pen[o] > R(0.5e9);
      const int nbs = int(std::floor(sc4[o] / quant));
      const int obs = empty ? -2147483640 : int(std::floor(score[o] / quant));
      const int obk = empty ? 0 : int(std::floor(pen[o] / quant));
      if (empty || nbs > obs || (nbs == obs && (nbk < obk || (nbk == obk && a < fa[o])))) {
        pos[o] = p;
        pen[o] = pe;
        nrm[o] = n;
        fa[o] = a;
        fb[o] = b;
        score[o] = sc4[o];
      }
    }
    ++samples;
  }
};

// voxel_sample_body (collision_detection.slang:1100-1269): every surface cell centre of the
// sampled body r1 against body r2's solid (voxel cells, or r2's box), for the pass `code`
// (axis code / 2, sign + when code is odd).  A sample joins the pass if the pass direction is
// an exit of r2's solid within a 0.15-voxel band of the shallowest exit; its depth is measured
// along the pass axis, with a hover band for centres in an empty cell just outside an occupied
// one.
template <class R>
void voxel_sample(const Body<R>& r1, const VoxelShape& s1, const Body<R>& r2, const VoxelShape* s2, bool s2_vox,
                  const VoxelPool& vp, VoxelReducer<R>& red, uint32_t code) {
  const R vs1 = s1.vs;
  const Vec3<R> a0 = rotate_vector_inverse(r2.rot, rotate_vector(r1.rot, Vec3<R>(1, 0, 0)));
  const Vec3<R> a1 = rotate_vector_inverse(r2.rot, rotate_vector(r1.rot, Vec3<R>(0, 1, 0)));
  const Vec3<R> a2 = rotate_vector_inverse(r2.rot, rotate_vector(r1.rot, Vec3<R>(0, 0, 1)));
  const Vec3<R> sup = R(0.5) * vs1 *
                      Vec3<R>(std::fabs(a0.x) + std::fabs(a1.x) + std::fabs(a2.x),
                              std::fabs(a0.y) + std::fabs(a1.y) + std::fabs(a2.y),
                              std::fabs(a0.z) + std::fabs(a1.z) + std::fabs(a2.z));
  const uint32_t axk = code / 2u;
  const R sgn = (code & 1u) ? R(1) : R(-1);
  const int isgn = (code & 1u) ? 1 : -1;
  const R sup_a = vget(sup, axk);
  Vec3<R> lo2, hi2;
  body_box(r2, vp, lo2, hi2);
  const Vec3<R> half2 = (hi2 - lo2) * R(0.5), co2 = (hi2 + lo2) * R(0.5);
  for (uint32_t i = 0; i < s1.surf_count; ++i) {
    const uint32_t e = vp.surf[s1.surf_off + i];
    const Vec3<R> local(R(s1.origin[0]) + (R(e & 0xFFu) + R(0.5)) * vs1,
                        R(s1.origin[1]) + (R((e >> 8) & 0xFFu) + R(0.5)) * vs1,
                        R(s1.origin[2]) + (R((e >> 16) & 0xFFu) + R(0.5)) * vs1);
    const Vec3<R> pw = r1.pos + rotate_vector(r1.rot, local);
    R pe, su, sv;
    Vec3<R> n_out;
    uint32_t fb;
    if (s2_vox) {
      const R vs2 = s2->vs;
      const Vec3<R> org2(s2->origin[0], s2->origin[1], s2->origin[2]);
      const Vec3<R> l2 = rotate_vector_inverse(r2.rot, pw - r2.pos);
      su = axk == 0 ? l2.y : l2.x;
      sv = axk == 2 ? l2.y : l2.z;
      const Vec3<R> g = (l2 - org2) / vs2;
      int c[3] = {int(std::floor(g.x)), int(std::floor(g.y)), int(std::floor(g.z))};
      if (!vp.bit(*s2, c[0], c[1], c[2])) {
        int ci[3] = {c[0], c[1], c[2]};
        ci[axk] -= isgn;
        if (!vp.bit(*s2, ci[0], ci[1], ci[2])) continue;
        const R dh = vget(l2, axk) - (vget(org2, axk) + (R(ci[axk]) + R(0.5)) * vs2);
        const R ovh = (R(0.5) * vs2 + sup_a) - sgn * dh;
        n_out = rotate_vector(r2.rot, unit_axis(axk, sgn));
        pe = -ovh;
        fb = pack_cell(ci[0], ci[1], ci[2]);
      } else {
        const Vec3<R> cell(static_cast<R>(c[0]), static_cast<R>(c[1]), static_cast<R>(c[2]));
        const Vec3<R> ccl = org2 + (cell + Vec3<R>(0.5, 0.5, 0.5)) * vs2;
        const Vec3<R> dl = l2 - ccl;
        R best = R(1e9);
        for (uint32_t ax = 0; ax < 3; ++ax) {
          const R di = vget(dl, ax);
          int nbc[3] = {c[0], c[1], c[2]};
          nbc[ax] += di >= R(0) ? 1 : -1;
          if (vp.bit(*s2, nbc[0], nbc[1], nbc[2])) continue;  // more solid that way: not an exit
          const R ov = (R(0.5) * vs2 + vget(sup, ax)) - std::fabs(di);
          if (ov < best) best = ov;
        }
        if (best > R(0.5e9)) {  // enclosed on the near sides: deep interior
          red.interior += 1;
          continue;
        }
        int pn[3] = {c[0], c[1], c[2]};
        pn[axk] += isgn;
        if (vp.bit(*s2, pn[0], pn[1], pn[2])) continue;  // the pass axis is no exit here
        const R ovp = (R(0.5) * vs2 + sup_a) - sgn * vget(dl, axk);
        if (ovp > best + R(0.15) * vs2) continue;  // dominated by a shallower exit
        n_out = rotate_vector(r2.rot, unit_axis(axk, sgn));
        pe = -ovp;
        fb = pack_cell(c[0], c[1], c[2]);
      }
    } else {
      const Vec3<R> l2 = rotate_vector_inverse(r2.rot, pw - r2.pos) - co2;
      su = axk == 0 ? l2.y : l2.x;
      sv = axk == 2 ? l2.y : l2.z;
      const Vec3<R> q = vabs(l2) - half2;
      if (q.x > sup.x || q.y > sup.y || q.z > sup.z) continue;
      const Vec3<R> qs = q - sup;
      const R best_q = std::max(qs.x, std::max(qs.y, qs.z));
      const R q_pass = sgn * vget(l2, axk) - vget(half2, axk) - sup_a;
      if (q_pass < best_q - R(0.15) * vs1) continue;
      n_out = rotate_vector(r2.rot, unit_axis(axk, R(1)) * sgn);
      pe = q_pass;
      fb = axk;
    }
    if (pe >= R(0.02)) continue;  // margin band
    pe = std::max(pe, s2_vox ? R(-0.5) * vs1 : -vs1);  // depth caps (:1262-1266)
    red.add(pw, pe, n_out, e & 0xFFFFFFu, fb, su, sv, R(0.5) * vs1);
  }
}

// voxel_obb_prefilter (collision_detection.slang:1276-1298): face-axis separation test of the
// two bodies' boxes with a 1 cm margin.
template <class R> bool voxel_prefilter(const Body<R>& a, const Body<R>& b, const VoxelPool& vp) {
  Vec3<R> la, ua, lb, ub;
  body_box(a, vp, la, ua);
  body_box(b, vp, lb, ub);
  const Vec3<R> ha = (ua - la) * R(0.5), hb = (ub - lb) * R(0.5);
  const Vec3<R> ca = a.pos + rotate_vector(a.rot, (ua + la) * R(0.5));
  const Vec3<R> cb = b.pos + rotate_vector(b.rot, (ub + lb) * R(0.5));
  const Vec3<R> d = cb - ca;
  Vec3<R> ax[3], bx[3];
  for (uint32_t k = 0; k < 3; ++k) {
    ax[k] = rotate_vector(a.rot, unit_axis(k, R(1)));
    bx[k] = rotate_vector(b.rot, unit_axis(k, R(1)));
  }
  const R haa[3] = {ha.x, ha.y, ha.z}, hbb[3] = {hb.x, hb.y, hb.z};
  for (int i = 0; i < 3; ++i) {
    const R rb = hbb[0] * std::fabs(dot(ax[i], bx[0])) + hbb[1] * std::fabs(dot(ax[i], bx[1])) +
                 hbb[2] * std::fabs(dot(ax[i], bx[2]));
    if (std::fabs(dot(d, ax[i])) > haa[i] + rb + R(0.01)) return false;
    const R ra = haa[0] * std::fabs(dot(bx[i], ax[0])) + haa[1] * std::fabs(dot(bx[i], ax[1])) +
                 haa[2] * std::fabs(dot(bx[i], ax[2]));
    if (std::fabs(dot(d, bx[i])) > hbb[i] + ra + R(0.01)) return false;
  }
  return true;
}

// voxel_corner_supported (collision_detection.slang:1305-1324): a face-corner contact point is
// kept only where r2 has material behind it (a cell just inside along the axis, or the face
// rectangle of r2's box).
template <class R>
bool voxel_corner_supported(Vec3<R> p, Vec3<R> n_sep, const Body<R>& r2, const VoxelShape* s2, bool s2_vox,
                            const VoxelPool& vp, uint32_t axk) {
  if (s2_vox) {
    const R vs2 = s2->vs;
    const Vec3<R> l2 = rotate_vector_inverse(r2.rot, (p - n_sep * (R(0.3) * vs2)) - r2.pos);
    const Vec3<R> g = (l2 - Vec3<R>(s2->origin[0], s2->origin[1], s2->origin[2])) / vs2;
    return vp.bit(*s2, int(std::floor(g.x)), int(std::floor(g.y)), int(std::floor(g.z)));
  }
  Vec3<R> lo2, hi2;
  body_box(r2, vp, lo2, hi2);
  const Vec3<R> half = (hi2 - lo2) * R(0.5), co = (hi2 + lo2) * R(0.5);
  const Vec3<R> l2 = rotate_vector_inverse(r2.rot, p - r2.pos) - co;
  const R lu = axk == 0 ? l2.y : l2.x, lv = axk == 2 ? l2.y : l2.z;
  const R hu = axk == 0 ? half.y : half.x, hv = axk == 2 ? half.y : half.z;
  return std::fabs(lu) <= hu + R(0.01) && std::fabs(lv) <= hv + R(0.01);
}

// voxel_emit_manifold (collision_detection.slang:1330-1448): at most four support points.  The
// surviving winners (in the band, aligned with the pass normal, distinct voxels) give their
// centres when three or four survive, two face corners each when two survive, the four face
// corners when one survives; corners without support behind them retreat halfway, then onto
// the centre, and a point that lands on an earlier one is dropped.  Depths are projected onto
// the manifold normal.  Feature ids: the sampled voxel (bits 0-23) and the corner (24-25).
template <class R>
bool voxel_emit(const VoxelReducer<R>& red, bool flip, Vec3<R> n_sep, R vs, const Body<R>& r2, const VoxelShape* s2,
                bool s2_vox, const VoxelPool& vp, uint32_t axk, SatResult<R>& out) {
  out.cc = 0;
  if (red.samples == 0) return false;
  out.normal = flip ? n_sep : -n_sep;
  uint32_t kept[4];
  R align_k[4];
  uint32_t kn = 0;
  for (uint32_t o = 0; o < 4; ++o) {
    if (red.pen[o] >= R(0.02)) continue;  // band contacts emit; empty slots (1e9) drop
    const R align = dot(red.nrm[o], n_sep);
    if (align <= R(0.1)) continue;
    bool dup = false;
    for (uint32_t q = 0; q < kn; ++q)
      if (red.fa[kept[q]] == red.fa[o]) dup = true;
    if (dup) continue;
    kept[kn] = o;
    align_k[kn] = align;
    ++kn;
  }
  const uint32_t reps = kn == 1 ? 4u : (kn == 2 ? 2u : 1u);
  const Vec3<R> t1 = normalize(cross(n_sep, std::fabs(n_sep.y) < R(0.9) ? Vec3<R>(0, 1, 0) : Vec3<R>(1, 0, 0)));
  const Vec3<R> t2 = cross(n_sep, t1);
  const Vec3<R> da = (t1 + t2) * (R(0.318) * vs), db = (t1 - t2) * (R(0.318) * vs);
  int n_out = 0;
  for (uint32_t k = 0; k < kn; ++k) {
    const uint32_t o = kept[k];
    const uint32_t vpar = (red.fa[o] ^ (red.fa[o] >> 8) ^ (red.fa[o] >> 16)) & 1u;
    Vec3<R> emitted[4];
    uint32_t en = 0;
    for (uint32_t c = 0; c < reps; ++c) {
      Vec3<R> p = red.pos[o];
      if (reps > 1) {
        const Vec3<R> offv = ((c < 2u) == (vpar == 0u)) ? da : db;
        const Vec3<R> off = offv * ((c & 1u) == 0u ? R(1) : R(-1));
        p = red.pos[o] + off;
        if (!voxel_corner_supported(p, n_sep, r2, s2, s2_vox, vp, axk)) {
          p = red.pos[o] + off * R(0.5);
          if (!voxel_corner_supported(p, n_sep, r2, s2, s2_vox, vp, axk)) p = red.pos[o];
        }
      }
      bool dup = false;
      for (uint32_t q = 0; q < en; ++q) {
        const Vec3<R> dp = p - emitted[q];
        if (dot(dp, dp) < R(1.0e-12)) dup = true;
      }
      if (dup) continue;
      emitted[en++] = p;
      out.pos[n_out] = p;
      out.pen[n_out] = red.pen[o] * align_k[k];
      out.fp[n_out].in_ref = flip ? 1u : 0u;
      out.fp[n_out].out_ref = red.fb[o];
      out.fp[n_out].in_inc = red.fa[o] | (c << 24);
      out.fp[n_out].out_inc = red.fa[o] | (c << 24);
      ++n_out;
    }
  }
  out.cc = n_out;
  return n_out > 0;
}

// voxel_axis_collision_detection (collision_detection.slang:1462-1512): the manifold of pass
// `code` between pair bodies A and B (sorted order).  The body with the smaller surface list is
// sampled (a non-voxel body never is); the normal is the exact world axis of the other body's
// face, pointing A -> B.  A pass with no sample but interior hits (code 0 only) emits one
// centre-to-centre contact so deeply interpenetrated bodies separate.
template <class R> bool voxel_collide(const Body<R>& A, const Body<R>& B, uint32_t code, const VoxelPool& vp, SatResult<R>& out) {
  out.cc = 0;
  out.key = VOXEL_KEY0 + int(code);
  if (!voxel_prefilter(A, B, vp)) return false;
  const bool a_vox = A.shape == BB_SHAPE_VOXEL, b_vox = B.shape == BB_SHAPE_VOXEL;
  const VoxelShape* sA = a_vox ? &vp.shapes[A.voxel] : nullptr;
  const VoxelShape* sB = b_vox ? &vp.shapes[B.voxel] : nullptr;
  const bool flip = !a_vox || (b_vox && sB->surf_count < sA->surf_count);  // sampled body = B
  const Body<R>& r1 = flip ? B : A;
  const Body<R>& r2 = flip ? A : B;
  const VoxelShape& s1 = flip ? *sB : *sA;
  const VoxelShape* s2 = flip ? sA : sB;
  const bool s2_vox = flip ? a_vox : b_vox;
  VoxelReducer<R> red;
  voxel_sample(r1, s1, r2, s2, s2_vox, vp, red, code);
  if (red.samples == 0) {
    if (code == 0 && red.interior > 0) {
      const Vec3<R> d = r1.pos - r2.pos;
      const Vec3<R> n_res = dot(d, d) > R(1e-8) ? normalize(d) : Vec3<R>(0, 1, 0);
      out.normal = flip ? n_res : -n_res;
      out.pos[0] = (r1.pos + r2.pos) * R(0.5);
      out.pen[0] = R(-0.5) * R(s1.vs);
      out.fp[0].in_ref = out.fp[0].out_ref = out.fp[0].in_inc = out.fp[0].out_inc = 0xFFFFFFu;
      out.cc = 1;
      return true;
    }
    return false;
  }
  const uint32_t ax = code / 2u;
  const R sgn = (code & 1u) ? R(1) : R(-1);
  const Vec3<R> n_world = rotate_vector(r2.rot, unit_axis(ax, sgn));
  return voxel_emit(red, flip, n_world, R(s1.vs), r2, s2, s2_vox, vp, ax, out);
}

}  // namespace bbo
