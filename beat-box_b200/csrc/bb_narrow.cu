// bb_narrow.cu -- narrow phase with persistent-contact warm start, manifold compaction and
// per-body manifold lists.
//
// Reference: narrow_phase (src/shaders/simulation/collision_detection.slang:1514-1755),
// OBBvsOBBCollision (:5-877: SAT :562-740, incident face :123-243, reference edges :245-336,
// clipping :352-449, edge contact :456-548), find_old_collision (:914-963),
// Manifold::compute_basis / update_from_old (src/shaders/extensions.slang:262-473),
// body_link_manifold (collision_detection.slang:881-905).
//
// B200 design: one thread per broad-phase pair writes its manifold into the pair's own slot
// (no atomic append), a scan over the hit flags gives the compact manifold order (= pair
// order), and each dynamic body gets a CSR list of its manifolds in ascending order built by
// count / scan / fill / per-body sort.  Warm-start lookup walks the previous substep's CSR
// list of the pair's dynamic body, which finds the same (unique) old manifold as the
// reference's linked-list walk.
#include "bb_common.cuh"
#include "bb_kernels.cuh"

namespace {

enum : uint32_t {
  POS_X_POS_Y = 0, POS_X_NEG_Y = 1, POS_X_POS_Z = 2, POS_X_NEG_Z = 3, NEG_X_POS_Y = 4, NEG_X_NEG_Y = 5,
  NEG_X_POS_Z = 6, NEG_X_NEG_Z = 7, POS_Y_POS_Z = 8, POS_Y_NEG_Z = 9, NEG_Y_POS_Z = 10, NEG_Y_NEG_Z = 11
};

// feature pair packed in one word: in_ref | out_ref << 8 | in_inc << 16 | out_inc << 24
__device__ __forceinline__ uint32_t fp_pack(uint32_t ir, uint32_t orf, uint32_t ii, uint32_t oi) {
  return (ir & 255u) | ((orf & 255u) << 8) | ((ii & 255u) << 16) | ((oi & 255u) << 24);
}
__device__ __forceinline__ uint32_t fp_in_ref(uint32_t f) { return f & 255u; }
__device__ __forceinline__ uint32_t fp_out_ref(uint32_t f) { return (f >> 8) & 255u; }
__device__ __forceinline__ uint32_t fp_in_inc(uint32_t f) { return (f >> 16) & 255u; }
__device__ __forceinline__ uint32_t fp_out_inc(uint32_t f) { return (f >> 24) & 255u; }
__device__ __forceinline__ uint32_t fp_set_in_ref(uint32_t f, uint32_t v) { return (f & ~255u) | (v & 255u); }
__device__ __forceinline__ uint32_t fp_set_out_ref(uint32_t f, uint32_t v) { return (f & ~(255u << 8)) | ((v & 255u) << 8); }
__device__ __forceinline__ uint32_t fp_swap_roles(uint32_t f) {
  return fp_pack(fp_in_inc(f), fp_out_inc(f), fp_in_ref(f), fp_out_ref(f));
}

// Slang-semantics transform: rows of r are the body axes; vectors multiply from the left.
struct Xf {
  float r[3][3];
  float3 p;
};
__device__ __forceinline__ float3 xf_rotate(const Xf& t, float3 v) {
  return make_float3(v.x * t.r[0][0] + v.y * t.r[1][0] + v.z * t.r[2][0], v.x * t.r[0][1] + v.y * t.r[1][1] + v.z * t.r[2][1],
                     v.x * t.r[0][2] + v.y * t.r[1][2] + v.z * t.r[2][2]);
}
__device__ __forceinline__ float3 xf_rotate_t(const Xf& t, float3 v) {
  return make_float3(t.r[0][0] * v.x + t.r[0][1] * v.y + t.r[0][2] * v.z, t.r[1][0] * v.x + t.r[1][1] * v.y + t.r[1][2] * v.z,
                     t.r[2][0] * v.x + t.r[2][1] * v.y + t.r[2][2] * v.z);
}
__device__ __forceinline__ float3 xf_transform(const Xf& t, float3 v) { return xf_rotate(t, v) + t.p; }
__device__ __forceinline__ float3 xf_transform_t(const Xf& t, float3 v) { return xf_rotate_t(t, v - t.p); }
__device__ __forceinline__ float3 row3(const float m[3][3], int i) { return make_float3(m[i][0], m[i][1], m[i][2]); }
__device__ __forceinline__ float3 col3(const float m[3][3], int j) { return make_float3(m[0][j], m[1][j], m[2][j]); }

__device__ __forceinline__ void body_axes(Quatf q, float r[3][3]) {
  float R[3][3];
  q_matrix(q, R);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r[i][j] = R[j][i];
}

struct CV {
  float3 v;
  uint32_t f;
};

// A manifold under construction.  Contact i lives at p[i * ST] (position, depth) and f[i * ST]
// (feature word): k_narrow points p and f at the thread's column of shared-memory buffers
// (ST = the block size), so the contact and clip arrays, which are indexed by run-time counts,
// stay on chip instead of in local memory; the voxel kernel's lanes use local arrays (ST = 1).
template <int ST>
struct ContactsT {
  int cc;
  int key;
  float3 normal;
  float4* p;
  uint32_t* f;
  __device__ __forceinline__ float3 pos(int i) const { return f3(p[i * ST]); }
  __device__ __forceinline__ float pen(int i) const { return p[i * ST].w; }
  __device__ __forceinline__ uint32_t fp(int i) const { return f[i * ST]; }
  __device__ __forceinline__ void set(int i, float3 v, float depth, uint32_t feature) {
    p[i * ST] = f4(v, depth);
    f[i * ST] = feature;
  }
  __device__ __forceinline__ void set_pos(int i, float3 v) { p[i * ST] = f4(v, p[i * ST].w); }
  __device__ __forceinline__ void set_pen(int i, float depth) { p[i * ST].w = depth; }
};
// clip vertex i of a column buffer: position and feature word
template <int ST>
__device__ __forceinline__ CV cv_get(const float4* b, int i) {
  const float4 x = b[i * ST];
  return CV{make_float3(x.x, x.y, x.z), __float_as_uint(x.w)};
}
template <int ST>
__device__ __forceinline__ void cv_put(float4* b, int i, const CV& c) {
  b[i * ST] = make_float4(c.v.x, c.v.y, c.v.z, __uint_as_float(c.f));
}

// compute_incident_face (collision_detection.slang:123-243)
__device__ void incident_face(const Xf& itx, float3 e, float3 n, CV out[4]) {
  n = -xf_rotate_t(itx, n);
  float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
  float3 v[4];
  uint32_t fi[4][2];
  auto set = [&](uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1, uint32_t c0, uint32_t c1, uint32_t d0, uint32_t d1) {
    fi[0][0] = a0; fi[0][1] = a1; fi[1][0] = b0; fi[1][1] = b1; fi[2][0] = c0; fi[2][1] = c1; fi[3][0] = d0; fi[3][1] = d1;
  };
  if (ax > ay && ax > az) {
    if (n.x > 0.f) {
      v[0] = make_float3(e.x, e.y, -e.z); v[1] = make_float3(e.x, e.y, e.z); v[2] = make_float3(e.x, -e.y, e.z); v[3] = make_float3(e.x, -e.y, -e.z);
      set(POS_Y_NEG_Z, POS_X_NEG_Y, POS_X_NEG_Y, POS_Y_POS_Z, POS_Y_POS_Z, NEG_X_NEG_Z, NEG_X_NEG_Z, POS_Y_NEG_Z);
    } else {
      v[0] = make_float3(-e.x, -e.y, e.z); v[1] = make_float3(-e.x, e.y, e.z); v[2] = make_float3(-e.x, e.y, -e.z); v[3] = make_float3(-e.x, -e.y, -e.z);
      set(NEG_X_NEG_Y, NEG_Y_NEG_Z, NEG_Y_NEG_Z, POS_X_NEG_Z, POS_X_NEG_Z, NEG_Y_POS_Z, NEG_Y_POS_Z, NEG_X_NEG_Y);
    }
  } else if (ay > ax && ay > az) {
    if (n.y > 0.f) {
      v[0] = make_float3(-e.x, e.y, e.z); v[1] = make_float3(e.x, e.y, e.z); v[2] = make_float3(e.x, e.y, -e.z); v[3] = make_float3(-e.x, e.y, -e.z);
      set(POS_X_NEG_Z, POS_X_POS_Y, POS_X_POS_Y, POS_X_NEG_Y, POS_X_NEG_Y, POS_X_POS_Z, POS_X_POS_Z, POS_X_NEG_Z);
    } else {
      v[0] = make_float3(e.x, -e.y, e.z); v[1] = make_float3(-e.x, -e.y, e.z); v[2] = make_float3(-e.x, -e.y, -e.z); v[3] = make_float3(e.x, -e.y, -e.z);
      set(NEG_X_NEG_Z, NEG_X_POS_Y, NEG_X_POS_Y, NEG_X_NEG_Y, NEG_X_NEG_Y, NEG_X_POS_Z, NEG_X_POS_Z, NEG_X_NEG_Z);
    }
  } else {
    if (n.z > 0.f) {
      v[0] = make_float3(-e.x, e.y, e.z); v[1] = make_float3(-e.x, -e.y, e.z); v[2] = make_float3(e.x, -e.y, e.z); v[3] = make_float3(e.x, e.y, e.z);
      set(POS_X_POS_Y, NEG_Y_NEG_Z, NEG_Y_NEG_Z, NEG_X_POS_Y, NEG_X_POS_Y, POS_Y_POS_Z, POS_Y_POS_Z, POS_X_POS_Y);
    } else {
      v[0] = make_float3(e.x, -e.y, -e.z); v[1] = make_float3(-e.x, -e.y, -e.z); v[2] = make_float3(-e.x, e.y, -e.z); v[3] = make_float3(e.x, e.y, -e.z);
      set(POS_Y_NEG_Z, NEG_X_POS_Z, NEG_X_POS_Z, NEG_Y_POS_Z, NEG_Y_POS_Z, POS_X_POS_Z, POS_X_POS_Z, POS_Y_NEG_Z);
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    out[i].v = xf_transform(itx, v[i]);
    out[i].f = fp_pack(0u, 0u, fi[i][0], fi[i][1]);
  }
}

// compute_reference_edges_and_basis (collision_detection.slang:245-336)
__device__ void reference_edges(float3 er, const Xf& rtx, float3 n, int axis, uint32_t clip[4], Xf& basis, float3& e) {
  n = xf_rotate_t(rtx, n);
  if (axis > 2) axis -= 3;
  float3 r0 = row3(rtx.r, 0), r1 = row3(rtx.r, 1), r2 = row3(rtx.r, 2);
  float3 b0, b1, b2;
  if (axis == 0) {
    if (n.x > 0.f) { clip[0] = POS_X_NEG_Y; clip[1] = POS_Y_POS_Z; clip[2] = NEG_X_NEG_Z; clip[3] = POS_Y_NEG_Z; e = make_float3(er.y, er.z, er.x); b0 = r1; b1 = r2; b2 = r0; }
    else { clip[0] = NEG_Y_NEG_Z; clip[1] = POS_X_NEG_Z; clip[2] = NEG_Y_POS_Z; clip[3] = NEG_X_NEG_Y; e = make_float3(er.z, er.y, er.x); b0 = r2; b1 = r1; b2 = -r0; }
  } else if (axis == 1) {
    if (n.y > 0.f) { clip[0] = POS_X_POS_Y; clip[1] = POS_X_NEG_Y; clip[2] = POS_X_POS_Z; clip[3] = POS_X_NEG_Z; e = make_float3(er.z, er.x, er.y); b0 = r2; b1 = r0; b2 = r1; }
    else { clip[0] = NEG_X_POS_Y; clip[1] = NEG_X_NEG_Y; clip[2] = NEG_X_POS_Z; clip[3] = NEG_X_NEG_Z; e = make_float3(er.z, er.x, er.y); b0 = r2; b1 = -r0; b2 = -r1; }
  } else {
    if (n.z > 0.f) { clip[0] = NEG_Y_NEG_Z; clip[1] = NEG_X_POS_Y; clip[2] = POS_Y_POS_Z; clip[3] = POS_X_POS_Y; e = make_float3(er.y, er.x, er.z); b0 = -r1; b1 = r0; b2 = r2; }
    else { clip[0] = NEG_X_POS_Z; clip[1] = NEG_Y_POS_Z; clip[2] = POS_X_POS_Z; clip[3] = POS_Y_NEG_Z; e = make_float3(er.y, er.x, er.z); b0 = -r1; b1 = -r0; b2 = -r2; }
  }
  basis.r[0][0] = b0.x; basis.r[0][1] = b0.y; basis.r[0][2] = b0.z;
  basis.r[1][0] = b1.x; basis.r[1][1] = b1.y; basis.r[1][2] = b1.z;
  basis.r[2][0] = b2.x; basis.r[2][1] = b2.y; basis.r[2][2] = b2.z;
  basis.p = rtx.p;
}

// ortographic_clip (collision_detection.slang:352-387); output capped at 8.  in and out are
// column buffers (vertex i at [i * ST]).
template <int ST>
__device__ int ortho_clip(float sign, float e, int axis, uint32_t clip_edge, const float4* in, int in_count, float4* out) {
  const float TH = 0.005f;
  int oc = 0;
  CV a = cv_get<ST>(in, in_count - 1);
  for (int i = 0; i < in_count; ++i) {
    CV b = cv_get<ST>(in, i);
    float da = sign * comp(a.v, axis) - e;
    float db = sign * comp(b.v, axis) - e;
    bool on_a = da < TH && da > -TH, on_b = db < TH && db > -TH;
    if ((da < 0.f && db < 0.f) || on_a || on_b) {
      if (oc < BB_MAX_CONTACTS) cv_put<ST>(out, oc++, b);
    } else if (da < 0.f && db >= 0.f) {
      CV cv;
      cv.f = fp_set_out_ref(b.f, clip_edge);
      cv.v = a.v + (b.v - a.v) * (da / (da - db));
      if (oc < BB_MAX_CONTACTS) cv_put<ST>(out, oc++, cv);
    } else if (da >= 0.f && db < 0.f) {
      CV cv;
      cv.f = fp_set_in_ref(a.f, clip_edge);
      cv.v = a.v + (b.v - a.v) * (da / (da - db));
      if (oc < BB_MAX_CONTACTS) cv_put<ST>(out, oc++, cv);
      if (oc < BB_MAX_CONTACTS) cv_put<ST>(out, oc++, b);
    }
    a = b;
  }
  return oc;
}

__device__ __forceinline__ float c_sign(float x) { return x < 0.f ? -1.f : 1.f; }

// support_edge (collision_detection.slang:456-497)
__device__ void support_edge(const Xf& tx, float3 e, float3 n, float3& ca, float3& cb) {
  n = xf_rotate_t(tx, n);
  float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
  int axis = (ax <= ay && ax <= az) ? 0 : ((ay <= ax && ay <= az) ? 1 : 2);
  float3 v0 = make_float3(c_sign(n.x) * e.x, c_sign(n.y) * e.y, c_sign(n.z) * e.z), v1 = v0;
  set_comp(v0, axis, comp(e, axis));
  set_comp(v1, axis, -comp(e, axis));
  ca = xf_transform(tx, v0);
  cb = xf_transform(tx, v1);
}

// edges_contact (collision_detection.slang:499-548)
__device__ void edges_contact(float3 pa, float3 qa, float3 pb, float3 qb, float3& ca, float3& cb) {
  float3 da = qa - pa, db = qb - pb, r = pa - pb;
  float a = dot3(da, da), e = dot3(db, db), f = dot3(db, r), c = dot3(da, r), b = dot3(da, db);
  float denom = a * e - b * b;
  if (denom == 0.f) {
    float t = fminf(fmaxf(dot3(r, da) / a, 0.f), 1.f);
    ca = pa + da * t;
    float u = fminf(fmaxf(dot3(ca - pb, db) / e, 0.f), 1.f);
    cb = pb + db * u;
    return;
  }
  float ta = fminf(fmaxf((b * f - c * e) / denom, 0.f), 1.f);
  float tb = (b * ta + f) / e;
  if (tb < 0.f) {
    tb = 0.f;
    ta = fminf(fmaxf(-c / a, 0.f), 1.f);
  } else if (tb > 1.f) {
    tb = 1.f;
    ta = fminf(fmaxf((b - c) / a, 0.f), 1.f);
  }
  ca = pa + da * ta;
  cb = pb + db * tb;
}

// OBBvsOBBCollision::collision_detection (collision_detection.slang:562-876).  The clip runs
// between the column buffer buf and the output's own buffer out.p: four passes end in buf, and
// the contacts are then written to out.p.
template <int ST>
__device__ bool box_box(Quatf qa, float3 pa, float3 ea, Quatf qb, float3 pb, float3 eb, bool sat_quirk, float4* buf,
                        ContactsT<ST>& out) {
  out.cc = 0;
  out.key = -1;
  Xf txa, txb;
  body_axes(qa, txa.r);
  txa.p = pa;
  body_axes(qb, txb.r);
  txb.p = pb;
  float C[3][3], aC[3][3];
  bool parallel = false;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      float v;
      if (sat_quirk) v = txa.r[0][i] * txb.r[0][j] + txa.r[1][i] * txb.r[1][j] + txa.r[2][i] * txb.r[2][j];
      else v = txb.r[i][0] * txa.r[j][0] + txb.r[i][1] * txa.r[j][1] + txb.r[i][2] * txa.r[j][2];
      C[i][j] = v;
      aC[i][j] = fabsf(v);
      if (aC[i][j] > 0.9998f) parallel = true;
    }
  float3 t = q_rotate_inv(qa, pb - pa);
  float a_max = -3.402823466e+38f, b_max = -3.402823466e+38f, e_max = -3.402823466e+38f;
  int a_axis = -1, b_axis = -1, e_axis = -1;
  float3 n_a = make_float3(0, 0, 0), n_b = n_a, n_e = n_a;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float s = fabsf(comp(t, i)) - (comp(ea, i) + dot3(col3(aC, i), eb));
    if (s > 0.f) return false;
    if (s > a_max) { a_max = s; a_axis = i; n_a = row3(txa.r, i); }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float proj = dot3(t, row3(C, i));
    float s = fabsf(proj) - (comp(eb, i) + dot3(row3(aC, i), ea));
    if (s > 0.f) return false;
    if (s > b_max) { b_max = s; b_axis = 3 + i; n_b = row3(txb.r, i); }
  }
  if (!parallel) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        float rA = comp(ea, i1) * aC[j][i2] + comp(ea, i2) * aC[j][i1];
        float rB = comp(eb, j1) * aC[j2][i] + comp(eb, j2) * aC[j1][i];
        float s = fabsf(comp(t, i2) * C[j][i1] - comp(t, i1) * C[j][i2]) - (rA + rB);
        float3 axis = make_float3(0, 0, 0);
        set_comp(axis, i1, -C[j][i2]);
        set_comp(axis, i2, C[j][i1]);
        if (s > 0.f) return false;
        float l = 1.0f / len3(axis);
        s *= l;
        if (s > e_max) { e_max = s; e_axis = 6 + i * 3 + j; n_e = axis * l; }
      }
    }
  }
  int axis;
  float s_max;
  float3 normal;
  float face_max = fmaxf(a_max, b_max);
  if (0.95f * e_max > face_max + 0.01f) { axis = e_axis; s_max = e_max; normal = n_e; }
  else if (0.95f * b_max > a_max + 0.01f) { axis = b_axis; s_max = b_max; normal = n_b; }
  else { axis = a_axis; s_max = a_max; normal = n_a; }
  if (dot3(normal, pb - pa) < 0.f) normal = -normal;
  if (axis == -1) return false;
  if (axis <= 5) {
    const Xf& rtx = axis <= 2 ? txa : txb;
    const Xf& itx = axis <= 2 ? txb : txa;
    float3 er = axis <= 2 ? ea : eb, ei = axis <= 2 ? eb : ea;
    bool flip = axis > 2;
    if (flip) normal = -normal;
    CV inc[4];
    incident_face(itx, ei, normal, inc);
    uint32_t clip[4];
    Xf basis;
    float3 e;
    reference_edges(er, rtx, normal, axis, clip, basis, e);
    float4* in = buf;
    float4* outv = out.p;
#pragma unroll
    for (int i = 0; i < 4; ++i) cv_put<ST>(in, i, CV{xf_transform_t(basis, inc[i].v), inc[i].f});
    int oc = ortho_clip<ST>(1.f, e.x, 0, clip[0], in, 4, outv);
    if (oc == 0) return false;
    int ic = ortho_clip<ST>(1.f, e.y, 1, clip[1], outv, oc, in);
    if (ic == 0) return false;
    oc = ortho_clip<ST>(-1.f, e.x, 0, clip[2], in, ic, outv);
    if (oc == 0) return false;
    ic = ortho_clip<ST>(-1.f, e.y, 1, clip[3], outv, oc, in);
    if (ic == 0) return false;
    int n = 0;
    for (int i = 0; i < ic; ++i) {
      const CV v = cv_get<ST>(in, i);
      float dd = v.v.z - e.z;
      if (dd <= 0.f) {
        out.set(n, xf_transform(basis, v.v), dd, flip ? fp_swap_roles(v.f) : v.f);
        ++n;
      }
    }
    if (n > 0) {
      out.cc = n;
      out.normal = flip ? -normal : normal;
    }
  } else {
    normal = xf_rotate(txa, normal);
    if (dot3(normal, pb - pa) < 0.f) normal = -normal;
    float3 p0, q0, p1, q1, ca, cb;
    support_edge(txa, ea, normal, p0, q0);
    support_edge(txb, eb, -normal, p1, q1);
    edges_contact(p0, q0, p1, q1, ca, cb);
    out.cc = 1;
    out.normal = normal;
    out.set(0, (ca + cb) * 0.5f, s_max, fp_pack(axis, axis, axis, axis));
  }
  out.key = axis;
  return out.cc > 0;
}

// Sphere contacts (first principles; the reference has no sphere collider).
template <int ST>
__device__ bool sphere_sphere(float3 pa, float ra, float3 pb, float rb, ContactsT<ST>& out) {
  float3 d = pb - pa;
  float dist = len3(d);
  if (dist > ra + rb) return false;
  float3 n = dist > 1e-9f ? d * (1.0f / dist) : make_float3(0, 1, 0);
  float pen = dist - (ra + rb);
  out.cc = 1;
  out.key = BB_KEY_SPHERE_SPHERE;
  out.normal = n;
  out.set(0, pa + n * (ra + pen * 0.5f), pen,
          fp_pack(BB_KEY_SPHERE_SPHERE, BB_KEY_SPHERE_SPHERE, BB_KEY_SPHERE_SPHERE, BB_KEY_SPHERE_SPHERE));
  return true;
}
__device__ bool box_sphere_core(Quatf qx, float3 px, float3 e, float3 ps, float r, float3& n, float& pen, float3& pos) {
  float3 c = q_rotate_inv(qx, ps - px);
  float3 q = make_float3(fminf(fmaxf(c.x, -e.x), e.x), fminf(fmaxf(c.y, -e.y), e.y), fminf(fmaxf(c.z, -e.z), e.z));
  bool inside = fabsf(c.x) < e.x && fabsf(c.y) < e.y && fabsf(c.z) < e.z;
  if (!inside) {
    float3 dl = c - q;
    float dist = len3(dl);
    if (dist > r) return false;
    float3 nl = dist > 1e-9f ? dl * (1.0f / dist) : make_float3(0, 1, 0);
    n = q_rotate(qx, nl);
    pen = dist - r;
    pos = ((px + q_rotate(qx, q)) + (ps - n * r)) * 0.5f;
    return true;
  }
  int ax = 0;
  float best = e.x - fabsf(c.x);
  if (e.y - fabsf(c.y) < best) { best = e.y - fabsf(c.y); ax = 1; }
  if (e.z - fabsf(c.z) < best) { best = e.z - fabsf(c.z); ax = 2; }
  float3 nl = make_float3(0, 0, 0);
  float sg = comp(c, ax) < 0.f ? -1.f : 1.f;
  set_comp(nl, ax, sg);
  n = q_rotate(qx, nl);
  pen = -best - r;
  float3 face = c;
  set_comp(face, ax, sg * comp(e, ax));
  pos = ((px + q_rotate(qx, face)) + (ps - n * r)) * 0.5f;
  return true;
}

__device__ __forceinline__ uint32_t warm_inc(uint32_t w) { return min(255u, w + 1u); }

}  // namespace

// Manifold slots.  Without voxel shapes a pair owns one slot (slot = pair).  In a world with
// voxel shapes every pair with a voxel body owns six consecutive slots, one per face direction
// (code 0..5, key 90 + code), the others one: a scan over the pairs places them, so slot order
// = (pair, code), which is the manifold order.
__device__ __forceinline__ uint32_t slot_total(const DevState& d) {
  return d.vox_on ? min(d.ctr->slot_count, d.pair_capacity) : min(d.ctr->pair_count, d.pair_capacity);
}
__device__ __forceinline__ uint32_t slot_pair_of(const DevState& d, uint32_t s) { return d.vox_on ? d.slot_pair[s] >> 3 : s; }
__device__ __forceinline__ bool pair_has_voxel(const DevState& d, uint32_t k) {
  const uint2 pr = d.pairs[k];
  const uint32_t ta = __float_as_uint(d.shape[d.vals[0][pr.x]].w), tb = __float_as_uint(d.shape[d.vals[0][pr.y]].w);
  return BB_SHAPE_KIND(ta) == BB_SHAPE_VOXEL || BB_SHAPE_KIND(tb) == BB_SHAPE_VOXEL;
}
__global__ void k_slot_count(const DevState d) {
  const uint32_t P = min(d.ctr->pair_count, d.pair_capacity);
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < P; k += gridDim.x * blockDim.x)
    d.slot_cnt[k] = pair_has_voxel(d, k) ? 6u : 1u;
}
__global__ void k_slot_fill(const DevState d) {
  const uint32_t P = min(d.ctr->pair_count, d.pair_capacity);
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < P; k += gridDim.x * blockDim.x) {
    const uint32_t off = d.slot_off[k], c = d.slot_cnt[k];
    for (uint32_t j = 0; j < c; ++j) {
      if (off + j < d.pair_capacity) d.slot_pair[off + j] = (k << 3) | j;
      else raise_error(d.ctr, BB_ERRF_PAIR_OVERFLOW);
    }
  }
}

__device__ __forceinline__ bool np_awake(uint32_t f) { return (f & BB_BODY_DYNAMIC) && !(f & BB_BODY_SLEEPING); }

// Work lists of the narrow phase: box-box slots from the front of np_list, slots with a sphere
// from the back, voxel pairs (their code-0 slot) in vox_list, frozen pairs (their first slot)
// in carry_list, static-static pairs (:1525) nowhere.  A pair is frozen when neither body is
// awake and both were asleep or static at the last narrow phase too, so both poses are those
// of the previous substep bit for bit.  Every slot starts as "no manifold".  Grouping by shape
// keeps the warps of k_narrow on one code path (the box-box clip is long, the sphere cases
// short); the outputs go to each slot's own place, so the order in which the lists fill does
// not matter.
#define BB_CLS_WARPS 8  // k_np_classify runs 256-thread blocks
__global__ void __launch_bounds__(32 * BB_CLS_WARPS) k_np_classify(const DevState d, int cur, int warm) {
  __shared__ uint32_t s_cnt[4][BB_CLS_WARPS];  // per kind, per warp: entries, then the warp's first index
  const uint32_t S = slot_total(d);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (blockIdx.x == 0 && threadIdx.x == 0) d.ctr->slots_of[cur] = S;  // read by the next substep's carry
  for (uint32_t base = blockIdx.x * blockDim.x; base < S; base += gridDim.x * blockDim.x) {  // block-uniform
    const uint32_t k = base + threadIdx.x;
    int kind = -1;  // 0 box-box, 1 with a sphere, 2 with a voxel body, 3 frozen
    uint2 ids = make_uint2(0u, 0u);
    bool paused = false, dyn_a = false;
    if (k < S) {
      d.hit[k] = 0;
      d.m_keycc[cur][k] = make_int2(-1, 0);
      const uint2 pr = d.pairs[slot_pair_of(d, k)];
      const uint32_t ida = d.vals[0][pr.x], idb = d.vals[0][pr.y];
      const uint32_t fa = d.flags[ida], fb = d.flags[idb];
      ids = make_uint2(ida, idb);
      paused = ((fa | fb) & BB_BODY_PAUSED) != 0u;
      dyn_a = (fa & BB_BODY_DYNAMIC) != 0u;
      if ((fa & BB_BODY_DYNAMIC) || (fb & BB_BODY_DYNAMIC)) {
        const uint32_t ta = BB_SHAPE_KIND(__float_as_uint(d.shape[ida].w)), tb = BB_SHAPE_KIND(__float_as_uint(d.shape[idb].w));
        const bool vox = ta == BB_SHAPE_VOXEL || tb == BB_SHAPE_VOXEL;
        const bool first = !vox || (d.slot_pair[k] & 7u) == 0u;  // a voxel pair is listed once
        // a paused world's pairs are always carried (exactly: see k_narrow_carry)
        if ((fa | fb) & BB_BODY_PAUSED) kind = first ? 3 : -1;
        else if (warm && !np_awake(fa) && !np_awake(fb) && d.frozen[ida] && d.frozen[idb]) kind = first ? 3 : -1;
        else if (vox) kind = first ? 2 : -1;
        else kind = (ta == BB_SHAPE_BOX && tb == BB_SHAPE_BOX) ? 0 : 1;
      }
    }
    // one list append per kind and block: warp counts, a block scan by four threads, one atomic each
    unsigned my_mask = 0;
#pragma unroll
    for (int kd = 0; kd < 4; ++kd) {
      const unsigned mask = __ballot_sync(0xFFFFFFFFu, kind == kd);
      if (kind == kd) my_mask = mask;
      if (lane == 0) s_cnt[kd][warp] = uint32_t(__popc(mask));
    }
    __syncthreads();
    if (threadIdx.x < 4) {
      const int kd = threadIdx.x;
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < BB_CLS_WARPS; ++w) {
        const uint32_t c = s_cnt[kd][w];
        s_cnt[kd][w] = run;
        run += c;
      }
      const uint32_t first = run ? atomicAdd(&d.ctr->np_counts[kd], run) : 0u;
#pragma unroll
      for (int w = 0; w < BB_CLS_WARPS; ++w) s_cnt[kd][w] += first;
    }
    __syncthreads();
    if (kind >= 0) {
      const uint32_t r = s_cnt[kind][warp] + uint32_t(__popc(my_mask & ((1u << lane) - 1u)));
      if (kind == 3) {  // slot | paused << 31 | body a dynamic << 30, and the two bodies
        d.carry_list[r] = k | (paused ? 0x80000000u : 0u) | (dyn_a ? 0x40000000u : 0u);
        d.carry_ids[r] = ids;
      } else if (kind == 2) d.vox_list[r] = k;
      else d.np_list[kind == 0 ? r : S - 1 - r] = k;
    }
    __syncthreads();  // s_cnt is rewritten by the next trip
  }
}

// Carry-over of a frozen pair: its manifold(s) of the previous substep in the same body order
// (voxel pairs: each face key into its own slot) are kept as they were -- contacts, features,
// impulses, penalties, stick anchors -- with warm-start counts + 1 and the extraction trend 0,
// which is what recomputing the same poses and matching every contact by feature gives.  A
// frozen pair without a manifold last substep goes to the ordinary lists and is computed.
// Old contact oi (its position, impulses, penalties and first anchor already loaded) written as
// new contact ni.  A paused world's manifold (exact) is carried as it is, every field
// (warm-start counts, trend, anchors, stick data), so the world resumes exactly where it stopped.
__device__ __forceinline__ void carry_loaded(const DevState& d, int prv, int cur, uint32_t oi, uint32_t ni, float4 cp,
                                             float4 cl, float4 kt, float4 aa, bool exact) {
  d.c_pos[cur][ni] = cp;
  d.c_lam[cur][ni] = cl;
  if (exact) {
    d.c_kt[cur][ni] = kt;
    d.c_anc_a[cur][ni] = aa;
    d.c_anc_b[cur][ni] = d.c_anc_b[prv][oi];
    return;
  }
  const bool stick = __float_as_uint(kt.z) != 0u;
  // the second anchor only of a sticking contact (else it is written as 0)
  const float4 ab = stick ? d.c_anc_b[prv][oi] : make_float4(0.f, 0.f, 0.f, 0.f);
  kt.w = __uint_as_float(min(255u, __float_as_uint(kt.w) + 1u));
  d.c_kt[cur][ni] = kt;
  d.c_anc_a[cur][ni] = stick ? aa : make_float4(0.f, 0.f, 0.f, aa.w);
  d.c_anc_b[cur][ni] = make_float4(ab.x, ab.y, ab.z, 0.f);
}
__device__ __forceinline__ void carry_contact(const DevState& d, int prv, int cur, uint32_t oi, uint32_t ni, bool exact) {
  carry_loaded(d, prv, cur, oi, ni, d.c_pos[prv][oi], d.c_lam[prv][oi], d.c_kt[prv][oi], d.c_anc_a[prv][oi], exact);
}

// Lane q (0..3) of the quad that carries a pair: the header (q = 0) and contacts q, q + 4.  The
// quad's four lanes read each contact array over 64 contiguous bytes.
__device__ __forceinline__ void carry_part(const DevState& d, int cur, uint32_t os, uint32_t dst, uint32_t ida,
                                           uint32_t idb, uint32_t q, bool exact) {
  const int prv = cur ^ 1;
  const int2 kc = d.m_keycc[prv][os];
  if (q == 0) {  // the same manifold as last substep: its colour carries over (colour reuse)
    const uint32_t sub_tag = d.ctr->substeps;
    const bool reuse_ok = d.ctr->gc_coloured + 1u == sub_tag;
    d.gc_reuse[dst] = reuse_ok ? d.gc_slot_color[prv][os] : BB_NONE;
    if (reuse_ok) d.gc_survived[os] = sub_tag;
  }
  if (exact) {
    if (q == 0) {
      d.m_bodies[cur][dst] = d.m_bodies[prv][os];
      d.m_keycc[cur][dst] = kc;
      d.m_normal[cur][dst] = d.m_normal[prv][os];
      d.m_t0[cur][dst] = d.m_t0[prv][os];
      d.m_t1[cur][dst] = d.m_t1[prv][os];
      d.m_anchor_a[cur][dst] = d.m_anchor_a[prv][os];
      d.m_anchor_b[cur][dst] = d.m_anchor_b[prv][os];
      d.hit[dst] = 1;
    }
    for (uint32_t c = q; c < uint32_t(kc.y); c += 4u)
      carry_contact(d, prv, cur, os * BB_MAX_CONTACTS + c, dst * BB_MAX_CONTACTS + c, true);
    return;
  }
  if (q == 0) {
    const float4 n4 = d.m_normal[prv][os], t04 = d.m_t0[prv][os], t14 = d.m_t1[prv][os];
    const float4 pa = d.pos[ida], pb = d.pos[idb];
    d.m_bodies[cur][dst] = make_uint2(ida, idb);
    d.m_keycc[cur][dst] = kc;
    d.m_normal[cur][dst] = make_float4(n4.x, n4.y, n4.z, __int_as_float(0));
    d.m_t0[cur][dst] = t04;
    d.m_t1[cur][dst] = t14;
    d.m_anchor_a[cur][dst] = make_float4(pa.x, pa.y, pa.z, 0.f);
    d.m_anchor_b[cur][dst] = make_float4(pb.x, pb.y, pb.z, 0.f);
    d.hit[dst] = 1;
  }
  for (uint32_t c = q; c < uint32_t(kc.y); c += 4u)
    carry_contact(d, prv, cur, os * BB_MAX_CONTACTS + c, dst * BB_MAX_CONTACTS + c, false);
}

// One quad of lanes per frozen pair.  The pair's manifold of the previous substep is found at
// the pair's own slot when the slot held a manifold of the same two bodies in the same order
// then: that is the pair's only non-voxel manifold (key < 90; a voxel pair's keys are 90..95),
// the one the search through the body's manifold list would find.  While no pair ahead of it
// came or went, every frozen pair takes this path; the others search.  Slots past the previous
// substep's count are not read (they hold older manifolds).
//
// The list entry carries the two bodies, the paused bit and whether body a is dynamic, so the
// probe of the pair's own slot and the bounds of the dynamic body's old list load in one round,
// with no chain through the pair, the sorted ids and the flags.  A pair whose slot moved searches
// that list with the quad's lanes splitting it (each entry carries its slot, csr_slot).  Then
// every load of the old manifold is issued at once: the quad's lanes split the header (lane 0
// the key, bodies and colour, 1 the normal and first tangent, 2 the second tangent and first
// anchor, 3 the second anchor) and lane q takes contact q.
//
// Short carry.  When this slot was carried the same way last substep (carry_tag = last
// substep), last substep's manifold was made from the one this substep writes over, and nothing
// has written either since: the frozen pair is not solved, and host calls that change contacts
// either reset both buffers' headers (refill), restore every array (state load, regrow) or
// unfreeze the bodies.  Its contacts then differ from last substep's only in the warm-start
// count, so only that word is rewritten (the header is written in full).  Not under AVBD
// (lazy_ok = 0), whose warm start decays the penalties and re-anchors every manifold, sleeping
// ones included; not for a paused world's exact carry.
__global__ void __launch_bounds__(256) k_narrow_carry(const DevState d, int cur, int lazy_ok) {
  const int prv = cur ^ 1;
  const uint32_t S = slot_total(d);
  const uint32_t S_prv = min(d.ctr->slots_of[prv], d.pair_capacity);
  const uint32_t nc = d.ctr->np_counts[3];
  const uint32_t sub_tag = d.ctr->substeps;
  const bool reuse_ok = d.ctr->gc_coloured + 1u == sub_tag;
  const bool lazy_on = lazy_ok != 0 && sub_tag > 1u;  // tags start at 0: substep 1 never matches
  const uint32_t q = threadIdx.x & 3u, quads = (gridDim.x * blockDim.x) >> 2;
  const uint32_t qbase = threadIdx.x & 28u;  // this quad's first lane
  const unsigned qmask = 0xFu << qbase;
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 2; t < nc; t += quads) {  // quad-uniform
    const uint32_t entry = d.carry_list[t];
    const uint2 ids = d.carry_ids[t];
    const uint32_t s = entry & 0x3FFFFFFFu, ida = ids.x, idb = ids.y;
    // A paused world's manifold is kept in the body order it was stored in: the first paused
    // substep sorts with the poses its world's last step integrated, which can swap a pair.
    const bool exact = (entry >> 31) != 0u;
    const uint32_t x = (entry & 0x40000000u) ? ida : idb, other = x == ida ? idb : ida;
    // one round of loads: the old manifold at the pair's own slot, and the bounds of the dynamic
    // body's list of old manifolds
    int2 okc = make_int2(-1, 0);
    uint2 ob = make_uint2(BB_NONE, BB_NONE);
    if (s < S_prv) {
      okc = d.m_keycc[prv][s];
      ob = d.m_bodies[prv][s];
    }
    const uint32_t l0 = d.csr_start[prv][x], l1 = d.csr_start[prv][x + 1];
    const bool in_place = okc.x >= 0 && okc.x < 90 &&
                          ((ob.x == ida && ob.y == idb) || (exact && ob.x == idb && ob.y == ida));
    uint32_t os = s;
    uint32_t ta = BB_SHAPE_BOX, tb = BB_SHAPE_BOX;
    if (!in_place) {
      ta = BB_SHAPE_KIND(__float_as_uint(d.shape[ida].w));
      tb = BB_SHAPE_KIND(__float_as_uint(d.shape[idb].w));
      const bool vox = ta == BB_SHAPE_VOXEL || tb == BB_SHAPE_VOXEL;
      os = BB_NONE;
      if (vox) {  // each face key into its own slot, in list order
        bool any = false;
        for (uint32_t e = l0; e < l1; ++e) {
          if (d.csr_partner[prv][e] != other) continue;
          const uint32_t vs = d.csr_slot[prv][e];
          if (!exact && d.m_bodies[prv][vs].x != ida) continue;  // same body order only
          const int key = d.m_keycc[prv][vs].x;
          if (key < 90 || key > 95) continue;
          carry_part(d, cur, vs, s + uint32_t(key - 90), ida, idb, q, exact);
          any = true;
        }
        // no manifold last substep: compute the pair with the others (a paused pair had none
        // when its world stopped, and keeps none)
        if (!any && q == 0 && !exact) d.vox_list[atomicAdd(&d.ctr->np_counts[2], 1u)] = s;
        continue;
      }
      // Not a voxel pair: one slot, so at most one old manifold, the entry of x's list whose
      // partner is the other body.  The quad's lanes split the list.
      uint32_t mine = BB_NONE;
      for (uint32_t e = l0 + q; e < l1; e += 4u) {
        const uint32_t pe = d.csr_partner[prv][e], se = d.csr_slot[prv][e];
        if (pe == other) mine = se;
      }
      const unsigned found = __ballot_sync(qmask, mine != BB_NONE) & qmask;
      if (found) os = __shfl_sync(qmask, mine, __ffs(found) - 1);
    }
    // the old manifold os, every load at once: the header split over the quad (lane 0 the key,
    // bodies and colour, 1 the normal and first tangent, 2 the second tangent and first anchor,
    // 3 the second anchor), contact q on lane q
    int2 kc = okc;
    uint2 ob2 = ob;
    float4 h0 = make_float4(0.f, 0.f, 0.f, 0.f), h1 = h0, kt = h0;
    uint32_t colour = BB_NONE, tag = 0u;
    if (os != BB_NONE) {
      if (!in_place) {
        kc = d.m_keycc[prv][os];
        ob2 = d.m_bodies[prv][os];
      }
      if (q == 0) {
        if (reuse_ok) colour = d.gc_slot_color[prv][os];
        if (lazy_on && in_place) tag = d.carry_tag[s];
      } else if (q == 1) {
        h0 = d.m_normal[prv][os];
        h1 = d.m_t0[prv][os];
      } else if (q == 2) {
        h0 = d.m_t1[prv][os];
        h1 = exact ? d.m_anchor_a[prv][os] : d.pos[ida];
      } else {
        h1 = exact ? d.m_anchor_b[prv][os] : d.pos[idb];
      }
      kt = d.c_kt[prv][os * BB_MAX_CONTACTS + q];
    }
    if (os == BB_NONE || (!exact && ob2.x != ida)) {  // same body order only
      // no manifold last substep: compute the pair with the others (a paused pair had none
      // when its world stopped, and keeps none)
      if (q != 0 || exact) continue;
      if (ta == BB_SHAPE_BOX && tb == BB_SHAPE_BOX) d.np_list[atomicAdd(&d.ctr->np_counts[0], 1u)] = s;
      else d.np_list[S - 1 - atomicAdd(&d.ctr->np_counts[1], 1u)] = s;
      continue;
    }
    const bool lazy = in_place && lazy_on && !exact && __shfl_sync(qmask, tag, qbase) == sub_tag - 1u;
    // the same writes as carry_part(d, cur, os, s, ida, idb, q, exact)
    if (q == 0) {  // the same manifold as last substep: its colour carries over (colour reuse)
      d.gc_reuse[s] = colour;
      if (reuse_ok) d.gc_survived[os] = sub_tag;
      d.m_bodies[cur][s] = exact ? ob2 : make_uint2(ida, idb);
      d.m_keycc[cur][s] = kc;
      d.hit[s] = 1;
      if (in_place && lazy_on && !exact) d.carry_tag[s] = sub_tag;
    } else if (q == 1) {
      d.m_normal[cur][s] = exact ? h0 : make_float4(h0.x, h0.y, h0.z, __int_as_float(0));
      d.m_t0[cur][s] = h1;
    } else if (q == 2) {
      d.m_t1[cur][s] = h0;
      d.m_anchor_a[cur][s] = exact ? h1 : make_float4(h1.x, h1.y, h1.z, 0.f);
    } else {
      d.m_anchor_b[cur][s] = exact ? h1 : make_float4(h1.x, h1.y, h1.z, 0.f);
    }
    if (lazy) {  // in place, carried in place last substep too: warm-start counts only
      for (uint32_t c = q; c < uint32_t(kc.y); c += 4u) {
        const uint32_t ci = s * BB_MAX_CONTACTS + c;
        float4 k4 = c == q ? kt : d.c_kt[prv][ci];
        k4.w = __uint_as_float(min(255u, __float_as_uint(k4.w) + 1u));
        d.c_kt[cur][ci] = k4;
      }
    } else {
      const uint32_t oi = os * BB_MAX_CONTACTS + q;
      if (q < uint32_t(kc.y))
        carry_loaded(d, prv, cur, oi, s * BB_MAX_CONTACTS + q, d.c_pos[prv][oi], d.c_lam[prv][oi], kt,
                     d.c_anc_a[prv][oi], exact);
      for (uint32_t c = q + 4u; c < uint32_t(kc.y); c += 4u)
        carry_contact(d, prv, cur, os * BB_MAX_CONTACTS + c, s * BB_MAX_CONTACTS + c, exact);
    }
  }
}

// Basis, warm start from the previous substep (Manifold::update_from_old,
// extensions.slang:306-473, after find_old_collision, collision_detection.slang:914-963) and
// the write of slot k.  Voxel manifolds (vox) inherit only from the old manifold of the same
// key in the same body order, match features by the whole voxel/corner id, and keep their
// own depth caps; other manifolds take the pair's old manifold under any key, either order.
// old_p / old_f are column buffers (stride ST) that receive the old manifold's contacts
// (position and depth, feature word) once, for the matching loops below.
template <int ST>
__device__ __forceinline__ void np_store(const DevState& d, const Params& p, int cur, int warm, uint32_t k,
                                         uint32_t ida, uint32_t idb, uint32_t fa, float3 pa, float3 pb,
                                         ContactsT<ST>& m, bool vox, float4* old_p, uint32_t* old_f) {
  const int prv = cur ^ 1;
  // compute_basis (extensions.slang:262-272)
  float3 n = m.normal, t0;
  if (fabsf(n.x) > fabsf(n.y)) t0 = make_float3(n.z, 0.f, -n.x);
  else t0 = make_float3(0.f, -n.z, n.y);
  t0 = t0 * (1.0f / len3(t0));
  float3 t1 = cross3(t0, n);
  const int cc = m.cc;
  if (!vox)
    for (int c = 0; c < cc; ++c) m.set_pen(c, fmaxf(m.pen(c), p.penetration_cap));  // extraction cap (:1575-1578)
  // Each new contact records the old contact it inherits from (src, -1: none) and whether the
  // proximity pass gave it (pass2: then the old features, the tangent sign and anchor roles of
  // a swapped pair apply); the inherited fields are read from the old contact when written.
  uint32_t src_lo = 0xFFFFFFFFu, src_hi = 0xFFFFFFFFu;  // 8 x 8-bit old index, 0xFF = none
  auto set_src = [&](int i, int j) {
    if (i < 4) src_lo = (src_lo & ~(0xFFu << (8 * i))) | (uint32_t(j) << (8 * i));
    else src_hi = (src_hi & ~(0xFFu << (8 * (i - 4)))) | (uint32_t(j) << (8 * (i - 4)));
  };
  auto get_src = [&](int i) -> int {
    const uint32_t v = i < 4 ? (src_lo >> (8 * i)) & 0xFFu : (src_hi >> (8 * (i - 4))) & 0xFFu;
    return v == 0xFFu ? -1 : int(v);
  };
  uint32_t pass2 = 0;
  uint32_t ob = 0;
  bool swapped = false;
  float sgn = 1.f;
  int32_t err = 0x7FFFFFFF;
  // Colour reuse: the same manifold (bodies and key) as last substep carries its colour, and
  // the old manifold is marked as taken over (an old manifold nobody takes over has ended).
  uint32_t reuse = BB_NONE;
  const uint32_t sub_tag = d.ctr->substeps;
  const bool reuse_ok = d.ctr->gc_coloured + 1u == sub_tag;
  if (warm) {
    // find the pair's manifold of the previous substep on the dynamic body's list
    uint32_t x = (fa & BB_BODY_DYNAMIC) ? ida : idb;
    const uint32_t other = x == ida ? idb : ida;
    uint32_t s0 = d.csr_start[prv][x], s1 = d.csr_start[prv][x + 1];
    uint32_t old_slot = BB_NONE;
    for (uint32_t e = s0; e < s1; ++e) {
      if (d.csr_partner[prv][e] != other) continue;
      const uint32_t os = d.csr_slot[prv][e];
      if (vox && (d.m_keycc[prv][os].x != m.key || d.m_bodies[prv][os].x != ida)) continue;
      old_slot = os;
      swapped = d.m_bodies[prv][os].x != ida;
      break;
    }
    if (old_slot != BB_NONE) {
      // Manifold::update_from_old (extensions.slang:306-473)
      int2 okc = d.m_keycc[prv][old_slot];
      if (reuse_ok && !vox && okc.x == m.key) {
        reuse = d.gc_slot_color[prv][old_slot];
        d.gc_survived[old_slot] = sub_tag;
      }
      float4 on4 = d.m_normal[prv][old_slot];
      sgn = swapped ? -1.f : 1.f;
      bool cross_key = m.key != okc.x || swapped;
      bool go = !cross_key || dot3(n, f3(on4) * sgn) > 0.7f;
      if (go) {
        const int occ = okc.y;
        uint32_t used_old = 0, matched_new = 0;
        ob = old_slot * BB_MAX_CONTACTS;
        for (int j = 0; j < occ; ++j) {
          old_p[j * ST] = d.c_pos[prv][ob + j];
          if (!cross_key) old_f[j * ST] = __float_as_uint(d.c_anc_a[prv][ob + j].w);
        }
        if (!cross_key) {
          for (int i = 0; i < cc; ++i) {
            for (int j = 0; j < occ; ++j) {
              if (used_old & (1u << j)) continue;
              float4 op = old_p[j * ST];
              uint32_t ofp = old_f[j * ST];
              const uint32_t nfp = m.fp(i);
              bool feat = vox ? ofp == nfp : (fp_in_inc(ofp) == fp_in_inc(nfp) && fp_out_inc(ofp) == fp_out_inc(nfp));
              float3 dp = f3(op) - m.pos(i);
              bool close = dot3(dp, dp) < 0.1f * 0.1f;
              if (feat && close) {
                set_src(i, j);
                float3 d2 = m.pos(i) - f3(op);
                if (dot3(d2, d2) < 0.01f) m.set_pos(i, f3(op));
                used_old |= 1u << j;
                matched_new |= 1u << i;
                break;
              }
            }
          }
        }
        for (int round = 0; round < cc; ++round) {
          float best = 0.1225f;
          int bi = -1, bj = -1;
          for (int i = 0; i < cc; ++i) {
            if (matched_new & (1u << i)) continue;
            for (int j = 0; j < occ; ++j) {
              if (used_old & (1u << j)) continue;
              float3 dp = m.pos(i) - f3(old_p[j * ST]);
              float d2 = dot3(dp, dp);
              if (d2 < best) { best = d2; bi = i; bj = j; }
            }
          }
          if (bi < 0) break;
          set_src(bi, bj);
          pass2 |= 1u << bi;
          matched_new |= 1u << bi;
          used_old |= 1u << bj;
        }
        float deep_new = 0.f, deep_old = 0.f;
        for (int i = 0; i < cc; ++i) deep_new = fminf(deep_new, m.pen(i));
        for (int j = 0; j < occ; ++j) deep_old = fminf(deep_old, old_p[j * ST].w);
        err = int32_t(fminf(fmaxf((deep_new - deep_old) * 10000.0f, -32000.0f), 32000.0f));
      }
    }
  }
  d.m_bodies[cur][k] = make_uint2(ida, idb);
  d.m_keycc[cur][k] = make_int2(m.key, cc);
  d.m_normal[cur][k] = f4(n, __int_as_float(err));
  d.m_t0[cur][k] = f4(t0, 0.f);
  d.m_t1[cur][k] = f4(t1, 0.f);
  d.m_anchor_a[cur][k] = make_float4(pa.x, pa.y, pa.z, 0.f);
  d.m_anchor_b[cur][k] = make_float4(pb.x, pb.y, pb.z, 0.f);
  const uint32_t cb = k * BB_MAX_CONTACTS;
  for (int c = 0; c < cc; ++c) {
    // new contacts start at zero; matched ones inherit impulses, penalties, stick and anchors
    float4 lam = make_float4(0.f, 0.f, 0.f, 0.f);
    float2 kt = make_float2(0.f, 0.f);
    uint32_t stick = 0, wc = 0, fp = m.fp(c);
    float3 aa = make_float3(0.f, 0.f, 0.f), ab = make_float3(0.f, 0.f, 0.f);
    const int j = get_src(c);
    if (j >= 0) {
      const uint32_t oi = ob + uint32_t(j);
      const bool p2 = (pass2 >> c) & 1u;
      const float4 ol = d.c_lam[prv][oi], okt = d.c_kt[prv][oi], oaa = d.c_anc_a[prv][oi];
      lam = p2 ? make_float4(ol.x, ol.y * sgn, ol.z, ol.w) : ol;
      kt = make_float2(okt.x, okt.y);
      stick = __float_as_uint(okt.z);
      if (stick != 0) {
        const float3 a0 = f3(oaa), b0 = f3(d.c_anc_b[prv][oi]);
        aa = (p2 && swapped) ? b0 : a0;
        ab = (p2 && swapped) ? a0 : b0;
      }
      if (p2) fp = __float_as_uint(oaa.w);
      wc = warm_inc(__float_as_uint(okt.w));
    }
    d.c_pos[cur][cb + c] = f4(m.pos(c), m.pen(c));
    d.c_lam[cur][cb + c] = lam;
    d.c_kt[cur][cb + c] = make_float4(kt.x, kt.y, __uint_as_float(stick), __uint_as_float(wc));
    d.c_anc_a[cur][cb + c] = f4(aa, __uint_as_float(fp));
    d.c_anc_b[cur][cb + c] = f4(ab, 0.f);
  }
  d.hit[k] = 1;
  d.gc_reuse[k] = reuse;
}

// Narrow phase + warm start: one thread per listed pair.  Each thread owns a column of three
// shared-memory buffers of eight entries: the clip polygon ping-pongs between columns 0 and 1,
// the contacts end in column 1 with their feature words beside them, and column 0 then takes
// the old manifold's contacts for the warm-start match (36 KB per 128-thread block).
#define BB_NARROW_THREADS 128
__global__ void __launch_bounds__(BB_NARROW_THREADS) k_narrow(const DevState d, Params p, int cur, int warm) {
  __shared__ float4 s_col[2][BB_MAX_CONTACTS][BB_NARROW_THREADS];
  __shared__ uint32_t s_feat[2][BB_MAX_CONTACTS][BB_NARROW_THREADS];
  constexpr int ST = BB_NARROW_THREADS;
  float4* const buf = &s_col[0][0][threadIdx.x];
  const uint32_t S = slot_total(d);
  const uint32_t nbb = d.ctr->np_counts[0], ntot = nbb + d.ctr->np_counts[1];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntot; t += gridDim.x * blockDim.x) {
    const uint32_t k = d.np_list[t < nbb ? t : S - 1 - (t - nbb)];
    uint2 pr = d.pairs[slot_pair_of(d, k)];
    uint32_t ida = d.vals[0][pr.x], idb = d.vals[0][pr.y];
    const uint32_t fa = d.flags[ida];
    float4 pa4 = d.pos[ida], pb4 = d.pos[idb];
    float4 sa = d.shape[ida], sb = d.shape[idb];
    Quatf qa = q_from(d.rot[ida]), qb = q_from(d.rot[idb]);
    float3 pa = f3(pa4), pb = f3(pb4);
    uint32_t ta = __float_as_uint(sa.w), tb = __float_as_uint(sb.w);
    ContactsT<ST> m;
    m.p = &s_col[1][0][threadIdx.x];
    m.f = &s_feat[1][0][threadIdx.x];
    bool hit;
    if (ta == BB_SHAPE_BOX && tb == BB_SHAPE_BOX) {
      hit = box_box<ST>(qa, pa, f3(sa), qb, pb, f3(sb), (p.quirks & BB_QUIRK_SAT_FRAME) != 0, buf, m);
    } else if (ta == BB_SHAPE_SPHERE && tb == BB_SHAPE_SPHERE) {
      hit = sphere_sphere<ST>(pa, sa.x, pb, sb.x, m);
    } else {
      float3 n, pos;
      float pen;
      if (ta == BB_SHAPE_BOX) {
        hit = box_sphere_core(qa, pa, f3(sa), pb, sb.x, n, pen, pos);
        m.key = BB_KEY_BOX_SPHERE;
      } else {
        hit = box_sphere_core(qb, pb, f3(sb), pa, sa.x, n, pen, pos);
        n = -n;
        m.key = BB_KEY_SPHERE_BOX;
      }
      if (hit) {
        m.cc = 1;
        m.normal = n;
        m.set(0, pos, pen, fp_pack(m.key, m.key, m.key, m.key));
      }
    }
    if (!hit) continue;
    np_store<ST>(d, p, cur, warm, k, ida, idb, fa, pa, pb, m, false, buf, &s_feat[0][0][threadIdx.x]);
  }
}

// ---- voxel bodies (collision_detection.slang:1001-1512) -----------------------------------------
// One warp per voxel slot (pair, face code).  The lanes split the sampled body's surface cells;
// each lane keeps the four extreme-direction winners of its own samples, and a warp reduction
// picks the winners under the reducer's ranking (score bucket, then depth bucket, then voxel
// id: a strict total order, since voxel ids are unique in a surface list), so the manifold does
// not depend on how the samples were split.  Lane 0 then builds the contacts and stores the
// slot as k_narrow does.
struct VBody {
  float3 p;
  float R[3][3];  // rotation: world = R * local
  uint32_t kind, vi;
  float3 lo, hi;  // body-frame box [minimum, maximum]
};
__device__ __forceinline__ void vbody(const DevState& d, uint32_t id, VBody& b) {
  b.p = f3(d.pos[id]);
  q_matrix(q_from(d.rot[id]), b.R);
  const float4 s = d.shape[id];
  const uint32_t t = __float_as_uint(s.w);
  b.kind = BB_SHAPE_KIND(t);
  b.vi = BB_SHAPE_VOXEL_INDEX(t);
  if (b.kind == BB_SHAPE_VOXEL) {
    const VoxDev& v = d.vox[b.vi];
    b.lo = make_float3(v.ox, v.oy, v.oz);
    b.hi = make_float3(v.hx, v.hy, v.hz);
  } else if (b.kind == BB_SHAPE_SPHERE) {  // read as its bounding cube, as the reference reads any non-voxel body
    b.lo = make_float3(-s.x, -s.x, -s.x);
    b.hi = make_float3(s.x, s.x, s.x);
  } else {
    b.lo = make_float3(-s.x, -s.y, -s.z);
    b.hi = make_float3(s.x, s.y, s.z);
  }
}
__device__ __forceinline__ float3 mat_mul(const float R[3][3], float3 v) {
  return make_float3(R[0][0] * v.x + R[0][1] * v.y + R[0][2] * v.z, R[1][0] * v.x + R[1][1] * v.y + R[1][2] * v.z,
                     R[2][0] * v.x + R[2][1] * v.y + R[2][2] * v.z);
}
__device__ __forceinline__ float3 mat_tmul(const float R[3][3], float3 v) {  // R^T v
  return make_float3(R[0][0] * v.x + R[1][0] * v.y + R[2][0] * v.z, R[0][1] * v.x + R[1][1] * v.y + R[2][1] * v.z,
                     R[0][2] * v.x + R[1][2] * v.y + R[2][2] * v.z);
}
__device__ __forceinline__ float3 mat_col(const float R[3][3], int k) { return make_float3(R[0][k], R[1][k], R[2][k]); }
__device__ __forceinline__ float3 axis_vec(uint32_t k, float s) {
  return make_float3(k == 0 ? s : 0.f, k == 1 ? s : 0.f, k == 2 ? s : 0.f);
}
__device__ __forceinline__ bool vox_bit(const DevState& d, const VoxDev& v, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= int(v.dx) || y >= int(v.dy) || z >= int(v.dz)) return false;
  const uint32_t b = uint32_t(x) + uint32_t(y) * v.dx + uint32_t(z) * v.dx * v.dy;
  return ((__ldg(&d.vox_occ[v.occ_off + b / 32u]) >> (b % 32u)) & 1u) != 0u;
}
__device__ __forceinline__ uint32_t pack_cell(int x, int y, int z) {
  return uint32_t(x & 0xFF) | (uint32_t(y & 0xFF) << 8) | (uint32_t(z & 0xFF) << 16);
}

// voxel_obb_prefilter (:1276-1298): face-axis separation of the two boxes, 1 cm margin
__device__ bool vox_prefilter(const VBody& a, const VBody& b) {
  const float3 ha = (a.hi - a.lo) * 0.5f, hb = (b.hi - b.lo) * 0.5f;
  const float3 ca = a.p + mat_mul(a.R, (a.hi + a.lo) * 0.5f), cb = b.p + mat_mul(b.R, (b.hi + b.lo) * 0.5f);
  const float3 dd = cb - ca;
  const float haa[3] = {ha.x, ha.y, ha.z}, hbb[3] = {hb.x, hb.y, hb.z};
  for (int i = 0; i < 3; ++i) {
    const float3 ai = mat_col(a.R, i), bi = mat_col(b.R, i);
    const float rb = hbb[0] * fabsf(dot3(ai, mat_col(b.R, 0))) + hbb[1] * fabsf(dot3(ai, mat_col(b.R, 1))) +
                     hbb[2] * fabsf(dot3(ai, mat_col(b.R, 2)));
    if (fabsf(dot3(dd, ai)) > haa[i] + rb + 0.01f) return false;
    const float ra = haa[0] * fabsf(dot3(bi, mat_col(a.R, 0))) + haa[1] * fabsf(dot3(bi, mat_col(a.R, 1))) +
                     haa[2] * fabsf(dot3(bi, mat_col(a.R, 2)));
    if (fabsf(dot3(dd, bi)) > hbb[i] + ra + 0.01f) return false;
  }
  return true;
}

// voxel_corner_supported (:1305-1324)
__device__ bool vox_corner_supported(const DevState& d, float3 pt, float3 n_sep, const VBody& r2, bool s2_vox, uint32_t axk) {
  if (s2_vox) {
    const VoxDev& v = d.vox[r2.vi];
    const float3 l2 = mat_tmul(r2.R, (pt - n_sep * (0.3f * v.vs)) - r2.p);
    const float3 g = make_float3((l2.x - v.ox) / v.vs, (l2.y - v.oy) / v.vs, (l2.z - v.oz) / v.vs);
    return vox_bit(d, v, int(floorf(g.x)), int(floorf(g.y)), int(floorf(g.z)));
  }
  const float3 half = (r2.hi - r2.lo) * 0.5f, co = (r2.hi + r2.lo) * 0.5f;
  const float3 l2 = mat_tmul(r2.R, pt - r2.p) - co;
  const float lu = axk == 0 ? l2.y : l2.x, lv = axk == 2 ? l2.y : l2.z;
  const float hu = axk == 0 ? half.y : half.x, hv = axk == 2 ? half.y : half.z;
  return fabsf(lu) <= hu + 0.01f && fabsf(lv) <= hv + 0.01f;
}

struct VWin {  // one reducer slot: the winning sample of one extreme direction
  float3 pos;
  float pen, score;
  uint32_t fa, fb;
};
// Rank of a reducer slot's sample as two 32-bit words for warp max-reductions: hi = (score
// bucket + 2^15) << 16 | (2^15 - 1 - depth bucket), lo = 2^24 - fa (lower voxel id wins).  Empty
// slots rank 0.  Buckets are clamped to 15 bits (|local coordinate| < 3276 half-voxels).
__device__ __forceinline__ uint32_t vrank_hi(const VWin& w, float quant) {
  if (w.pen > 0.5e9f) return 0u;
  const int sb = min(max(int(floorf(w.score / quant)), -32767), 32767);
  const int pb = min(max(int(floorf(w.pen / quant)), -32767), 32767);
  return (uint32_t(sb + 32768) << 16) | uint32_t(32767 - pb);
}
__device__ __forceinline__ uint32_t vrank_lo(const VWin& w) { return w.pen > 0.5e9f ? 0u : (1u << 24) - w.fa; }

// One sample's code-independent geometry (a surface cell centre of the sampled body).
struct VSample {
  float3 pw, l2;  // world position; position in r2's frame (minus r2's box centre when r2 is a box)
  int c[3];       // r2's cell (voxel r2)
  bool occ;       // that cell is solid (voxel r2)
  float best;     // shallowest exit over the near faces (voxel r2, occupied cell); 1e9: interior
  float3 dl;      // offset from the cell centre (voxel r2, occupied cell)
  float3 q;       // |l2| - half (box r2)
  uint32_t fa;    // sampled voxel id
};

__device__ __forceinline__ void vox_sample_geom(const DevState& d, const VBody& r1, const VoxDev& s1, const VBody& r2,
                                                bool s2_vox, const VoxDev& s2, float3 sup, float3 half2, float3 co2,
                                                uint32_t i, VSample& g) {
  const float vs1 = s1.vs;
  const uint32_t e = __ldg(&d.vox_surf[s1.surf_off + i]);
  g.fa = e & 0xFFFFFFu;
  const float3 local = make_float3(s1.ox + (float(e & 0xFFu) + 0.5f) * vs1, s1.oy + (float((e >> 8) & 0xFFu) + 0.5f) * vs1,
                                   s1.oz + (float((e >> 16) & 0xFFu) + 0.5f) * vs1);
  g.pw = r1.p + mat_mul(r1.R, local);
  const float3 l2w = mat_tmul(r2.R, g.pw - r2.p);
  if (s2_vox) {
    g.l2 = l2w;
    const float vs2 = s2.vs;
    const float3 gg = make_float3((l2w.x - s2.ox) / vs2, (l2w.y - s2.oy) / vs2, (l2w.z - s2.oz) / vs2);
    g.c[0] = int(floorf(gg.x));
    g.c[1] = int(floorf(gg.y));
    g.c[2] = int(floorf(gg.z));
    g.occ = vox_bit(d, s2, g.c[0], g.c[1], g.c[2]);
    g.best = 1e9f;
    g.dl = make_float3(0.f, 0.f, 0.f);
    if (g.occ) {
      // cell-face contact (:1185-1208): the shallowest feasible exit over the near faces
      const float3 org2 = make_float3(s2.ox, s2.oy, s2.oz);
      g.dl = l2w - (org2 + (make_float3(float(g.c[0]), float(g.c[1]), float(g.c[2])) + make_float3(0.5f, 0.5f, 0.5f)) * vs2);
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const float di = comp(g.dl, ax);
        int nb[3] = {g.c[0], g.c[1], g.c[2]};
        nb[ax] += di >= 0.f ? 1 : -1;
        if (vox_bit(d, s2, nb[0], nb[1], nb[2])) continue;
        const float ov = (0.5f * vs2 + comp(sup, ax)) - fabsf(di);
        if (ov < g.best) g.best = ov;
      }
    }
  } else {
    g.l2 = l2w - co2;
    g.q = make_float3(fabsf(g.l2.x) - half2.x, fabsf(g.l2.y) - half2.y, fabsf(g.l2.z) - half2.z);
  }
}

// The sample's membership in pass `code` (axis axk, sign sgn) and its depth (:1148-1266);
// returns false when it does not join.  `interior` is set for occupied cells with no exit.
__device__ __forceinline__ bool vox_sample_pass(const DevState& d, const VSample& g, bool s2_vox, const VoxDev& s2,
                                                float3 sup, float3 half2, float vs1, uint32_t axk, float sgn, int isgn,
                                                float& pe, uint32_t& fb, bool& interior) {
  interior = false;
  const float sup_a = comp(sup, int(axk));
  if (s2_vox) {
    const float vs2 = s2.vs;
    if (!g.occ) {
      // hover band: centre in an empty cell just outside an occupied one (:1155-1183)
      int ci[3] = {g.c[0], g.c[1], g.c[2]};
      ci[axk] -= isgn;
      if (!vox_bit(d, s2, ci[0], ci[1], ci[2])) return false;
      const float org_a = axk == 0 ? s2.ox : (axk == 1 ? s2.oy : s2.oz);
      const float dh = comp(g.l2, int(axk)) - (org_a + (float(ci[axk]) + 0.5f) * vs2);
      const float ovh = (0.5f * vs2 + sup_a) - sgn * dh;
      pe = -ovh;
      fb = pack_cell(ci[0], ci[1], ci[2]);
    } else {
      if (g.best > 0.5e9f) {
        interior = true;
        return false;
      }
      int pn[3] = {g.c[0], g.c[1], g.c[2]};
      pn[axk] += isgn;
      if (vox_bit(d, s2, pn[0], pn[1], pn[2])) return false;  // the pass axis is no exit here
      const float ovp = (0.5f * vs2 + sup_a) - sgn * comp(g.dl, int(axk));
      if (ovp > g.best + 0.15f * vs2) return false;  // dominated by a shallower exit
      pe = -ovp;
      fb = pack_cell(g.c[0], g.c[1], g.c[2]);
    }
  } else {
    // r2 is a box: sample centre with support radius against the box faces (:1235-1258)
    if (g.q.x > sup.x || g.q.y > sup.y || g.q.z > sup.z) return false;
    const float3 qs = g.q - sup;
    const float best_q = fmaxf(qs.x, fmaxf(qs.y, qs.z));
    const float q_pass = sgn * comp(g.l2, int(axk)) - comp(half2, int(axk)) - sup_a;
    if (q_pass < best_q - 0.15f * vs1) return false;
    pe = q_pass;
    fb = axk;
  }
  if (pe >= 0.02f) return false;  // margin band
  pe = fmaxf(pe, s2_vox ? -0.5f * vs1 : -vs1);  // depth caps (:1262-1266)
  return true;
}

// VoxelManifoldReducer::add (:1064-1092)
__device__ __forceinline__ void vox_reduce_add(VWin w[4], float3 pw, float pe, uint32_t fa, uint32_t fb, float su, float sv,
                                               float quant) {
  const float sc4[4] = {su + sv, su - sv, -su + sv, -su - sv};
  const int nbk = int(floorf(pe / quant));
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    const bool empty = w[o].pen > 0.5e9f;
    const int nbs = int(floorf(sc4[o] / quant));
    const int obs = empty ? -2147483640 : int(floorf(w[o].score / quant));
    const int obk = empty ? 0 : int(floorf(w[o].pen / quant));
    if (empty || nbs > obs || (nbs == obs && (nbk < obk || (nbk == obk && fa < w[o].fa)))) {
      w[o].pos = pw;
      w[o].pen = pe;
      w[o].fa = fa;
      w[o].fb = fb;
      w[o].score = sc4[o];
    }
  }
}

// One warp per voxel pair.  The prefilter and each sample's geometry are computed once; the six
// passes (face codes) then reuse them.  Per pass every lane ranks its own samples, a warp
// max-reduction of the packed ranks picks each extreme direction's winner, and lane `code`
// keeps the pass's winners.  Lanes 0..5 then build and store the six manifolds in parallel.
#define BB_VOX_CACHE 32  // samples whose geometry stays in registers (one per lane)
__global__ void __launch_bounds__(256) k_voxel_narrow(const DevState d, Params p, int cur, int warm) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t nv = d.ctr->np_counts[2];
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < nv; t += warps) {
    const uint32_t slot0 = d.vox_list[t];  // the pair's code-0 slot; codes 1..5 follow it
    const uint2 pr = d.pairs[d.slot_pair[slot0] >> 3];
    const uint32_t ida = d.vals[0][pr.x], idb = d.vals[0][pr.y];
    VBody A, B;
    vbody(d, ida, A);
    vbody(d, idb, B);
    if (!vox_prefilter(A, B)) continue;  // warp-uniform
    const bool a_vox = A.kind == BB_SHAPE_VOXEL, b_vox = B.kind == BB_SHAPE_VOXEL;
    const uint32_t sa_n = a_vox ? d.vox[A.vi].surf_count : 0u, sb_n = b_vox ? d.vox[B.vi].surf_count : 0u;
    const bool flip = !a_vox || (b_vox && sb_n < sa_n);  // sampled body = B
    const VBody& r1 = flip ? B : A;
    const VBody& r2 = flip ? A : B;
    const bool s2_vox = flip ? a_vox : b_vox;
    const VoxDev s1 = d.vox[r1.vi];
    VoxDev s2 = {};
    if (s2_vox) s2 = d.vox[r2.vi];
    const float vs1 = s1.vs, quant = 0.5f * vs1;
    // per-axis support radius of a rotated sample cell in r2's frame (:1110-1117)
    float A12[3][3];  // r2^T r1
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) A12[i][j] = r2.R[0][i] * r1.R[0][j] + r2.R[1][i] * r1.R[1][j] + r2.R[2][i] * r1.R[2][j];
    const float3 sup = make_float3(fabsf(A12[0][0]) + fabsf(A12[0][1]) + fabsf(A12[0][2]),
                                   fabsf(A12[1][0]) + fabsf(A12[1][1]) + fabsf(A12[1][2]),
                                   fabsf(A12[2][0]) + fabsf(A12[2][1]) + fabsf(A12[2][2])) * (0.5f * vs1);
    const float3 half2 = (r2.hi - r2.lo) * 0.5f, co2 = (r2.hi + r2.lo) * 0.5f;
    VSample cache;
    const bool cached = lane < s1.surf_count;
    if (cached) vox_sample_geom(d, r1, s1, r2, s2_vox, s2, sup, half2, co2, lane, cache);
    VWin mine[4];  // lane `code`: the winners of pass `code`
    uint32_t my_samples = 0, my_interior = 0;
#pragma unroll 1
    for (uint32_t code = 0; code < 6; ++code) {
      const uint32_t axk = code >> 1;
      const float sgn = (code & 1u) ? 1.f : -1.f;
      const int isgn = (code & 1u) ? 1 : -1;
      VWin w[4];
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        w[o].pen = 1.0e9f;
        w[o].score = -1.0e30f;
        w[o].fa = 0;
        w[o].fb = 0;
        w[o].pos = make_float3(0.f, 0.f, 0.f);
      }
      uint32_t samples = 0, interior = 0;
      for (uint32_t i = lane; i < s1.surf_count; i += 32u) {
        VSample g;
        if (i < BB_VOX_CACHE) g = cache;
        else vox_sample_geom(d, r1, s1, r2, s2_vox, s2, sup, half2, co2, i, g);
        float pe;
        uint32_t fb;
        bool in;
        if (!vox_sample_pass(d, g, s2_vox, s2, sup, half2, vs1, axk, sgn, isgn, pe, fb, in)) {
          interior += in ? 1u : 0u;
          continue;
        }
        const float su = axk == 0 ? g.l2.y : g.l2.x, sv = axk == 2 ? g.l2.y : g.l2.z;
        vox_reduce_add(w, g.pw, pe, g.fa, fb, su, sv, quant);
        ++samples;
      }
      samples = __reduce_add_sync(0xFFFFFFFFu, samples);
      interior = __reduce_add_sync(0xFFFFFFFFu, interior);
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        const uint32_t hi = vrank_hi(w[o], quant), lo = vrank_lo(w[o]);
        const uint32_t mh = __reduce_max_sync(0xFFFFFFFFu, hi);
        const uint32_t ml = __reduce_max_sync(0xFFFFFFFFu, hi == mh ? lo : 0u);
        const unsigned win = __ballot_sync(0xFFFFFFFFu, hi == mh && lo == ml);
        const int src = __ffs(win) - 1;
        VWin b;
        b.pos.x = __shfl_sync(0xFFFFFFFFu, w[o].pos.x, src);
        b.pos.y = __shfl_sync(0xFFFFFFFFu, w[o].pos.y, src);
        b.pos.z = __shfl_sync(0xFFFFFFFFu, w[o].pos.z, src);
        b.pen = __shfl_sync(0xFFFFFFFFu, w[o].pen, src);
        b.score = __shfl_sync(0xFFFFFFFFu, w[o].score, src);
        b.fa = __shfl_sync(0xFFFFFFFFu, w[o].fa, src);
        b.fb = __shfl_sync(0xFFFFFFFFu, w[o].fb, src);
        if (lane == code) mine[o] = b;
      }
      if (lane == code) {
        my_samples = samples;
        my_interior = interior;
      }
    }
    if (lane < 6) {  // the manifold of pass `lane` and its store: serial, small
      const uint32_t code = lane, axk = code >> 1;
      const float3 n_sep = mat_col(r2.R, int(axk)) * ((code & 1u) ? 1.f : -1.f);  // the face normal, world
      bool store = true;
      float4 lp[BB_MAX_CONTACTS], lo[BB_MAX_CONTACTS];
      uint32_t lf[BB_MAX_CONTACTS], lof[BB_MAX_CONTACTS];
      ContactsT<1> m;
      m.p = lp;
      m.f = lf;
      m.cc = 0;
      m.key = 90 + int(code);
      if (my_samples == 0) {
        store = code == 0 && my_interior > 0;
        // deep-interpenetration rescue (:1487-1506): one centre-to-centre contact
        const float3 dd = r1.p - r2.p;
        const float3 n_res = dot3(dd, dd) > 1e-8f ? dd * (1.0f / len3(dd)) : make_float3(0.f, 1.f, 0.f);
        m.normal = flip ? n_res : -n_res;
        m.set(0, (r1.p + r2.p) * 0.5f, -0.5f * vs1, 0xFFFFFFu);
        m.cc = 1;
      } else {
        // voxel_emit_manifold (:1330-1448); every sample of a pass has the normal n_sep
        m.normal = flip ? n_sep : -n_sep;
        const float align = dot3(n_sep, n_sep);
        uint32_t kept[4];
        uint32_t kn = 0;
        for (uint32_t o = 0; o < 4; ++o) {
          if (mine[o].pen >= 0.02f) continue;
          if (align <= 0.1f) continue;
          bool dup = false;
          for (uint32_t q = 0; q < kn; ++q)
            if (mine[kept[q]].fa == mine[o].fa) dup = true;
          if (dup) continue;
          kept[kn++] = o;
        }
        const uint32_t reps = kn == 1 ? 4u : (kn == 2 ? 2u : 1u);
        float3 t1 = cross3(n_sep, fabsf(n_sep.y) < 0.9f ? make_float3(0.f, 1.f, 0.f) : make_float3(1.f, 0.f, 0.f));
        t1 = t1 * (1.0f / len3(t1));
        const float3 t2 = cross3(n_sep, t1);
        const float3 da = (t1 + t2) * (0.318f * vs1), db = (t1 - t2) * (0.318f * vs1);
        int n_emit = 0;
        for (uint32_t k2 = 0; k2 < kn; ++k2) {
          const VWin& wo = mine[kept[k2]];
          const uint32_t vpar = (wo.fa ^ (wo.fa >> 8) ^ (wo.fa >> 16)) & 1u;
          float3 emitted[4];
          uint32_t en = 0;
          for (uint32_t c = 0; c < reps; ++c) {
            float3 pt = wo.pos;
            if (reps > 1) {
              const float3 offv = ((c < 2u) == (vpar == 0u)) ? da : db;
              const float3 off = offv * ((c & 1u) == 0u ? 1.f : -1.f);
              pt = wo.pos + off;
              if (!vox_corner_supported(d, pt, n_sep, r2, s2_vox, axk)) {
                pt = wo.pos + off * 0.5f;
                if (!vox_corner_supported(d, pt, n_sep, r2, s2_vox, axk)) pt = wo.pos;
              }
            }
            bool dup = false;
            for (uint32_t q = 0; q < en; ++q) {
              const float3 dp = pt - emitted[q];
              if (dot3(dp, dp) < 1.0e-12f) dup = true;
            }
            if (dup) continue;
            emitted[en++] = pt;
            m.set(n_emit, pt, wo.pen * align, wo.fa | (c << 24));
            ++n_emit;
          }
        }
        m.cc = n_emit;
        store = n_emit > 0;
      }
      if (store) np_store<1>(d, p, cur, warm, slot0 + code, ida, idb, d.flags[ida], A.p, B.p, m, true, lo, lof);
    }
    __syncwarp();
  }
}

// man_slot[man_index[k]] = k for every slot that collided; per-manifold statistics summed by
// each thread over its slots, then reduced over the block before one atomic per block (a few
// thousand updates of three counters instead of one per warp and slot group).
__global__ void k_compact(const DevState d, int cur) {
  __shared__ uint32_t s_red[3][32];
  const uint32_t S = slot_total(d);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, stride = gridDim.x * blockDim.x;
  uint32_t cc_sum = 0, fresh = 0, deep_bits = 0;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < S; k += stride) {
    if (!d.hit[k]) continue;
    d.man_slot[cur][d.man_index[k]] = k;
    const uint32_t cc = uint32_t(d.m_keycc[cur][k].y);
    cc_sum += cc;
    float deep = 0.f;
#pragma unroll
    for (uint32_t c = 0; c < BB_MAX_CONTACTS; ++c) {  // unrolled: the contacts' loads go out together
      if (c < cc) {
        const uint32_t ci = k * BB_MAX_CONTACTS + c;
        if (__float_as_uint(d.c_kt[cur][ci].w) == 0u) ++fresh;
        deep = fmaxf(deep, -d.c_pos[cur][ci].w);
      }
    }
    if (deep > 0.f) deep_bits = max(deep_bits, __float_as_uint(deep));  // positive floats order as their bits
  }
  cc_sum = __reduce_add_sync(0xFFFFFFFFu, cc_sum);
  fresh = __reduce_add_sync(0xFFFFFFFFu, fresh);
  deep_bits = __reduce_max_sync(0xFFFFFFFFu, deep_bits);
  if (lane == 0) {
    s_red[0][warp] = cc_sum;
    s_red[1][warp] = fresh;
    s_red[2][warp] = deep_bits;
  }
  __syncthreads();
  if (warp == 0) {
    const uint32_t nw = blockDim.x >> 5;
    cc_sum = lane < nw ? s_red[0][lane] : 0u;
    fresh = lane < nw ? s_red[1][lane] : 0u;
    deep_bits = lane < nw ? s_red[2][lane] : 0u;
    cc_sum = __reduce_add_sync(0xFFFFFFFFu, cc_sum);
    fresh = __reduce_add_sync(0xFFFFFFFFu, fresh);
    deep_bits = __reduce_max_sync(0xFFFFFFFFu, deep_bits);
    if (lane == 0) {
      if (cc_sum) atomicAdd(&d.ctr->contact_count, cc_sum);
      if (fresh) atomicAdd(&d.ctr->fresh, fresh);
      if (deep_bits) atomicMax(&d.ctr->max_pen_bits, deep_bits);
    }
  }
}

// per-body manifold lists: count, (scan), fill, sort
__global__ void k_csr_count(const DevState d, int cur) {
  const uint32_t M = d.ctr->manifold_count;
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    uint2 b = d.m_bodies[cur][d.man_slot[cur][m]];
    if (d.flags[b.x] & BB_BODY_DYNAMIC) atomicAdd(&d.csr_cursor[b.x], 1u);
    if (d.flags[b.y] & BB_BODY_DYNAMIC) atomicAdd(&d.csr_cursor[b.y], 1u);
  }
}
__global__ void k_csr_fill(const DevState d, int cur) {
  const uint32_t M = d.ctr->manifold_count;
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    uint2 b = d.m_bodies[cur][d.man_slot[cur][m]];
    if (d.flags[b.x] & BB_BODY_DYNAMIC) d.csr_list[cur][d.csr_start[cur][b.x] + atomicAdd(&d.csr_cursor[b.x], 1u)] = m;
    if (d.flags[b.y] & BB_BODY_DYNAMIC) d.csr_list[cur][d.csr_start[cur][b.y] + atomicAdd(&d.csr_cursor[b.y], 1u)] = m;
  }
}
__global__ void k_csr_sort(const DevState d, int cur, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // bit 0: not awake now (read by the next substep's classification); bit 1: not awake at the
  // last narrow phase either, so every pair of two such bodies is carried or recomputed from
  // unchanged poses (read by this substep's connected components)
  const uint32_t now = np_awake(d.flags[i]) ? 0u : 1u;
  d.frozen[i] = now | ((d.frozen[i] & now) << 1);
  uint32_t s0 = d.csr_start[cur][i], s1 = d.csr_start[cur][i + 1];
  uint32_t* L = d.csr_list[cur];
  if (s1 - s0 <= 8u) {  // short list: registers, a 19-comparator sorting network, loads issued together
    const uint32_t len = s1 - s0;
    uint32_t v[8];
#pragma unroll
    for (uint32_t j = 0; j < 8; ++j) v[j] = j < len ? L[s0 + j] : 0xFFFFFFFFu;
    auto cx = [&](int a, int b) {
      const uint32_t lo = min(v[a], v[b]), hi = max(v[a], v[b]);
      v[a] = lo;
      v[b] = hi;
    };
    cx(0, 2); cx(1, 3); cx(4, 6); cx(5, 7);
    cx(0, 4); cx(1, 5); cx(2, 6); cx(3, 7);
    cx(0, 1); cx(2, 3); cx(4, 5); cx(6, 7);
    cx(2, 4); cx(3, 5);
    cx(1, 4); cx(3, 6);
    cx(1, 2); cx(3, 4); cx(5, 6);
    uint32_t slot[8];
#pragma unroll
    for (uint32_t j = 0; j < 8; ++j) slot[j] = j < len ? d.man_slot[cur][v[j]] : 0u;
    uint2 b[8];
#pragma unroll
    for (uint32_t j = 0; j < 8; ++j) b[j] = j < len ? d.m_bodies[cur][slot[j]] : make_uint2(0u, 0u);
#pragma unroll
    for (uint32_t j = 0; j < 8; ++j) {
      if (j < len) {
        L[s0 + j] = v[j];
        d.csr_partner[cur][s0 + j] = b[j].x == i ? b[j].y : b[j].x;
        d.csr_slot[cur][s0 + j] = slot[j];
      }
    }
    return;
  }
  for (uint32_t a = s0 + 1; a < s1; ++a) {
    uint32_t v = L[a];
    uint32_t b = a;
    while (b > s0 && L[b - 1] > v) {
      L[b] = L[b - 1];
      --b;
    }
    L[b] = v;
  }
  // partner body and slot of every entry, so lookups by pair scan contiguous arrays
  for (uint32_t e = s0; e < s1; ++e) {
    const uint32_t slot = d.man_slot[cur][L[e]];
    const uint2 b = d.m_bodies[cur][slot];
    d.csr_partner[cur][e] = b.x == i ? b.y : b.x;
    d.csr_slot[cur][e] = slot;
  }
}

void bb_narrow_phase(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, const StepScratch& sc, int sms,
                     int cur, bool warm) {
  const int T = BB_THREADS;
  int grid = sms * 8;
  if (d.vox_on) {  // six slots per voxel pair: count, scan, fill
    k_slot_count<<<grid, T, 0, s>>>(d);
    bb_launch_scan(s, d.slot_cnt, d.slot_off, &d.ctr->pair_count, d.pair_capacity, &d.ctr->slot_count,
                   sc.scan_status + 6 * size_t(sc.scan_tiles), sc.scan_tile_ctr + 6, d.ctr);
    k_slot_fill<<<grid, T, 0, s>>>(d);
  }
  k_np_classify<<<sms * 8, 32 * BB_CLS_WARPS, 0, s>>>(d, cur, warm ? 1 : 0);
  k_narrow_carry<<<sms * 8, 256, 0, s>>>(d, cur, p.solver != BB_SOLVER_AVBD ? 1 : 0);
  k_narrow<<<sms * (p.narrow_blocks_per_sm ? p.narrow_blocks_per_sm : 16u), 128, 0, s>>>(d, p, cur, warm ? 1 : 0);
  if (d.vox_on) k_voxel_narrow<<<sms * 8, 256, 0, s>>>(d, p, cur, warm ? 1 : 0);
  // compact order: exclusive scan of the hit flags over the slots
  bb_launch_scan(s, d.hit, d.man_index, d.vox_on ? &d.ctr->slot_count : &d.ctr->pair_count, d.pair_capacity,
                 &d.ctr->manifold_count, sc.scan_status + sc.scan_tiles, sc.scan_tile_ctr + 1, d.ctr);
  k_compact<<<grid, T, 0, s>>>(d, cur);
  // per-body lists
  cudaMemsetAsync(d.csr_cursor, 0, sizeof(uint32_t) * (n + 1), s);
  k_csr_count<<<grid, T, 0, s>>>(d, cur);
  bb_launch_scan(s, d.csr_cursor, d.csr_start[cur], nullptr, n + 1, nullptr, sc.scan_status + 2 * sc.scan_tiles,
                 sc.scan_tile_ctr + 2, d.ctr);
  cudaMemsetAsync(d.csr_cursor, 0, sizeof(uint32_t) * (n + 1), s);
  k_csr_fill<<<grid, T, 0, s>>>(d, cur);
  k_csr_sort<<<(n + T - 1) / T, T, 0, s>>>(d, cur, n);
}
