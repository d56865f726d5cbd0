// bb_oracle_math.hpp -- TEST INFRASTRUCTURE ONLY (the oracle).  Never linked into the
// product library; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// load it.
//
// Vector / quaternion / 3x3 matrix helpers restated from the reference's shared math
// (include/math.hpp, include/shared.inl, src/shaders/extensions.slang), templated on the
// real type R (double for the checker, float for the timed CPU baseline).
//
// Matrix convention: Mat3::m[r][c] is row r, column c, exactly as a Slang matrix built
// from three row vectors.  mul_mv(M, v) = M*v (Slang mul(M, v)); mul_vm(v, M) = v^T*M
// (Slang mul(v, M)).
#pragma once
#include <cmath>
#include <cstring>
#include <cstdint>
#include <cfloat>
#include <algorithm>

namespace bbo {

template <class R> struct Vec3 {
  R x, y, z;
  Vec3() : x(0), y(0), z(0) {}
  Vec3(R a, R b, R c) : x(a), y(b), z(c) {}
  R& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class R> inline Vec3<R> operator+(Vec3<R> a, Vec3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline Vec3<R> operator-(Vec3<R> a, Vec3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline Vec3<R> operator-(Vec3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline Vec3<R> operator*(Vec3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline Vec3<R> operator*(R s, Vec3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline Vec3<R> operator/(Vec3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline Vec3<R> cmul(Vec3<R> a, Vec3<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class R> inline R dot(Vec3<R> a, Vec3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline Vec3<R> cross(Vec3<R> a, Vec3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline R length(Vec3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> inline Vec3<R> normalize(Vec3<R> a) { return a * (R(1) / length(a)); }
template <class R> inline Vec3<R> vabs(Vec3<R> a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
template <class T, class R> inline Vec3<T> vcast(Vec3<R> a) { return {T(a.x), T(a.y), T(a.z)}; }

// Quaternion with vector part v and scalar w (include/math.hpp:262-355).
template <class R> struct Quat {
  Vec3<R> v;
  R w;
  Quat() : v(), w(1) {}
  Quat(Vec3<R> vv, R ww) : v(vv), w(ww) {}
  Quat conjugate() const { return Quat({-v.x, -v.y, -v.z}, w); }
  R magnitude() const { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z + w * w); }
  Quat normalize() const {
    R mag = magnitude();
    return Quat(v / mag, w / mag);
  }
};
// Hamilton product, term order of include/math.hpp:357-364.
template <class R> inline Quat<R> operator*(Quat<R> q1, Quat<R> q2) {
  return Quat<R>(Vec3<R>(q1.w * q2.v.x + q1.v.x * q2.w + q1.v.y * q2.v.z - q1.v.z * q2.v.y,
                         q1.w * q2.v.y + q1.v.y * q2.w + q1.v.z * q2.v.x - q1.v.x * q2.v.z,
                         q1.w * q2.v.z + q1.v.z * q2.w + q1.v.x * q2.v.y - q1.v.y * q2.v.x),
                 q1.w * q2.w - q1.v.x * q2.v.x - q1.v.y * q2.v.y - q1.v.z * q2.v.z);
}

template <class R> struct Mat3 {
  R m[3][3];
  Mat3() {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) m[i][j] = 0;
  }
  static Mat3 rows(Vec3<R> a, Vec3<R> b, Vec3<R> c) {
    Mat3 r;
    for (int j = 0; j < 3; ++j) {
      r.m[0][j] = a[j];
      r.m[1][j] = b[j];
      r.m[2][j] = c[j];
    }
    return r;
  }
  Vec3<R> row(int i) const { return {m[i][0], m[i][1], m[i][2]}; }
  Vec3<R> col(int j) const { return {m[0][j], m[1][j], m[2][j]}; }
};
template <class R> inline Mat3<R> transpose(const Mat3<R>& a) {
  Mat3<R> r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
  return r;
}
template <class R> inline Mat3<R> mabs(const Mat3<R>& a) {
  Mat3<R> r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = std::fabs(a.m[i][j]);
  return r;
}
template <class R> inline Mat3<R> mul_mm(const Mat3<R>& a, const Mat3<R>& b) {
  Mat3<R> r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
  return r;
}
template <class R> inline Vec3<R> mul_mv(const Mat3<R>& a, Vec3<R> v) {
  return {a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z, a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
          a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}
template <class R> inline Vec3<R> mul_vm(Vec3<R> v, const Mat3<R>& a) {
  return {v.x * a.m[0][0] + v.y * a.m[1][0] + v.z * a.m[2][0], v.x * a.m[0][1] + v.y * a.m[1][1] + v.z * a.m[2][1],
          v.x * a.m[0][2] + v.y * a.m[1][2] + v.z * a.m[2][2]};
}
template <class R> inline Mat3<R> diag(Vec3<R> d) {
  Mat3<R> r;
  r.m[0][0] = d.x;
  r.m[1][1] = d.y;
  r.m[2][2] = d.z;
  return r;
}

// Quaternion::to_matrix (include/math.hpp:287-304): rows of the standard rotation matrix.
template <class R> inline Mat3<R> to_matrix(const Quat<R>& q) {
  R x2 = q.v.x + q.v.x, y2 = q.v.y + q.v.y, z2 = q.v.z + q.v.z;
  R xx = q.v.x * x2, xy = q.v.x * y2, xz = q.v.x * z2;
  R yy = q.v.y * y2, yz = q.v.y * z2, zz = q.v.z * z2;
  R wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
  return Mat3<R>::rows(Vec3<R>(1 - (yy + zz), xy - wz, xz + wy), Vec3<R>(xy + wz, 1 - (xx + zz), yz - wx),
                       Vec3<R>(xz - wy, yz + wx, 1 - (xx + yy)));
}

// RigidBody::rotate_vector / rotate_vector_inverse (include/shared.inl:455-463): two
// Hamilton products.
template <class R> inline Vec3<R> rotate_vector(const Quat<R>& q, Vec3<R> v) {
  return (q * Quat<R>(v, R(0)) * q.conjugate()).v;
}
template <class R> inline Vec3<R> rotate_vector_inverse(const Quat<R>& q, Vec3<R> v) {
  return (q.conjugate() * Quat<R>(v, R(0)) * q).v;
}

// Transform with Slang semantics (include/math.hpp:400-422, extensions.slang:212-258):
// `rot` is the matrix whose ROWS are the body axes; vectors multiply from the left.
template <class R> struct Transform {
  Mat3<R> rot;
  Vec3<R> pos;
  Vec3<R> rotate(Vec3<R> v) const { return mul_vm(v, rot); }
  Vec3<R> rotate_transpose(Vec3<R> v) const { return mul_vm(v, transpose(rot)); }
  Vec3<R> transform(Vec3<R> v) const { return mul_vm(v, rot) + pos; }
  Vec3<R> transform_transpose(Vec3<R> v) const { return mul_vm(v - pos, transpose(rot)); }
  Vec3<R> get_axis(int i) const { return rot.row(i); }
  Vec3<R> get_inverse_axis(int i) const { return transpose(rot).row(i); }
};

// Order-preserving float<->uint map (include/math.hpp:228-256).
inline uint32_t float_to_ordered(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  uint32_t mask = uint32_t(-int32_t(u >> 31)) | 0x80000000u;
  return u ^ mask;
}

}  // namespace bbo
