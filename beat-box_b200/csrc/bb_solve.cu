// bb_solve.cu -- PGS_SOFT and AVBD contact solvers.
//
// Reference: PGS_SOFT::pre_step / solve (src/shaders/simulation/solvers.slang:142-279) run
// per colour (RB_sim.slang:1408-1578) in the order of RBM:1369-1389 (pre-step, I solve sweeps,
// integrate positions RB_sim.slang:1287-1326, I relax sweeps), each sweep colours 0..31 then
// the serial overflow bucket.  AVBD (src/shaders/simulation/avbd.slang): body colouring
// (:812-981), prepare (:70-128), warm start (:390-473), support depth (:667-724), primal
// (:478-658) with the 6x6 LDL^T of avbd_solve6 (:329-387), dual (:728-808), finalize
// (:132-202), post-stabilisation sweeps (RBM:1400-1425).
//
// B200 design: each solver phase is ONE persistent cooperative kernel that walks compact
// colour buckets and separates colours with a grid barrier, instead of the reference's
// (2I+1) x 33 dispatches that each scan every manifold and filter by colour.  Contact rows
// are 64-byte float4 groups per contact; body velocities and the world inverse inertia are
// float4 loads.  The 6x6 block solve stays in registers.
#include "bb_common.cuh"
#include <algorithm>

#include "bb_kernels.cuh"

// ---------------------------------------------------------------------------------------
// PGS_SOFT
struct BodyVel {
  float3 v, w;
};

__device__ __forceinline__ Sym3 load_iw(const DevState& d, uint32_t i) {
  float4 a = d.iw[2 * i], b = d.iw[2 * i + 1];
  return Sym3{a.x, a.y, a.z, a.w, b.x, b.y};
}
__device__ __forceinline__ void store_iw(const DevState& d, uint32_t i, const Sym3& s) {
  d.iw[2 * i] = make_float4(s.xx, s.xy, s.xz, s.yy);
  d.iw[2 * i + 1] = make_float4(s.yz, s.zz, 0.f, 0.f);
}
__device__ __forceinline__ bool awake(uint32_t f) { return (f & BB_BODY_DYNAMIC) && !(f & BB_BODY_SLEEPING); }

// Quaternion integration (extensions.slang:148-166)
__device__ __forceinline__ Quatf apply_angular_velocity(Quatf rot, float3 w, float dt) {
  float angle = len3(w) * dt;
  Quatf q;
  if (angle > 0.0001f) {
    float3 axis = w * (1.0f / len3(w));
    float half = angle / 2.0f;
    float sh, ch;
    sincosf(half, &sh, &ch);
    q = Quatf{axis.x * sh, axis.y * sh, axis.z * sh, ch};
  } else {
    float3 dr = w * dt * 0.5f;
    q = Quatf{dr.x, dr.y, dr.z, 1.0f};
  }
  return q_normalize(q_mul(q, rot));
}

// ---- PGS_SOFT arithmetic of one contact, shared by both schedules (same expressions, so the
// schedules agree bit for bit) -------------------------------------------------------------

// Every operation below is an explicitly rounded intrinsic (fma where a product feeds a sum),
// so the compiler has nothing left to contract: each inlined copy of this arithmetic -- the
// barrier schedule's register-held and streamed contacts, the dataflow schedule -- produces
// the same bits.
__device__ __forceinline__ float3 xadd(float3 a, float3 b) {
  return make_float3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z));
}
__device__ __forceinline__ float3 xsub(float3 a, float3 b) {
  return make_float3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}
__device__ __forceinline__ float3 xscale(float3 a, float s) {
  return make_float3(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s));
}
__device__ __forceinline__ float3 xaxpy(float3 a, float s, float3 y) {  // a * s + y
  return make_float3(__fmaf_rn(a.x, s, y.x), __fmaf_rn(a.y, s, y.y), __fmaf_rn(a.z, s, y.z));
}
__device__ __forceinline__ float xdot(float3 a, float3 b) {
  return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x)));
}
__device__ __forceinline__ float3 xcross(float3 a, float3 b) {
  return make_float3(__fmaf_rn(a.y, b.z, -__fmul_rn(a.z, b.y)), __fmaf_rn(a.z, b.x, -__fmul_rn(a.x, b.z)),
                     __fmaf_rn(a.x, b.y, -__fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float3 xsym(const Sym3& s, float3 v) {
  return make_float3(__fmaf_rn(s.xz, v.z, __fmaf_rn(s.xy, v.y, __fmul_rn(s.xx, v.x))),
                     __fmaf_rn(s.yz, v.z, __fmaf_rn(s.yy, v.y, __fmul_rn(s.xy, v.x))),
                     __fmaf_rn(s.zz, v.z, __fmaf_rn(s.yz, v.y, __fmul_rn(s.xz, v.x))));
}
// v_a -= P m_a, w_a -= I_a (r1 x P), v_b += P m_b, w_b += I_b (r2 x P)
__device__ __forceinline__ void xapply(float3 P, float3 r1, float3 r2, float ima, float imb, const Sym3& IA,
                                       const Sym3& IB, float3& va, float3& wa, float3& vb, float3& wb) {
  va = xaxpy(P, -ima, va);
  wa = xsub(wa, xsym(IA, xcross(r1, P)));
  vb = xaxpy(P, imb, vb);
  wb = xadd(wb, xsym(IB, xcross(r2, P)));
}

// soft-constraint coefficients of a manifold (solvers.slang:150-158)
struct SoftCoef {
  float bf, mcoef, icoef, inv_h;
};
__device__ __forceinline__ SoftCoef pgs_soft_coef(float ima, float imb, float h, float hertz) {
  const float ch = (ima == 0.f || imb == 0.f) ? __fmul_rn(2.0f, hertz) : hertz;
  const float zeta = 10.0f;
  const float omega = __fmul_rn(2.0f * 3.14159265359f, ch);
  const float ho = __fmul_rn(h, omega);
  const float den = __fadd_rn(2.0f * zeta, ho);
  const float c = __fmul_rn(ho, den);
  SoftCoef s;
  s.bf = __fdiv_rn(omega, den);
  s.icoef = __fdiv_rn(1.0f, __fadd_rn(1.0f, c));
  s.mcoef = __fmul_rn(c, s.icoef);
  s.inv_h = h > 0.f ? __fdiv_rn(1.0f, h) : 0.f;
  return s;
}

// effective mass of one row along direction u: 1 / (m_a + m_b + (r1 x u) I_a (r1 x u) + ...)
__device__ __forceinline__ float xrow_mass(float3 r1, float3 r2, float3 u, float ima, float imb, const Sym3& IA,
                                           const Sym3& IB) {
  const float3 c1 = xcross(r1, u), c2 = xcross(r2, u);
  const float k = __fadd_rn(__fadd_rn(__fadd_rn(ima, imb), xdot(c1, xsym(IA, c1))), xdot(c2, xsym(IB, c2)));
  return k == 0.f ? 0.f : __fdiv_rn(1.0f, k);
}

// rows of one contact (solvers.slang:160-190): R1 = (r1, normal mass), R2 = (r2, tangent
// mass 0), K = (tangent mass 1, bias, mass coefficient, impulse coefficient)
__device__ __forceinline__ void pgs_contact_rows(float4 pp, float3 aa, float3 ab, float3 n, float3 t0, float3 t1,
                                                 float ima, float imb, const Sym3& IA, const Sym3& IB,
                                                 const SoftCoef& s, float4& R1, float4& R2, float4& K) {
  const float3 r1 = xsub(f3(pp), aa), r2 = xsub(f3(pp), ab);
  const float nmass = xrow_mass(r1, r2, n, ima, imb, IA, IB);
  const float tm0 = xrow_mass(r1, r2, t0, ima, imb, IA, IB);
  const float tm1 = xrow_mass(r1, r2, t1, ima, imb, IA, IB);
  const float pen = pp.w;
  const float bias_value = pen > 0.f ? __fmul_rn(pen, s.inv_h) : fmaxf(__fmul_rn(s.bf, pen), -4.0f);
  R1 = f4(r1, nmass);
  R2 = f4(r2, tm0);
  K = make_float4(tm1, bias_value, s.mcoef, s.icoef);
}

// warm start of one contact: apply the accumulated impulse (solvers.slang:191-195)
__device__ __forceinline__ void pgs_contact_warm(float3 r1, float3 r2, float4 lam, float3 n, float3 t0, float3 t1,
                                                 bool fric, float ima, float imb, const Sym3& IA, const Sym3& IB,
                                                 float3& va, float3& wa, float3& vb, float3& wb) {
  float3 P = xscale(n, lam.x);
  if (fric) P = xaxpy(t1, lam.z, xaxpy(t0, lam.y, P));
  xapply(P, r1, r2, ima, imb, IA, IB, va, wa, vb, wb);
}

// relative velocity at the contact: (v_b + w_b x r2) - (v_a + w_a x r1)
__device__ __forceinline__ float3 xrel(float3 r1, float3 r2, float3 va, float3 wa, float3 vb, float3 wb) {
  return xsub(xadd(vb, xcross(wb, r2)), xadd(va, xcross(wa, r1)));
}

// one contact of PGS_SOFT::solve (solvers.slang:209-277): two friction rows, then the normal row.
// Both friction rows take their impulse from the same relative velocity (computed once, before
// either is applied, as the reference does), so their two impulses are applied as one sum: the
// same result up to rounding, with one body update instead of two.
__device__ __forceinline__ void pgs_contact_solve(float4 R1, float4 R2, float4 K, float4& lam, float3 n, float3 t0,
                                                  float3 t1, float mu, bool use_bias, bool accum, bool fric, float ima,
                                                  float imb, const Sym3& IA, const Sym3& IB, float3& va, float3& wa,
                                                  float3& vb, float3& wb) {
  const float3 r1 = f3(R1), r2 = f3(R2);
  if (fric) {
    const float3 rv = xrel(r1, r2, va, wa, vb, wb);
    float imp_t[2] = {lam.y, lam.z}, ti[2];
    const float tmass[2] = {R2.w, K.x};
    const float maxf = __fmul_rn(mu, lam.x);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const float3 t = k == 0 ? t0 : t1;
      ti[k] = __fmul_rn(tmass[k], -xdot(rv, t));
      if (accum) {
        const float old = imp_t[k];
        imp_t[k] = fminf(fmaxf(__fadd_rn(old, ti[k]), -maxf), maxf);
        ti[k] = __fsub_rn(imp_t[k], old);
      } else {
        ti[k] = fminf(fmaxf(ti[k], -maxf), maxf);
      }
    }
    xapply(xaxpy(t1, ti[1], xscale(t0, ti[0])), r1, r2, ima, imb, IA, IB, va, wa, vb, wb);
    lam.y = imp_t[0];
    lam.z = imp_t[1];
  }
  const float vn = xdot(xrel(r1, r2, va, wa, vb, wb), n);
  float bias = 0.f, ms = 1.f, is = 0.f;
  if (K.y > 0.f) {
    bias = K.y;
  } else if (use_bias) {
    bias = K.y;
    ms = K.z;
    is = K.w;
  }
  float imp = __fsub_rn(__fmul_rn(__fmul_rn(-R1.w, ms), __fadd_rn(vn, bias)), __fmul_rn(is, lam.x));
  if (accum) {
    const float old = lam.x;
    lam.x = fmaxf(__fadd_rn(old, imp), 0.f);
    imp = __fsub_rn(lam.x, old);
  } else {
    imp = fmaxf(imp, 0.f);
  }
  xapply(xscale(n, imp), r1, r2, ima, imb, IA, IB, va, wa, vb, wb);
}

// PGS_SOFT::pre_step (solvers.slang:143-196) of one manifold slot: rows, then warm start
__device__ void pgs_pre_step_slot(const DevState& d, const Params& p, int cur, uint32_t slot, uint2 b, float h,
                                  float hertz) {
  const uint32_t fa = d.flags[b.x], fb = d.flags[b.y];
  if (!awake(fa) && !awake(fb)) return;
  const float ima = d.pos[b.x].w, imb = d.pos[b.y].w;
  const Sym3 IA = load_iw(d, b.x), IB = load_iw(d, b.y);
  float3 va = f3(d.vel[b.x]), wa = f3(d.omega[b.x]), vb = f3(d.vel[b.y]), wb = f3(d.omega[b.y]);
  const float3 n = f3(d.m_normal[cur][slot]);
  const float3 t0 = f3(d.m_t0[cur][slot]), t1 = f3(d.m_t1[cur][slot]);
  const float3 aa = f3(d.m_anchor_a[cur][slot]), ab = f3(d.m_anchor_b[cur][slot]);
  const int cc = d.m_keycc[cur][slot].y;
  const bool accum = p.flags & BB_SIM_ACCUM_IMPULSE, fric = p.flags & BB_SIM_FRICTION;
  const SoftCoef s = pgs_soft_coef(ima, imb, h, hertz);
  for (int j = 0; j < cc; ++j) {
    const uint32_t ci = slot * BB_MAX_CONTACTS + j;
    float4 R1, R2, K;
    pgs_contact_rows(d.c_pos[cur][ci], aa, ab, n, t0, t1, ima, imb, IA, IB, s, R1, R2, K);
    d.c_r1[ci] = R1;
    d.c_r2[ci] = R2;
    d.c_k[ci] = K;
    float4 lam = d.c_lam[cur][ci];
    // the reference writes its mass coefficient / tangent masses into the persistent contact
    d.c_lam[cur][ci] = make_float4(lam.x, lam.y, lam.z, s.mcoef);
    float4 kt4 = d.c_kt[cur][ci];
    d.c_kt[cur][ci] = make_float4(R2.w, K.x, kt4.z, kt4.w);
    if (accum) pgs_contact_warm(f3(R1), f3(R2), lam, n, t0, t1, fric, ima, imb, IA, IB, va, wa, vb, wb);
  }
  if (fa & BB_BODY_DYNAMIC) {
    d.vel[b.x] = f4(va, d.vel[b.x].w);
    d.omega[b.x] = f4(wa, 0.f);
  }
  if (fb & BB_BODY_DYNAMIC) {
    d.vel[b.y] = f4(vb, d.vel[b.y].w);
    d.omega[b.y] = f4(wb, 0.f);
  }
}

// PGS_SOFT::solve (solvers.slang:199-278) of one manifold slot
__device__ void pgs_solve_slot(const DevState& d, const Params& p, int cur, uint32_t slot, uint2 b, bool use_bias) {
  const uint32_t fa = d.flags[b.x], fb = d.flags[b.y];
  if (!awake(fa) && !awake(fb)) return;
  const float ima = d.pos[b.x].w, imb = d.pos[b.y].w;
  const Sym3 IA = load_iw(d, b.x), IB = load_iw(d, b.y);
  float4 va4 = d.vel[b.x], vb4 = d.vel[b.y];
  float3 va = f3(va4), wa = f3(d.omega[b.x]), vb = f3(vb4), wb = f3(d.omega[b.y]);
  const float mu = sqrtf(d.iinv[b.x].w * d.iinv[b.y].w);
  const float3 n = f3(d.m_normal[cur][slot]);
  const float3 t0 = f3(d.m_t0[cur][slot]), t1 = f3(d.m_t1[cur][slot]);
  const int cc = d.m_keycc[cur][slot].y;
  const bool accum = p.flags & BB_SIM_ACCUM_IMPULSE, fric = p.flags & BB_SIM_FRICTION;
  for (int j = 0; j < cc; ++j) {
    const uint32_t ci = slot * BB_MAX_CONTACTS + j;
    float4 lam = d.c_lam[cur][ci];
    pgs_contact_solve(d.c_r1[ci], d.c_r2[ci], d.c_k[ci], lam, n, t0, t1, mu, use_bias, accum, fric, ima, imb, IA, IB,
                      va, wa, vb, wb);
    d.c_lam[cur][ci] = lam;
  }
  if (fa & BB_BODY_DYNAMIC) {
    d.vel[b.x] = f4(va, va4.w);
    d.omega[b.x] = f4(wa, 0.f);
  }
  if (fb & BB_BODY_DYNAMIC) {
    d.vel[b.y] = f4(vb, vb4.w);
    d.omega[b.y] = f4(wb, 0.f);
  }
}

// integrate one body (RB_sim.slang:1287-1326) and refresh its world inverse inertia
// Compiled once (not inlined) so both schedules integrate with the same instructions.
__device__ __noinline__ void pgs_integrate_body(float4* pos, float4* rot, const float4* vel, const float4* omega,
                                                const float4* iinv, const float4* ioff, bool full, float4* iw,
                                                uint32_t i, float h, bool tq) {
  const float4 ps = pos[i];
  const float3 v = f3(vel[i]);
  pos[i] = make_float4(ps.x + v.x * h, ps.y + v.y * h, ps.z + v.z * h, ps.w);
  const Quatf q = apply_angular_velocity(q_from(rot[i]), f3(omega[i]), h);
  rot[i] = q_to4(q);
  const Sym3 s = body_world_inv_inertia(iinv, ioff, full, i, q, tq);
  iw[2 * i] = make_float4(s.xx, s.xy, s.xz, s.yy);
  iw[2 * i + 1] = make_float4(s.yz, s.zz, 0.f, 0.f);
}
__device__ __noinline__ void pgs_world_inertia_body(const float4* rot, const float4* iinv, const float4* ioff,
                                                    bool full, float4* iw, uint32_t i, bool tq) {
  const Sym3 s = body_world_inv_inertia(iinv, ioff, full, i, q_from(rot[i]), tq);
  iw[2 * i] = make_float4(s.xx, s.xy, s.xz, s.yy);
  iw[2 * i + 1] = make_float4(s.yz, s.zz, 0.f, 0.f);
}
__device__ __forceinline__ void pgs_world_inertia(const DevState& d, uint32_t i, bool tq) {
  pgs_world_inertia_body(d.rot, d.iinv, d.iinv_off, d.full_inertia != 0, d.iw, i, tq);
}
__device__ __forceinline__ void pgs_integrate(const DevState& d, uint32_t i, float h, bool tq) {
  pgs_integrate_body(d.pos, d.rot, d.vel, d.omega, d.iinv, d.iinv_off, d.full_inertia != 0, d.iw, i, h, tq);
}

// ---------------------------------------------------------------------------------------
// PGS_SOFT, colour-barrier schedule: one persistent cooperative kernel.
//
// Every sweep walks the colour buckets in order with a grid barrier after each colour; item k
// of a colour (a manifold) always belongs to the same thread, so the thread can load the
// next colour's item -- its record, contact frame, rows and impulses, none of which another
// thread writes -- BEFORE the barrier, and after the barrier only the two bodies' velocities
// and inertias remain to be fetched: one memory round trip per colour on the critical path.
#define BB_PGS_THREADS 256  // one block per SM: up to 255 registers for the held item
#define BB_PGS_SKIP (1u << 10)

// The kernel works on a compact copy in colour order: item k's record, masses and contact frame
// at index k, its contacts' rows (c_r1, c_r2, c_k reused with compact indexing) and impulses
// (pgs_lam) at pgs_coff[k] + j.  The impulses go back to the persistent slot-indexed contacts
// when the kernel ends.  Dense arrays keep the per-sweep working set (about 80 B per manifold,
// 64 B per contact, 64 B per body) resident in L2.
template <int PF>  // contacts of an item held in registers across the barrier
struct PgsItem {
  uint4 rec;    // contact offset, body a, body b, contact count | dynamic a << 8 | dynamic b << 9 | skip << 10
  float4 mass;  // inverse mass a, inverse mass b, friction, -
  float4 n, t0, t1;
  float4 R1[PF], R2[PF], K[PF], lam[PF];
};

// Contacts beyond the PF register-held ones (up to BB_MAX_CONTACTS - PF) are staged in this
// thread's slot of dynamic shared memory with cp.async at prefetch time, so the run does not
// pay one global round trip per extra contact.  Slot layout: [contact][R1, R2, K, lam].
#define BB_PGS_EXTRA (BB_MAX_CONTACTS - 4)
// Next-item staging (k_pgs_soft): the item a thread runs after the current one in the same
// colour -- masses, frame, up to four contacts' rows and impulses, and both bodies' velocities
// and world inverse inertias -- copied with cp.async while the current item computes.  Element e
// of thread t sits at e * BB_PGS_THREADS + t, so a warp's 16-byte accesses hit distinct banks.
#define BB_PGS_NEXT 28  // float4 per thread: mass, n, t0, t1, 4 x (R1, R2, K, lam), 8 body words
#define BB_PGS_SMEM_EXTRA (BB_PGS_THREADS * BB_PGS_EXTRA * 4 * 16)
#define BB_PGS_SMEM (BB_PGS_SMEM_EXTRA + BB_PGS_THREADS * BB_PGS_NEXT * 16)
__device__ __forceinline__ float4* pgs_extra_slot() {
  extern __shared__ float4 s_pgs_extra[];
  return s_pgs_extra + threadIdx.x * (BB_PGS_EXTRA * 4);
}
__device__ __forceinline__ float4* pgs_next_base() {
  extern __shared__ float4 s_pgs_extra[];
  return s_pgs_extra + BB_PGS_THREADS * BB_PGS_EXTRA * 4 + threadIdx.x;
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t s = uint32_t(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// STAGED: extra contacts go to shared memory (the persistent kernels); else they stay in global
// memory and the run reads them there (the serial overflow path, which must not disturb the
// slot of the item already prefetched for the next colour).
template <int PF, bool STAGED>
__device__ __forceinline__ void pgs_item_fill(const DevState& d, uint32_t k, PgsItem<PF>& x) {
  x.mass = d.pgs_mass[k];
  x.n = d.pgs_frame[3 * k];
  x.t0 = d.pgs_frame[3 * k + 1];
  x.t1 = d.pgs_frame[3 * k + 2];
  const uint32_t c0 = x.rec.x, cc = x.rec.w & 0xFFu;
#pragma unroll
  for (int j = 0; j < PF; ++j) {
    if (uint32_t(j) < cc) {
      x.R1[j] = d.c_r1[c0 + j];
      x.R2[j] = d.c_r2[c0 + j];
      x.K[j] = d.c_k[c0 + j];
      x.lam[j] = d.pgs_lam[c0 + j];
    }
  }
  if (STAGED && cc > uint32_t(PF)) {
    float4* slot = pgs_extra_slot();
    for (uint32_t j = PF; j < cc; ++j) {
      float4* e = slot + (j - PF) * 4;
      cp_async16(e + 0, d.c_r1 + c0 + j);
      cp_async16(e + 1, d.c_r2 + c0 + j);
      cp_async16(e + 2, d.c_k + c0 + j);
      cp_async16(e + 3, d.pgs_lam + c0 + j);
    }
    cp_async_commit();
  }
}

// item k given its record (loaded ahead): masses, frame, rows, impulses
template <int PF, bool STAGED = true>
__device__ __forceinline__ void pgs_item_load_rest(const DevState& d, uint32_t k, uint4 rec, PgsItem<PF>& x) {
  x.rec = rec;
  pgs_item_fill<PF, STAGED>(d, k, x);
}

template <int PF, bool STAGED = true>
__device__ __forceinline__ void pgs_item_load(const DevState& d, uint32_t k, PgsItem<PF>& x) {
  x.rec = d.pgs_rec[k];
  pgs_item_fill<PF, STAGED>(d, k, x);
}

// contacts per colour-ordered item (0 for items whose bodies both sleep): scanned into pgs_coff
__global__ void k_pgs_count(const DevState d, int cur) {
  const uint32_t M = d.ctr->manifold_count;
  const uint32_t* list = d.bucket_vals[1];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < M; k += gridDim.x * blockDim.x) {
    const uint32_t slot = d.man_slot[cur][list[k]];
    const uint2 b = d.m_bodies[cur][slot];
    const bool skip = !awake(d.flags[b.x]) && !awake(d.flags[b.y]);
    d.pgs_cnt[k] = skip ? 0u : uint32_t(d.m_keycc[cur][slot].y);
    const uint32_t act = __ballot_sync(__activemask(), !skip);
    if ((threadIdx.x & 31u) == uint32_t(__ffs(__activemask()) - 1) && act) atomicAdd(&d.ctr->pgs_manifolds, __popc(act));
    if (!skip) {  // set once: most threads only read the flag (33 hot words otherwise take every store)
      uint32_t* f = &d.colour_awake[min(d.gc_color[list[k]], uint32_t(BB_MAX_COLORS))];
      if (*f == 0u) *f = 1u;
    }
  }
}

// compact record + rows of colour-ordered item k (the pre-step's row half; no body is touched)
__device__ void pgs_item_build(const DevState& d, int cur, uint32_t k, uint32_t m, float h, float hertz) {
  const uint32_t slot = d.man_slot[cur][m];
  const uint2 b = d.m_bodies[cur][slot];
  const uint32_t fa = d.flags[b.x], fb = d.flags[b.y];
  const uint32_t cc = d.pgs_cnt[k];  // 0 when both bodies sleep
  const uint32_t c0 = d.pgs_coff[k];
  const bool skip = !awake(fa) && !awake(fb);
  const float ima = d.pos[b.x].w, imb = d.pos[b.y].w;
  d.pgs_rec[k] = make_uint4(c0, b.x, b.y,
                            cc | ((fa & BB_BODY_DYNAMIC) ? 1u << 8 : 0u) | ((fb & BB_BODY_DYNAMIC) ? 1u << 9 : 0u) |
                                (skip ? BB_PGS_SKIP : 0u));
  d.pgs_mass[k] = make_float4(ima, imb, sqrtf(d.iinv[b.x].w * d.iinv[b.y].w), 0.f);
  d.pgs_slot[k] = slot;
  if (skip) return;
  const float4 n4 = d.m_normal[cur][slot], t04 = d.m_t0[cur][slot], t14 = d.m_t1[cur][slot];
  d.pgs_frame[3 * k] = n4;
  d.pgs_frame[3 * k + 1] = t04;
  d.pgs_frame[3 * k + 2] = t14;
  const Sym3 IA = load_iw(d, b.x), IB = load_iw(d, b.y);
  const float3 n = f3(n4), t0 = f3(t04), t1 = f3(t14);
  const float3 aa = f3(d.m_anchor_a[cur][slot]), ab = f3(d.m_anchor_b[cur][slot]);
  const SoftCoef s = pgs_soft_coef(ima, imb, h, hertz);
  for (uint32_t j = 0; j < cc; ++j) {
    const uint32_t ci = slot * BB_MAX_CONTACTS + j;
    float4 R1, R2, K;
    pgs_contact_rows(d.c_pos[cur][ci], aa, ab, n, t0, t1, ima, imb, IA, IB, s, R1, R2, K);
    d.c_r1[c0 + j] = R1;
    d.c_r2[c0 + j] = R2;
    d.c_k[c0 + j] = K;
    const float4 lam = d.c_lam[cur][ci];
    // the reference writes its mass coefficient / tangent masses into the persistent contact
    d.pgs_lam[c0 + j] = make_float4(lam.x, lam.y, lam.z, s.mcoef);
    const float4 kt4 = d.c_kt[cur][ci];
    d.c_kt[cur][ci] = make_float4(R2.w, K.x, kt4.z, kt4.w);
  }
}

// an item's two bodies: velocities and world inverse inertias
struct PgsBodies {
  float4 va, wa, ia0, ia1, vb, wb, ib0, ib1;
};
__device__ __forceinline__ PgsBodies pgs_bodies_load(const DevState& d, uint32_t a, uint32_t b) {
  PgsBodies B;
  B.va = d.vel[a];
  B.wa = d.omega[a];
  B.ia0 = d.iw[2 * a];
  B.ia1 = d.iw[2 * a + 1];
  B.vb = d.vel[b];
  B.wb = d.omega[b];
  B.ib0 = d.iw[2 * b];
  B.ib1 = d.iw[2 * b + 1];
  return B;
}

// mode 0: warm start, 1: solve sweep (soft bias), 2: relax sweep; B holds the item's bodies
template <int PF, bool STAGED = true>
__device__ __forceinline__ void pgs_item_compute(const DevState& d, const Params& p, PgsItem<PF>& x,
                                                 const PgsBodies& B, int mode) {
  if (x.rec.w & BB_PGS_SKIP) return;
  const bool accum = p.flags & BB_SIM_ACCUM_IMPULSE, fric = p.flags & BB_SIM_FRICTION;
  if (mode == 0 && !accum) return;
  const uint32_t a = x.rec.y, b = x.rec.z, c0 = x.rec.x, cc = x.rec.w & 0xFFu;
  const float4 va4 = B.va, vb4 = B.vb;
  float3 va = f3(va4), wa = f3(B.wa), vb = f3(vb4), wb = f3(B.wb);
  const Sym3 IA{B.ia0.x, B.ia0.y, B.ia0.z, B.ia0.w, B.ia1.x, B.ia1.y};
  const Sym3 IB{B.ib0.x, B.ib0.y, B.ib0.z, B.ib0.w, B.ib1.x, B.ib1.y};
  const float ima = x.mass.x, imb = x.mass.y, mu = x.mass.z;
  const float3 n = f3(x.n), t0 = f3(x.t0), t1 = f3(x.t1);
#pragma unroll
  for (int j = 0; j < PF; ++j) {
    if (uint32_t(j) < cc) {
      if (mode == 0) {
        pgs_contact_warm(f3(x.R1[j]), f3(x.R2[j]), x.lam[j], n, t0, t1, fric, ima, imb, IA, IB, va, wa, vb, wb);
      } else {
        pgs_contact_solve(x.R1[j], x.R2[j], x.K[j], x.lam[j], n, t0, t1, mu, mode == 1, accum, fric, ima, imb, IA,
                          IB, va, wa, vb, wb);
        d.pgs_lam[c0 + j] = x.lam[j];
      }
    }
  }
  if (cc > uint32_t(PF)) {  // contacts beyond the register-held ones
    const float4* slot = pgs_extra_slot();
    if (STAGED) cp_async_wait_all();
    for (uint32_t j = PF; j < cc; ++j) {
      const uint32_t ci = c0 + j;
      const float4* e = slot + (j - PF) * 4;
      const float4 R1 = STAGED ? e[0] : d.c_r1[ci], R2 = STAGED ? e[1] : d.c_r2[ci];
      float4 lam = STAGED ? e[3] : d.pgs_lam[ci];
      if (mode == 0) {
        pgs_contact_warm(f3(R1), f3(R2), lam, n, t0, t1, fric, ima, imb, IA, IB, va, wa, vb, wb);
      } else {
        const float4 K = STAGED ? e[2] : d.c_k[ci];
        pgs_contact_solve(R1, R2, K, lam, n, t0, t1, mu, mode == 1, accum, fric, ima, imb, IA, IB, va, wa, vb, wb);
        d.pgs_lam[ci] = lam;
      }
    }
  }
  if (x.rec.w & (1u << 8)) {
    d.vel[a] = f4(va, va4.w);
    d.omega[a] = f4(wa, 0.f);
  }
  if (x.rec.w & (1u << 9)) {
    d.vel[b] = f4(vb, vb4.w);
    d.omega[b] = f4(wb, 0.f);
  }
}

template <int PF, bool STAGED = true>
__device__ __forceinline__ void pgs_item_run(const DevState& d, const Params& p, int cur, PgsItem<PF>& x, int mode) {
  (void)cur;
  if (x.rec.w & BB_PGS_SKIP) return;
  if (mode == 0 && !(p.flags & BB_SIM_ACCUM_IMPULSE)) return;
  const PgsBodies B = pgs_bodies_load(d, x.rec.y, x.rec.z);
  pgs_item_compute<PF, STAGED>(d, p, x, B, mode);
}

// cp.async of the next item k (record r) of this thread's colour into its staging slot: the
// bodies cannot change before this thread runs the item (the colour's items share no body),
// and the rows and impulses are only written by the item itself.
template <int PF>
__device__ __forceinline__ void pgs_stage_next(const DevState& d, uint32_t k, uint4 r) {
  float4* nb = pgs_next_base();
  const uint32_t T = BB_PGS_THREADS, c0 = r.x, cc = min(r.w & 0xFFu, uint32_t(PF)), a = r.y, b = r.z;
  cp_async16(nb + 0 * T, d.pgs_mass + k);
  cp_async16(nb + 1 * T, d.pgs_frame + 3 * k);
  cp_async16(nb + 2 * T, d.pgs_frame + 3 * k + 1);
  cp_async16(nb + 3 * T, d.pgs_frame + 3 * k + 2);
  for (uint32_t j = 0; j < cc; ++j) {
    cp_async16(nb + (4 + 4 * j) * T, d.c_r1 + c0 + j);
    cp_async16(nb + (5 + 4 * j) * T, d.c_r2 + c0 + j);
    cp_async16(nb + (6 + 4 * j) * T, d.c_k + c0 + j);
    cp_async16(nb + (7 + 4 * j) * T, d.pgs_lam + c0 + j);
  }
  cp_async16(nb + 20 * T, d.vel + a);
  cp_async16(nb + 21 * T, d.omega + a);
  cp_async16(nb + 22 * T, d.iw + 2 * a);
  cp_async16(nb + 23 * T, d.iw + 2 * a + 1);
  cp_async16(nb + 24 * T, d.vel + b);
  cp_async16(nb + 25 * T, d.omega + b);
  cp_async16(nb + 26 * T, d.iw + 2 * b);
  cp_async16(nb + 27 * T, d.iw + 2 * b + 1);
  cp_async_commit();
}

// the staged item into registers (after cp.async.wait_all); its contacts beyond PF are staged
// in the extra slot as pgs_item_fill does
template <int PF>
__device__ __forceinline__ void pgs_take_next(const DevState& d, uint4 r, PgsItem<PF>& x, PgsBodies& B) {
  const float4* nb = pgs_next_base();
  const uint32_t T = BB_PGS_THREADS, cc = r.w & 0xFFu;
  x.rec = r;
  x.mass = nb[0];
  x.n = nb[T];
  x.t0 = nb[2 * T];
  x.t1 = nb[3 * T];
#pragma unroll
  for (int j = 0; j < PF; ++j) {
    if (uint32_t(j) < cc) {
      x.R1[j] = nb[(4 + 4 * j) * T];
      x.R2[j] = nb[(5 + 4 * j) * T];
      x.K[j] = nb[(6 + 4 * j) * T];
      x.lam[j] = nb[(7 + 4 * j) * T];
    }
  }
  B.va = nb[20 * T];
  B.wa = nb[21 * T];
  B.ia0 = nb[22 * T];
  B.ia1 = nb[23 * T];
  B.vb = nb[24 * T];
  B.wb = nb[25 * T];
  B.ib0 = nb[26 * T];
  B.ib1 = nb[27 * T];
  if (cc > uint32_t(PF)) {
    float4* slot = pgs_extra_slot();
    for (uint32_t j = PF; j < cc; ++j) {
      float4* e = slot + (j - PF) * 4;
      cp_async16(e + 0, d.c_r1 + r.x + j);
      cp_async16(e + 1, d.c_r2 + r.x + j);
      cp_async16(e + 2, d.c_k + r.x + j);
      cp_async16(e + 3, d.pgs_lam + r.x + j);
    }
    cp_async_commit();
  }
}

// one sweep over colours 0..C-1 and the overflow bucket.  On entry x holds this thread's first
// item of colour 0 and rec_next the record of its first item of colour 1 (or of colour 0 when
// C == 1); on exit both are set the same way for the next sweep.  Records run one colour ahead
// of the rest of the item, so the loads issued between barrier arrival and wait never wait on
// an address; and they are issued after this block's arrival, so the arrival's fence does not
// wait for them either.
__device__ __forceinline__ uint32_t pgs_next_colour(uint32_t c, uint32_t C) { return c + 1 < C ? c + 1 : 0u; }

template <int PF, bool STAGE_NEXT>
__device__ void pgs_sweep(const DevState& d, const Params& p, int cur, int mode, const uint32_t* bs, const uint32_t* aw,
                          uint32_t C, PgsItem<PF>& x, uint4& rec_next, uint32_t& epoch) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  uint32_t* sync = &d.ctr->sync_count[1];
  for (uint32_t c = 0; c < C; ++c) {
    // A colour whose manifolds all sleep has no work (every item is skipped) and needs no
    // barrier: its neighbours are ordered by the barriers of the colours that do run.
    const bool run = aw[c] != 0;
    if (run && !STAGE_NEXT) {  // later items of the colour load after the one before has run
      const uint32_t end = bs[c + 1];
      for (uint32_t k = bs[c] + tid; k < end;) {
        pgs_item_run(d, p, cur, x, mode);
        k += stride;
        if (k < end) pgs_item_load(d, k, x);
      }
    } else if (run) {
      // The colour's first item is in x.  Its bodies and the next item's record load now; each
      // later item (with its bodies) is staged by cp.async while the one before computes, and
      // the record after it loads meanwhile, so a later item costs no dependent round trip.
      const uint32_t end = bs[c + 1];
      uint32_t k = bs[c] + tid;
      if (k < end) {
        uint4 rn = make_uint4(0, 0, 0, 0);
        if (k + stride < end) rn = d.pgs_rec[k + stride];
        PgsBodies B = pgs_bodies_load(d, x.rec.y, x.rec.z);
        for (;;) {
          const uint32_t kn = k + stride;
          const bool more = kn < end;
          uint4 rnn = make_uint4(0, 0, 0, 0);
          if (more) {
            pgs_stage_next<PF>(d, kn, rn);
            if (kn + stride < end) rnn = d.pgs_rec[kn + stride];
          }
          pgs_item_compute<PF>(d, p, x, B, mode);
          if (!more) break;
          cp_async_wait_all();
          pgs_take_next<PF>(d, rn, x, B);
          rn = rnn;
          k = kn;
        }
      }
    }
    const uint32_t cn = pgs_next_colour(c, C), cnn = pgs_next_colour(cn, C);
    const uint32_t kn = bs[cn] + tid, knn = bs[cnn] + tid;
    if (!run) {  // keep the prefetch one colour ahead
      if (kn < bs[cn + 1]) pgs_item_load_rest(d, kn, rec_next, x);
      if (knn < bs[cnn + 1]) rec_next = d.pgs_rec[knn];
      continue;
    }
    // This colour and the next one that runs, both fitting in block 0 (items map to threads by
    // their index in the colour), need only a CTA barrier between them: every item and every
    // body write of both lives in block 0.  The test reads shared bucket starts and flags, so
    // every block decides alike.
    uint32_t ne = c + 1;
    while (ne < C && !aw[ne]) ++ne;
    const bool local = ne < C && bs[c + 1] - bs[c] <= blockDim.x && bs[ne + 1] - bs[ne] <= blockDim.x;
    if (!local) grid_arrive(sync, epoch);
    if (kn < bs[cn + 1]) pgs_item_load_rest(d, kn, rec_next, x);
    if (knn < bs[cnn + 1]) rec_next = d.pgs_rec[knn];
    if (local) __syncthreads();
    else grid_wait(d.ctr, sync, epoch);
  }
  const uint32_t o0 = bs[BB_MAX_COLORS], o1 = bs[BB_MAX_COLORS + 1];
  if (o0 != o1) {  // overflow bucket: serial, in manifold order
    if (tid == 0) {
      for (uint32_t k = o0; k < o1; ++k) {
        PgsItem<PF> y;
        pgs_item_load<PF, false>(d, k, y);
        pgs_item_run<PF, false>(d, p, cur, y, mode);
      }
    }
    grid_sync(d.ctr, sync, epoch);
  }
}

// PF = 4 contacts held per item (one 255-register block per SM).  Holding fewer would let
// two blocks share an SM but puts the other contacts' loads on the critical path, one round
// trip each.  A streaming variant that held nothing across barriers (each item's contacts
// copied to shared memory by cp.async while its bodies load) ran 2 or 3 blocks per SM and
// measured slower on the 1M-box pyramids (solve 3.32 and 6.55 against 3.23 ms per substep).
template <int PF, bool STAGE_NEXT>
__global__ void __launch_bounds__(BB_PGS_THREADS, PF == 4 ? 1 : 2) k_pgs_soft(const DevState d, Params p, int cur, uint32_t n, float h) {
  __shared__ uint32_t bs[BB_MAX_COLORS + 2];
  __shared__ uint32_t aw[BB_MAX_COLORS + 1];
  // test switch (bb_debug_wait_limit): the last block leaves, so the others' first grid barrier
  // waits for a block that never arrives until its bounded wait gives up
  if (gridDim.x > 1 && blockIdx.x == gridDim.x - 1 && d.ctr->abandon_block) return;
  if (threadIdx.x < BB_MAX_COLORS + 2) bs[threadIdx.x] = d.bucket_start[threadIdx.x];
  if (threadIdx.x < BB_MAX_COLORS + 1) aw[threadIdx.x] = d.colour_awake[threadIdx.x];
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  const bool tq = p.quirks & BB_QUIRK_INERTIA_TRANSPOSE;
  uint32_t* sync = &d.ctr->sync_count[1];
  uint32_t epoch = 0;
  // the world inverse inertias and the items' records and rows were written by k_pgs_inertia
  // and k_pgs_build before this launch
  __syncthreads();  // bs and aw
  const uint32_t C = d.ctr->gc_colors;
  PgsItem<PF> x;
  uint4 rec_next = make_uint4(0, 0, 0, 0);
  if (C > 0 && bs[0] + tid < bs[1]) pgs_item_load(d, bs[0] + tid, x);
  if (C > 0) {
    const uint32_t c1 = pgs_next_colour(0, C);
    if (bs[c1] + tid < bs[c1 + 1]) rec_next = d.pgs_rec[bs[c1] + tid];
  }
  pgs_sweep<PF, STAGE_NEXT>(d, p, cur, 0, bs, aw, C, x, rec_next, epoch);
  for (uint32_t it = 0; it < p.iterations; ++it) pgs_sweep<PF, STAGE_NEXT>(d, p, cur, 1, bs, aw, C, x, rec_next, epoch);
  if (p.flags & BB_SIM_ADVECTION) {
    for (uint32_t i = tid; i < n; i += stride)
      if (awake(d.flags[i])) pgs_integrate(d, i, h, tq);
    grid_sync(d.ctr, sync, epoch);
  }
  for (uint32_t it = 0; it < p.relax_iterations; ++it) pgs_sweep<PF, STAGE_NEXT>(d, p, cur, 2, bs, aw, C, x, rec_next, epoch);
  // k_pgs_writeback copies the impulses back to the persistent contacts after this launch
}

// Before k_pgs_soft, at full occupancy (the persistent kernel runs one 256-thread block per
// SM, where these passes of one item or body per thread were latency-bound): the world
// inverse inertias, then the records and rows of every swept item (colours and the overflow
// bucket, [0, bucket_start[33])).  After it, the impulses back to the persistent contacts.
__global__ void k_pgs_inertia(const DevState d, uint32_t n, Params p) {
  const bool tq = p.quirks & BB_QUIRK_INERTIA_TRANSPOSE;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) pgs_world_inertia(d, i, tq);
}
__global__ void k_pgs_build(const DevState d, Params p, int cur, float h) {
  const float inv_h = h > 0.f ? 1.0f / h : 0.f;
  const float hertz = fminf(p.contact_hertz, inv_h * 0.3333333333333333f);
  const uint32_t end = d.bucket_start[BB_MAX_COLORS + 1];
  const uint32_t* list = d.bucket_vals[1];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < end; k += gridDim.x * blockDim.x)
    pgs_item_build(d, cur, k, list[k], h, hertz);
}
__global__ void k_pgs_writeback(const DevState d, int cur) {
  const uint32_t M = d.ctr->manifold_count;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < M; k += gridDim.x * blockDim.x) {
    const uint32_t cc = d.pgs_cnt[k];
    if (cc == 0) continue;
    const uint32_t slot = d.pgs_slot[k], c0 = d.pgs_coff[k];
    for (uint32_t j = 0; j < cc; ++j) d.c_lam[cur][slot * BB_MAX_CONTACTS + j] = d.pgs_lam[c0 + j];
  }
}



// ---------------------------------------------------------------------------------------
// PGS_SOFT, dataflow schedule.
//
// The per-colour sweeps give every body b the ordered sequence L_b of the manifolds touching
// it, sorted by (colour, manifold) with the overflow bucket last; one sweep processes L_b in
// that order, and a manifold's result depends only on its two bodies' states.  So instead of a
// grid barrier after each colour, each dynamic body carries a sequence counter: item k of sweep
// s waits until counter[b] == s * deg(b) + rank_b(k) for both its dynamic bodies, runs, and
// releases +1 on each.  The outcome is bit-identical to the barrier schedule.
//
// The kernel is cooperative (all blocks resident) and thread t owns the items k = t, t + T, ...
// of the colour-ordered list, which it runs in increasing (sweep, k) order.  Every wait points
// at an item earlier in that order, owned by a thread that reaches it without waiting on a
// later item of t, so the schedule cannot deadlock.  The items are the barrier schedule's
// compact records (built by their owners), so a thread loads its next item while waiting.
__device__ __forceinline__ void red_release_add(uint32_t* p, uint32_t v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void flow_wait(DevCounters* c, const uint32_t* ctr, uint32_t target) {
  uint32_t spins = 0;
  while (ld_acquire_gpu(ctr) < target)
    if (spin_gave_up(c, ++spins, BB_SITE_FLOW)) return;
}

// per colour-ordered item k: (rank_a | rank_b << 16, deg_a | deg_b << 16) where rank_x is the
// item's position in L_x (colour-major, then manifold order) and deg_x = |L_x|
__global__ void k_flow_prep(const DevState d, int cur) {
  const uint32_t M = d.ctr->manifold_count;
  const uint32_t* list = d.bucket_vals[1];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < M; k += gridDim.x * blockDim.x) {
    const uint32_t m = list[k];
    const uint2 b = d.m_bodies[cur][d.man_slot[cur][m]];
    const uint32_t cm = min(d.gc_color[m], uint32_t(BB_MAX_COLORS));
    uint32_t rank[2] = {0, 0}, deg[2] = {0, 0};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const uint32_t x = q == 0 ? b.x : b.y;
      if (!(d.flags[x] & BB_BODY_DYNAMIC)) continue;
      const uint32_t s0 = d.csr_start[cur][x], s1 = d.csr_start[cur][x + 1];
      uint32_t r = 0;
      for (uint32_t e = s0; e < s1; ++e) {
        const uint32_t m2 = d.csr_list[cur][e];
        const uint32_t c2 = min(d.gc_color[m2], uint32_t(BB_MAX_COLORS));
        r += (c2 < cm || (c2 == cm && m2 < m)) ? 1u : 0u;
      }
      rank[q] = r;
      deg[q] = s1 - s0;
    }
    d.flow_rec[k] = make_uint4((rank[0] & 0xFFFFu) | (rank[1] << 16), (deg[0] & 0xFFFFu) | (deg[1] << 16), 0u, 0u);
  }
}

// world inverse inertia cache and zeroed sequence counters
__global__ void k_flow_init(const DevState d, Params p, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  pgs_world_inertia(d, i, p.quirks & BB_QUIRK_INERTIA_TRANSPOSE);
  d.flow_counter[i] = 0;
}

// one dataflow sweep s (mode 0 warm start, 1 solve, 2 relax) over this thread's items
template <int PF>
__device__ void flow_sweep(const DevState& d, const Params& p, int cur, uint32_t s, int mode, uint32_t M, PgsItem<PF>& x,
                           uint4& fr) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (uint32_t k = tid; k < M; k += stride) {
    const uint32_t a = x.rec.y, b = x.rec.z;
    const bool da = x.rec.w & (1u << 8), db = x.rec.w & (1u << 9);
    if (da) flow_wait(d.ctr, &d.flow_counter[a], s * (fr.y & 0xFFFFu) + (fr.x & 0xFFFFu));
    if (db) flow_wait(d.ctr, &d.flow_counter[b], s * (fr.y >> 16) + (fr.x >> 16));
    pgs_item_run(d, p, cur, x, mode);
    if (da) red_release_add(&d.flow_counter[a], 1u);
    if (db) red_release_add(&d.flow_counter[b], 1u);
    // this thread's next item (wrapping to its first for the next sweep)
    const uint32_t kn = k + stride < M ? k + stride : tid;
    pgs_item_load(d, kn, x);
    fr = d.flow_rec[kn];
  }
}

template <int PF>
__global__ void __launch_bounds__(BB_PGS_THREADS, PF == 4 ? 1 : 2) k_pgs_flow(const DevState d, Params p, int cur,
                                                                               uint32_t n, float h) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  const bool tq = p.quirks & BB_QUIRK_INERTIA_TRANSPOSE;
  const float inv_h = h > 0.f ? 1.0f / h : 0.f;
  const float hertz = fminf(p.contact_hertz, inv_h * 0.3333333333333333f);
  uint32_t* sync = &d.ctr->sync_count[1];
  uint32_t epoch = 0;
  const uint32_t M = d.ctr->manifold_count;
  const uint32_t* list = d.bucket_vals[1];
  for (uint32_t k = tid; k < M; k += stride) pgs_item_build(d, cur, k, list[k], h, hertz);
  PgsItem<PF> x;
  uint4 fr = make_uint4(0, 0, 0, 0);
  if (tid < M) {
    pgs_item_load(d, tid, x);
    fr = d.flow_rec[tid];
  }
  uint32_t s = 0;
  flow_sweep(d, p, cur, s++, 0, M, x, fr);
  for (uint32_t it = 0; it < p.iterations; ++it) flow_sweep(d, p, cur, s++, 1, M, x, fr);
  if (p.flags & BB_SIM_ADVECTION) {
    grid_sync(d.ctr, sync, epoch);
    for (uint32_t i = tid; i < n; i += stride)
      if (awake(d.flags[i])) pgs_integrate(d, i, h, tq);
    grid_sync(d.ctr, sync, epoch);
  }
  for (uint32_t it = 0; it < p.relax_iterations; ++it) flow_sweep(d, p, cur, s++, 2, M, x, fr);
  grid_sync(d.ctr, sync, epoch);
  for (uint32_t k = tid; k < M; k += stride) {  // impulses back to the persistent contacts
    const uint32_t cc = d.pgs_cnt[k];
    if (cc == 0) continue;
    const uint32_t slot = d.pgs_slot[k], c0 = d.pgs_coff[k];
    for (uint32_t j = 0; j < cc; ++j) d.c_lam[cur][slot * BB_MAX_CONTACTS + j] = d.pgs_lam[c0 + j];
  }
}

int bb_pgs_soft_blocks(int sms) {
  cudaFuncSetAttribute((const void*)k_pgs_soft<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, BB_PGS_SMEM_EXTRA);
  cudaFuncSetAttribute((const void*)k_pgs_soft<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, BB_PGS_SMEM);
  cudaFuncSetAttribute((const void*)k_pgs_flow<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, BB_PGS_SMEM_EXTRA);
  return bb_coop_blocks((const void*)k_pgs_soft<4, false>, BB_PGS_THREADS, sms);
}

void bb_solve_pgs_soft(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, float h, int cur,
                       const StepScratch& sc, int coop_blocks, int sms) {
  cudaMemsetAsync(d.colour_awake, 0, sizeof(uint32_t) * (BB_MAX_COLORS + 1), s);
  k_pgs_count<<<sms * 8, BB_THREADS, 0, s>>>(d, cur);
  bb_launch_scan(s, d.pgs_cnt, d.pgs_coff, &d.ctr->manifold_count, d.pair_capacity, &d.ctr->pgs_contacts,
                 sc.scan_status + 4 * size_t(sc.scan_tiles), sc.scan_tile_ctr + 4, d.ctr);
  if (p.schedule == BB_SCHEDULE_DATAFLOW) {
    k_flow_prep<<<sms * 8, BB_THREADS, 0, s>>>(d, cur);
    k_flow_init<<<(n + BB_THREADS - 1) / BB_THREADS, BB_THREADS, 0, s>>>(d, p, n);
    DevState dd = d;
    Params pp = p;
    int cc = cur;
    uint32_t nn = n;
    float hh = h;
    void* args[] = {&dd, &pp, &cc, &nn, &hh};
    const void* kern = (const void*)k_pgs_flow<4>;
    bb_launch_coop(kern, coop_blocks, BB_PGS_THREADS, args, s, BB_PGS_SMEM_EXTRA);
    return;
  }
  DevState dd = d;
  Params pp = p;
  int cc = cur;
  uint32_t nn = n;
  float hh = h;
  void* args[] = {&dd, &pp, &cc, &nn, &hh};
  if (n) k_pgs_inertia<<<(n + BB_THREADS - 1) / BB_THREADS, BB_THREADS, 0, s>>>(d, n, p);
  k_pgs_build<<<sms * 8, BB_THREADS, 0, s>>>(d, p, cur, h);
  // staging the next item needs 112 KB more shared memory (less L1): it pays when threads run
  // several items per colour (large worlds), which is what the autotuner measures
  if (p.pgs_stage_next)
    bb_launch_coop((const void*)k_pgs_soft<4, true>, coop_blocks, BB_PGS_THREADS, args, s, BB_PGS_SMEM);
  else bb_launch_coop((const void*)k_pgs_soft<4, false>, coop_blocks, BB_PGS_THREADS, args, s, BB_PGS_SMEM_EXTRA);
  k_pgs_writeback<<<sms * 8, BB_THREADS, 0, s>>>(d, cur);
}

// ---------------------------------------------------------------------------------------
// Per-island path (USE_GRAPH_COLORING off, RBM:1390-1399; RB_sim.slang:1122-1406): one thread
// per contact island runs the island's manifolds serially, in manifold order -- PGS_SOFT's
// pre-step and solve sweeps, or the Baumgarte PGS of solvers.slang:3-136 -- then all bodies
// integrate, then (PGS_SOFT only) the relax sweeps run per island again.  Manifolds are grouped
// by island with a stable sort keyed by the island id of their dynamic body.

// PGS::pre_step (solvers.slang:3-66) of one manifold slot
__device__ void baum_pre_step_slot(const DevState& d, const Params& p, int cur, uint32_t slot, uint2 b, float inv_h) {
  const uint32_t fa = d.flags[b.x], fb = d.flags[b.y];
  if (!awake(fa) && !awake(fb)) return;
  const float ima = d.pos[b.x].w, imb = d.pos[b.y].w;
  const Sym3 IA = load_iw(d, b.x), IB = load_iw(d, b.y);
  float3 va = f3(d.vel[b.x]), wa = f3(d.omega[b.x]), vb = f3(d.vel[b.y]), wb = f3(d.omega[b.y]);
  const float3 n = f3(d.m_normal[cur][slot]);
  const float3 t0 = f3(d.m_t0[cur][slot]), t1 = f3(d.m_t1[cur][slot]);
  const float3 pa = f3(d.pos[b.x]), pb = f3(d.pos[b.y]);
  const int cc = d.m_keycc[cur][slot].y;
  const bool accum = p.flags & BB_SIM_ACCUM_IMPULSE, fric = p.flags & BB_SIM_FRICTION;
  for (int j = 0; j < cc; ++j) {
    const uint32_t ci = slot * BB_MAX_CONTACTS + j;
    const float4 pp = d.c_pos[cur][ci];
    const float3 r1 = xsub(f3(pp), pa), r2 = xsub(f3(pp), pb);
    const float nmass = xrow_mass(r1, r2, n, ima, imb, IA, IB);
    const float tm0 = xrow_mass(r1, r2, t0, ima, imb, IA, IB), tm1 = xrow_mass(r1, r2, t1, ima, imb, IA, IB);
    const float bias = -0.2f * inv_h * fminf(pp.w + 0.01f, 0.f);
    d.c_r1[ci] = f4(r1, nmass);
    d.c_r2[ci] = f4(r2, tm0);
    d.c_k[ci] = make_float4(tm1, bias, 0.f, 0.f);
    const float4 lam = d.c_lam[cur][ci];
    if (accum) pgs_contact_warm(r1, r2, lam, n, t0, t1, fric, ima, imb, IA, IB, va, wa, vb, wb);
  }
  if (fa & BB_BODY_DYNAMIC) {
    d.vel[b.x] = f4(va, d.vel[b.x].w);
    d.omega[b.x] = f4(wa, 0.f);
  }
  if (fb & BB_BODY_DYNAMIC) {
    d.vel[b.y] = f4(vb, d.vel[b.y].w);
    d.omega[b.y] = f4(wb, 0.f);
  }
}

// PGS::solve (solvers.slang:68-136) of one manifold slot
__device__ void baum_solve_slot(const DevState& d, const Params& p, int cur, uint32_t slot, uint2 b) {
  const uint32_t fa = d.flags[b.x], fb = d.flags[b.y];
  if (!awake(fa) && !awake(fb)) return;
  const float ima = d.pos[b.x].w, imb = d.pos[b.y].w;
  const Sym3 IA = load_iw(d, b.x), IB = load_iw(d, b.y);
  float4 va4 = d.vel[b.x], vb4 = d.vel[b.y];
  float3 va = f3(va4), wa = f3(d.omega[b.x]), vb = f3(vb4), wb = f3(d.omega[b.y]);
  const float mu = sqrtf(d.iinv[b.x].w * d.iinv[b.y].w);
  const float3 n = f3(d.m_normal[cur][slot]);
  const float3 t0 = f3(d.m_t0[cur][slot]), t1 = f3(d.m_t1[cur][slot]);
  const int cc = d.m_keycc[cur][slot].y;
  const bool accum = p.flags & BB_SIM_ACCUM_IMPULSE, fric = p.flags & BB_SIM_FRICTION;
  for (int j = 0; j < cc; ++j) {
    const uint32_t ci = slot * BB_MAX_CONTACTS + j;
    const float4 R1 = d.c_r1[ci], R2 = d.c_r2[ci], K = d.c_k[ci];
    float4 lam = d.c_lam[cur][ci];
    const float3 r1 = f3(R1), r2 = f3(R2);
    if (fric) {
      const float3 rv = xrel(r1, r2, va, wa, vb, wb);
      const float tmass[2] = {R2.w, K.x};
      float imp_t[2] = {lam.y, lam.z};
      const float maxf = mu * lam.x;
      for (int k = 0; k < 2; ++k) {
        const float3 t = k == 0 ? t0 : t1;
        float ti = tmass[k] * -xdot(rv, t);
        if (accum) {
          const float old = imp_t[k];
          imp_t[k] = fminf(fmaxf(old + ti, -maxf), maxf);
          ti = imp_t[k] - old;
        } else {
          ti = fminf(fmaxf(ti, -maxf), maxf);
        }
        xapply(xscale(t, ti), r1, r2, ima, imb, IA, IB, va, wa, vb, wb);
      }
      lam.y = imp_t[0];
      lam.z = imp_t[1];
    }
    float imp = R1.w * (K.y - xdot(xrel(r1, r2, va, wa, vb, wb), n));
    if (accum) {
      const float old = lam.x;
      lam.x = fmaxf(old + imp, 0.f);
      imp = lam.x - old;
    } else {
      imp = fmaxf(imp, 0.f);
    }
    xapply(xscale(n, imp), r1, r2, ima, imb, IA, IB, va, wa, vb, wb);
    d.c_lam[cur][ci] = lam;
  }
  if (fa & BB_BODY_DYNAMIC) {
    d.vel[b.x] = f4(va, va4.w);
    d.omega[b.x] = f4(wa, 0.f);
  }
  if (fb & BB_BODY_DYNAMIC) {
    d.vel[b.y] = f4(vb, vb4.w);
    d.omega[b.y] = f4(wb, 0.f);
  }
}

// key of every manifold: the island of its dynamic body
__global__ void k_island_keys(const DevState d, int cur) {
  const uint32_t M = d.ctr->manifold_count;
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    const uint2 b = d.m_bodies[cur][d.man_slot[cur][m]];
    const uint32_t ia = d.island[b.x];
    d.bucket_keys[0][m] = ia != BB_NONE ? ia : d.island[b.y];
    d.bucket_vals[0][m] = m;
  }
}
// island_start[v] = first sorted position with key >= v, v = 0..island_count
__global__ void k_island_starts(const DevState d, uint32_t* starts, uint32_t n) {
  const uint32_t M = d.ctr->manifold_count, nb = d.ctr->island_count;
  const uint32_t* keys = d.bucket_keys[1];
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= nb && v <= n; v += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = M;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (keys[mid] < v) lo = mid + 1;
      else hi = mid;
    }
    starts[v] = lo;
  }
}
// phase 0: pre-step + solve sweeps; phase 1: relax sweeps (PGS_SOFT)
__global__ void k_island_solve(const DevState d, Params p, int cur, const uint32_t* starts, float h, int phase) {
  const uint32_t nb = d.ctr->island_count;
  const uint32_t* list = d.bucket_vals[1];
  const float inv_h = h > 0.f ? 1.0f / h : 0.f;
  const float hertz = fminf(p.contact_hertz, inv_h * 0.3333333333333333f);
  const bool soft = p.solver == BB_SOLVER_PGS_SOFT;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nb; v += gridDim.x * blockDim.x) {
    const uint32_t s0 = starts[v], s1 = starts[v + 1];
    auto each = [&](auto&& fn) {
      for (uint32_t k = s0; k < s1; ++k) {
        const uint32_t slot = d.man_slot[cur][list[k]];
        fn(slot, d.m_bodies[cur][slot]);
      }
    };
    if (phase == 0) {
      each([&](uint32_t slot, uint2 b) {
        if (soft) pgs_pre_step_slot(d, p, cur, slot, b, h, hertz);
        else baum_pre_step_slot(d, p, cur, slot, b, inv_h);
      });
      for (uint32_t it = 0; it < p.iterations; ++it)
        each([&](uint32_t slot, uint2 b) {
          if (soft) pgs_solve_slot(d, p, cur, slot, b, true);
          else baum_solve_slot(d, p, cur, slot, b);
        });
    } else {
      for (uint32_t it = 0; it < p.relax_iterations; ++it)
        each([&](uint32_t slot, uint2 b) { pgs_solve_slot(d, p, cur, slot, b, false); });
    }
  }
}
__global__ void k_island_integrate(const DevState d, Params p, uint32_t n, float h) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && awake(d.flags[i])) pgs_integrate(d, i, h, p.quirks & BB_QUIRK_INERTIA_TRANSPOSE);
}

void bb_solve_islands(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, float h, int cur,
                      const StepScratch& sc, int sms) {
  if (n == 0) return;
  const int T = BB_THREADS;
  const uint32_t blocks = (n + T - 1) / T;
  k_flow_init<<<blocks, T, 0, s>>>(d, p, n);  // world inverse inertia of every body
  k_island_keys<<<sms * 8, T, 0, s>>>(d, cur);
  uint32_t* keys[2] = {d.bucket_keys[0], d.bucket_keys[1]};
  uint32_t* vals[2] = {d.bucket_vals[0], d.bucket_vals[1]};
  // 3 digits (islands < 2^24): histogram region 1 and status slots 6..8 (the colouring's, unused here)
  uint32_t* hist = sc.sort_hist + 1 * BB_HIST_REGION;
  bb_launch_sort(s, keys, vals, &d.ctr->manifold_count, d.pair_capacity, 3, 0, hist,
                 sc.sort_status + 6 * size_t(sc.sort_tiles) * 256, sc.sort_tile_ctr + 6, d.ctr, sms);
  k_island_starts<<<(n + 1 + T - 1) / T, T, 0, s>>>(d, d.island_start, n);
  k_island_solve<<<(n + 127) / 128, 128, 0, s>>>(d, p, cur, d.island_start, h, 0);
  if (p.flags & BB_SIM_ADVECTION) k_island_integrate<<<blocks, T, 0, s>>>(d, p, n, h);
  if (p.solver == BB_SOLVER_PGS_SOFT) k_island_solve<<<(n + 127) / 128, 128, 0, s>>>(d, p, cur, d.island_start, h, 1);
}

// ---------------------------------------------------------------------------------------
// AVBD
__device__ __forceinline__ uint32_t avbd_priority(uint32_t body, uint32_t round) {
  uint32_t x = body * 0x9e3779b9u + round * 0x85ebca6bu;
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return ((x & 0xFFFu) << 20) | (body & 0xFFFFFu);
}
__device__ __forceinline__ float3 small_angle_delta(Quatf now, Quatf start) {
  Quatf dq = q_mul(now, q_conj(start));
  float sg = dq.w < 0.f ? -1.f : 1.f;
  return make_float3(dq.x, dq.y, dq.z) * (2.0f * sg);
}
__device__ __forceinline__ float3 avbd_q_rotate(Quatf q, float3 u) {
  float3 qv = make_float3(q.x, q.y, q.z);
  return u + 2.0f * cross3(qv, cross3(qv, u) + u * q.w);
}

// Jones-Plassmann colouring with start-of-round semantics: body_color holds
// ((round + 1) << 8) | colour while the kernel runs, so a neighbour coloured in the current
// round still counts as uncoloured.
__global__ void __launch_bounds__(BB_COOP_THREADS, 1) k_avbd_color(const DevState d, Params p, int cur, uint32_t n) {
  DevCounters* c = d.ctr;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  uint32_t* uncol = c->round_flags;
  uint32_t* sync = &c->sync_count[2];
  uint32_t ep = 0;
  for (uint32_t i = tid; i < n; i += stride) d.body_color[i] = BB_UNCOLORED;
  if (tid == 0) {
    uncol[0] = 0;
    uncol[1] = 0;
    c->avbd_colors = 0;
  }
  grid_sync(c, sync, ep);
  for (uint32_t rd = 0; rd < p.avbd_color_rounds; ++rd) {
    uint32_t left = 0;
    for (uint32_t i = tid; i < n; i += stride) {
      if (d.body_color[i] != BB_UNCOLORED || !(d.flags[i] & BB_BODY_DYNAMIC)) continue;
      const uint32_t mine = avbd_priority(local_id(d, i), rd);
      uint32_t used = 0;
      bool wait = false;
      const uint32_t s0 = d.csr_start[cur][i], s1 = d.csr_start[cur][i + 1];
      for (uint32_t e = s0; e < s1 && !wait; ++e) {
        const uint32_t q = d.csr_partner[cur][e];
        if (q == i || !(d.flags[q] & BB_BODY_DYNAMIC)) continue;
        uint32_t pc = *(volatile uint32_t*)&d.body_color[q];
        bool unc = pc == BB_UNCOLORED || (pc >> 8) == rd + 1u;
        if (unc) {
          if (avbd_priority(local_id(d, q), rd) > mine) wait = true;
        } else {
          used |= 1u << (pc & 255u);
        }
      }
      if (wait || used == 0xFFFFFFFFu) {
        ++left;
        continue;
      }
      uint32_t col = uint32_t(__ffs(~used) - 1);
      d.body_color[i] = ((rd + 1u) << 8) | col;
      atomicMax(&c->avbd_colors, col + 1u);
    }
    if (left) atomicAdd(&uncol[rd & 1], left);
    grid_sync(c, sync, ep);
    if (*(volatile uint32_t*)&uncol[rd & 1] == 0u) break;
    if (tid == 0) uncol[(rd + 1) & 1] = 0;
    grid_sync(c, sync, ep);
  }
  for (uint32_t i = tid; i < n; i += stride) {
    uint32_t v = d.body_color[i];
    d.body_color[i] = v == BB_UNCOLORED ? BB_UNCOLORED : (v & 255u);
  }
}

__global__ void k_avbd_prepare(const DevState d, Params p, uint32_t n, float dt) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t f = d.flags[i];
  if (!awake(f)) return;
  float3 w = f3(d.omega[i]);
  float om = len3(w);
  if (om > 50.0f) {
    w = w * (50.0f / om);
    d.omega[i] = f4(w, 0.f);
  }
  float grav = (f & BB_BODY_GRAVITY) ? p.gravity : 0.f;
  float4 ps = d.pos[i];
  float3 pos = f3(ps), v = f3(d.vel[i]);
  Quatf q = q_from(d.rot[i]);
  d.a_pos_start[i] = f4(pos, 0.f);
  d.a_rot_start[i] = q_to4(q);
  d.a_pos_tilde[i] = f4(pos + v * dt + make_float3(0.f, grav, 0.f) * (dt * dt), 0.f);
  Quatf qt = apply_angular_velocity(q, w, dt);
  d.a_rot_tilde[i] = q_to4(qt);
  float aw = 0.f;
  if (fabsf(grav) > 1e-6f) {
    float ay = (v.y - d.pvel[i].y) / dt;
    float sg = grav > 0.f ? 1.f : -1.f;
    aw = fminf(fmaxf(ay * sg / fabsf(grav), 0.f), 1.f);
  }
  d.pos[i] = f4(pos + v * dt + make_float3(0.f, grav, 0.f) * (aw * dt * dt), ps.w);
  d.rot[i] = q_to4(qt);
}

__global__ void k_avbd_warmstart(const DevState d, Params p, int cur) {
  const uint32_t M = d.ctr->manifold_count;
  const bool warm = p.flags & BB_SIM_WARM_STARTING;
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    const uint32_t slot = d.man_slot[cur][m];
    const uint2 b = d.m_bodies[cur][slot];
    const uint32_t fa = d.flags[b.x], fb = d.flags[b.y];
    // a paused world's manifolds are carried unchanged (no penalty decay, no new anchors), so
    // the world resumes exactly as it stopped
    if ((fa | fb) & BB_BODY_PAUSED) continue;
    bool d1 = awake(fa), d2 = awake(fb);
    float3 c1 = d1 ? f3(d.a_pos_start[b.x]) : f3(d.pos[b.x]);
    float3 c2 = d2 ? f3(d.a_pos_start[b.y]) : f3(d.pos[b.y]);
    Quatf q1c = q_conj(d1 ? q_from(d.a_rot_start[b.x]) : q_from(d.rot[b.x]));
    Quatf q2c = q_conj(d2 ? q_from(d.a_rot_start[b.y]) : q_from(d.rot[b.y]));
    const int cc = d.m_keycc[cur][slot].y;
    uint32_t sticks = 0;
    for (int j = 0; j < cc; ++j) {
      const uint32_t ci = slot * BB_MAX_CONTACTS + j;
      float4 lam = d.c_lam[cur][ci];
      float4 kt = d.c_kt[cur][ci];
      uint32_t wcount = __float_as_uint(kt.w), stick = __float_as_uint(kt.z);
      bool matched = wcount != 0u && warm;
      if (!matched) {
        lam = make_float4(0.f, 0.f, 0.f, p.avbd_k_min);
        kt.x = kt.y = p.avbd_k_min;
        stick = 0;
      } else {
        lam.w = fminf(fmaxf(lam.w * p.avbd_gamma, p.avbd_k_min), p.avbd_k_max);
        lam.x = fminf(lam.x, 0.f);
        kt.x = fminf(fmaxf(kt.x * p.avbd_gamma, p.avbd_k_min), p.avbd_k_max);
        kt.y = fminf(fmaxf(kt.y * p.avbd_gamma, p.avbd_k_min), p.avbd_k_max);
      }
      bool sticking = matched && stick != 0u;
      if (!sticking) {
        float4 cp = d.c_pos[cur][ci];
        float4 aa = d.c_anc_a[cur][ci];
        d.c_anc_a[cur][ci] = f4(avbd_q_rotate(q1c, f3(cp) - c1), aa.w);
        d.c_anc_b[cur][ci] = f4(avbd_q_rotate(q2c, f3(cp) - c2), 0.f);
      } else {
        ++sticks;
      }
      d.c_lam[cur][ci] = lam;
      d.c_kt[cur][ci] = make_float4(kt.x, kt.y, __uint_as_float(stick), kt.w);
    }
    if (sticks) atomicAdd(&d.ctr->stick, sticks);
  }
}

__global__ void k_avbd_depth_reset(const DevState d, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  d.a_depth[i] = awake(d.flags[i]) ? BB_NONE : 0u;
}
__global__ void k_avbd_depth_relax(const DevState d, int cur) {
  const uint32_t M = d.ctr->manifold_count;
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    const uint32_t slot = d.man_slot[cur][m];
    if (d.m_keycc[cur][slot].y <= 0) continue;
    const uint2 b = d.m_bodies[cur][slot];
    uint32_t d1 = *(volatile uint32_t*)&d.a_depth[b.x], d2 = *(volatile uint32_t*)&d.a_depth[b.y];
    if (d2 != BB_NONE && d2 + 1u < d1) atomicMin(&d.a_depth[b.x], d2 + 1u);
    if (d1 != BB_NONE && d1 + 1u < d2) atomicMin(&d.a_depth[b.y], d1 + 1u);
  }
}

// bucket keys of awake coloured bodies: pass 0 = colour (main sweeps),
// pass 1 = min(depth, L-1) * 32 + colour (post-stabilisation cascade); others sort last
__global__ void k_avbd_keys(const DevState d, Params p, uint32_t n, int post) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t col = d.body_color[i];
  uint32_t key = 0xFFFFu;
  if (awake(d.flags[i]) && col < BB_MAX_COLORS) {
    if (post) {
      uint32_t layer = min(d.a_depth[i], p.avbd_shock_layers - 1u);
      key = layer * BB_MAX_COLORS + col;
    } else {
      key = col;
    }
  }
  d.a_bucket_keys[0][i] = key;
  d.a_bucket_vals[0][i] = i;
}
// starts[v] = first sorted position with key >= v, for v in [0, nb]
__global__ void k_lower_bounds(const uint32_t* keys, uint32_t n, uint32_t* starts, uint32_t nb) {
  uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v > nb) return;
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (keys[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  starts[v] = lo;
}

struct AvbdCtx {
  float dt;
};

__device__ float avbd_contact_C(const DevState& d, const Params& p, int cur, uint32_t slot, uint32_t ci, uint2 b,
                                bool d1, bool d2, float alpha, float3 n, float3& rr1, float3& rr2) {
  float4 cp = d.c_pos[cur][ci];
  float3 c1 = d1 ? f3(d.a_pos_start[b.x]) : f3(d.pos[b.x]);
  float3 c2 = d2 ? f3(d.a_pos_start[b.y]) : f3(d.pos[b.y]);
  rr1 = f3(cp) - c1;
  rr2 = f3(cp) - c2;
  float C = (cp.w + p.avbd_margin) * (1.0f - alpha);
  if (d1) {
    float3 dp = f3(d.pos[b.x]) - c1;
    float3 dth = small_angle_delta(q_from(d.rot[b.x]), q_from(d.a_rot_start[b.x]));
    C -= dot3(n, dp + cross3(dth, rr1));
  }
  if (d2) {
    float3 dp = f3(d.pos[b.y]) - c2;
    float3 dth = small_angle_delta(q_from(d.rot[b.y]), q_from(d.a_rot_start[b.y]));
    C += dot3(n, dp + cross3(dth, rr2));
  }
  (void)slot;
  return C;
}

__device__ float avbd_dir_C(const DevState& d, const Params& p, int cur, uint32_t ci, uint2 b, bool d1, bool d2,
                            float alpha, float3 dir, float3& ar1, float3& ar2, float& C0t) {
  float3 c1 = d1 ? f3(d.a_pos_start[b.x]) : f3(d.pos[b.x]);
  float3 c2 = d2 ? f3(d.a_pos_start[b.y]) : f3(d.pos[b.y]);
  Quatf q1 = d1 ? q_from(d.a_rot_start[b.x]) : q_from(d.rot[b.x]);
  Quatf q2 = d2 ? q_from(d.a_rot_start[b.y]) : q_from(d.rot[b.y]);
  ar1 = avbd_q_rotate(q1, f3(d.c_anc_a[cur][ci]));
  ar2 = avbd_q_rotate(q2, f3(d.c_anc_b[cur][ci]));
  C0t = dot3(dir, (c2 + ar2) - (c1 + ar1));
  float sg = C0t > 0.f ? 1.f : (C0t < 0.f ? -1.f : 0.f);
  float c0e = sg * fmaxf(0.f, fabsf(C0t) - p.avbd_stick_slop);
  float C = c0e * (1.0f - alpha);
  if (d1) {
    float3 dp = f3(d.pos[b.x]) - c1;
    float3 dth = small_angle_delta(q_from(d.rot[b.x]), q_from(d.a_rot_start[b.x]));
    C -= dot3(dir, dp + cross3(dth, ar1));
  }
  if (d2) {
    float3 dp = f3(d.pos[b.y]) - c2;
    float3 dth = small_angle_delta(q_from(d.rot[b.y]), q_from(d.a_rot_start[b.y]));
    C += dot3(dir, dp + cross3(dth, ar2));
  }
  return C;
}

// entry_avbd_primal (avbd.slang:478-658): Gauss-Newton step of body i on its 6 DoF.
// A group of AVBD_LANES lanes per body.  Lane l of the group takes manifolds l, l + AVBD_LANES, ...
// of the body's list and sums their contacts' gradient and Hessian terms in order; a butterfly
// over the group adds the lanes' sums (a fixed order, so the result does not depend on
// scheduling or on which bodies share a warp; it differs from a serial sum in the last bits),
// and the group's lane 0 adds the inertial terms, solves the 6x6 system and moves the body.
// Serially, a body's whole contact loop was one dependent chain per colour step (a box in a
// pile: 15-30 us); a warp per body cut the chain but left too few bodies in flight where a
// colour holds tens of thousands of them.  i == BB_NONE: the group only takes part in the
// shuffles (the trips over a colour's bodies are warp-uniform).
// H is kept as its lower triangle, row-major: entry (a, b), b <= a, at a * (a + 1) / 2 + b.
#define AVBD_LANES 8
#define AVBD_GROUPS (32 / AVBD_LANES)
__device__ __forceinline__ int avbd_lt(int a, int b) { return a * (a + 1) / 2 + b; }
__device__ __forceinline__ void avbd_primal(const DevState& d, const Params& p, int cur, uint32_t i, float dt, float alpha) {
  const int lane = threadIdx.x & (AVBD_LANES - 1);
  float g[6], H[21];
#pragma unroll
  for (int a = 0; a < 6; ++a) g[a] = 0.f;
#pragma unroll
  for (int a = 0; a < 21; ++a) H[a] = 0.f;
  const uint32_t s0 = i == BB_NONE ? 0u : d.csr_start[cur][i], s1 = i == BB_NONE ? 0u : d.csr_start[cur][i + 1];
  for (uint32_t e = s0 + uint32_t(lane); e < s1; e += AVBD_LANES) {
    const uint32_t slot = d.man_slot[cur][d.csr_list[cur][e]];
    const int cc = d.m_keycc[cur][slot].y;
    const uint2 b = d.m_bodies[cur][slot];
    const bool i1 = b.x == i;
    const bool d1 = awake(d.flags[b.x]), d2 = awake(d.flags[b.y]);
    const float mu = sqrtf(fmaxf(d.iinv[b.x].w, 0.f) * fmaxf(d.iinv[b.y].w, 0.f));
    const float3 n = f3(d.m_normal[cur][slot]);
    const float3 td[2] = {f3(d.m_t0[cur][slot]), f3(d.m_t1[cur][slot])};
    for (int j = 0; j < cc; ++j) {
      const uint32_t ci = slot * BB_MAX_CONTACTS + uint32_t(j);
      float3 rr1, rr2;
      const float C = avbd_contact_C(d, p, cur, slot, ci, b, d1, d2, alpha, n, rr1, rr2);
      const float4 lam = d.c_lam[cur][ci];
      const float4 kt = d.c_kt[cur][ci];
      const float f = fminf(lam.w * C + lam.x, 0.f);
      const float3 Jl = i1 ? -n : n;
      const float3 Ja = i1 ? -cross3(rr1, n) : cross3(rr2, n);
      const float J[6] = {Jl.x, Jl.y, Jl.z, Ja.x, Ja.y, Ja.z};
#pragma unroll
      for (int a = 0; a < 6; ++a) g[a] += f * J[a];
#pragma unroll
      for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int bb = 0; bb <= a; ++bb) H[avbd_lt(a, bb)] += lam.w * J[a] * J[bb];
      const float bound = mu * fabsf(lam.x);
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        float3 ar1, ar2;
        float C0t;
        const float Ct = avbd_dir_C(d, p, cur, ci, b, d1, d2, alpha, td[t], ar1, ar2, C0t);
        const float ktt = t == 0 ? kt.x : kt.y;
        const float lt = t == 0 ? lam.y : lam.z;
        const float ft = fminf(fmaxf(ktt * Ct + lt, -bound), bound);
        const float3 Jlt = i1 ? -td[t] : td[t];
        const float3 Jat = i1 ? -cross3(ar1, td[t]) : cross3(ar2, td[t]);
        const float Jt[6] = {Jlt.x, Jlt.y, Jlt.z, Jat.x, Jat.y, Jat.z};
#pragma unroll
        for (int a = 0; a < 6; ++a) g[a] += ft * Jt[a];
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
          for (int bb = 0; bb <= a; ++bb) H[avbd_lt(a, bb)] += ktt * Jt[a] * Jt[bb];
      }
    }
  }
#pragma unroll
  for (int o = AVBD_LANES / 2; o > 0; o >>= 1) {
#pragma unroll
    for (int a = 0; a < 6; ++a) g[a] += __shfl_xor_sync(0xFFFFFFFFu, g[a], o);
#pragma unroll
    for (int a = 0; a < 21; ++a) H[a] += __shfl_xor_sync(0xFFFFFFFFu, H[a], o);
  }
  if (lane != 0 || i == BB_NONE) return;
  const bool tq = p.quirks & BB_QUIRK_INERTIA_TRANSPOSE;
  const float inv_dt2 = dt > 0.f ? 1.0f / (dt * dt) : 0.f;
  const float m_lin = d.vel[i].w * inv_dt2;
  Quatf rot = q_from(d.rot[i]);
  Sym3 wi = body_world_inv_inertia(d.iinv, d.iinv_off, d.full_inertia != 0, i, rot, tq);
  // avbd_inverse3 (avbd.slang:309-326) of the symmetric world inverse inertia
  float3 c0 = make_float3(wi.xx, wi.xy, wi.xz), c1 = make_float3(wi.xy, wi.yy, wi.yz), c2 = make_float3(wi.xz, wi.yz, wi.zz);
  float3 r0 = cross3(c1, c2), r1 = cross3(c2, c0), r2 = cross3(c0, c1);
  float det = dot3(c0, r0);
  float inv = fabsf(det) > 1e-12f ? 1.0f / det : 0.f;
  r0 = r0 * inv;
  r1 = r1 * inv;
  r2 = r2 * inv;
  const float Iw[3][3] = {{r0.x, r0.y, r0.z}, {r1.x, r1.y, r1.z}, {r2.x, r2.y, r2.z}};
  H[avbd_lt(0, 0)] += m_lin;
  H[avbd_lt(1, 1)] += m_lin;
  H[avbd_lt(2, 2)] += m_lin;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int bb = 0; bb <= a; ++bb) H[avbd_lt(3 + a, 3 + bb)] += Iw[a][bb] * inv_dt2;
  const float3 dpos = f3(d.pos[i]) - f3(d.a_pos_tilde[i]);
  const float3 dth = small_angle_delta(rot, q_from(d.a_rot_tilde[i]));
  g[0] += m_lin * dpos.x;
  g[1] += m_lin * dpos.y;
  g[2] += m_lin * dpos.z;
  const float3 ga = make_float3(Iw[0][0] * dth.x + Iw[0][1] * dth.y + Iw[0][2] * dth.z,
                                Iw[1][0] * dth.x + Iw[1][1] * dth.y + Iw[1][2] * dth.z,
                                Iw[2][0] * dth.x + Iw[2][1] * dth.y + Iw[2][2] * dth.z) * inv_dt2;
  g[3] += ga.x;
  g[4] += ga.y;
  g[5] += ga.z;
  // avbd_solve6: in-place LDL^T, diagonal floor 1e-8
  float x[6], rhs[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) rhs[a] = -g[a];
#pragma unroll
  for (int jj = 0; jj < 6; ++jj) {
    float dd = H[avbd_lt(jj, jj)];
#pragma unroll
    for (int kk = 0; kk < 6; ++kk)
      if (kk < jj) dd -= H[avbd_lt(jj, kk)] * H[avbd_lt(jj, kk)] * H[avbd_lt(kk, kk)];
    dd = fmaxf(dd, 1e-8f);
    H[avbd_lt(jj, jj)] = dd;
#pragma unroll
    for (int ii = 0; ii < 6; ++ii) {
      if (ii > jj) {
        float sm = H[avbd_lt(ii, jj)];
#pragma unroll
        for (int kk = 0; kk < 6; ++kk)
          if (kk < jj) sm -= H[avbd_lt(ii, kk)] * H[avbd_lt(jj, kk)] * H[avbd_lt(kk, kk)];
        H[avbd_lt(ii, jj)] = sm / dd;
      }
    }
  }
#pragma unroll
  for (int ii = 0; ii < 6; ++ii) {
    float sm = rhs[ii];
#pragma unroll
    for (int kk = 0; kk < 6; ++kk)
      if (kk < ii) sm -= H[avbd_lt(ii, kk)] * rhs[kk];
    rhs[ii] = sm;
  }
#pragma unroll
  for (int ii = 0; ii < 6; ++ii) rhs[ii] /= H[avbd_lt(ii, ii)];
#pragma unroll
  for (int ii = 5; ii >= 0; --ii) {
    float sm = rhs[ii];
#pragma unroll
    for (int kk = 0; kk < 6; ++kk)
      if (kk > ii) sm -= H[avbd_lt(kk, ii)] * x[kk];
    x[ii] = sm;
  }
  float4 ps = d.pos[i];
  d.pos[i] = make_float4(ps.x + x[0], ps.y + x[1], ps.z + x[2], ps.w);
  Quatf dq{x[3] * 0.5f, x[4] * 0.5f, x[5] * 0.5f, 1.0f};
  d.rot[i] = q_to4(q_normalize(q_mul(dq, rot)));
}

// entry_avbd_dual (avbd.slang:728-808)
__device__ void avbd_dual(const DevState& d, const Params& p, int cur, uint32_t m) {
  const uint32_t slot = d.man_slot[cur][m];
  const uint2 b = d.m_bodies[cur][slot];
  const bool d1 = awake(d.flags[b.x]), d2 = awake(d.flags[b.y]);
  if (!d1 && !d2) return;
  const float mu = sqrtf(fmaxf(d.iinv[b.x].w, 0.f) * fmaxf(d.iinv[b.y].w, 0.f));
  const float3 n = f3(d.m_normal[cur][slot]);
  const float3 td[2] = {f3(d.m_t0[cur][slot]), f3(d.m_t1[cur][slot])};
  const int cc = d.m_keycc[cur][slot].y;
  for (int j = 0; j < cc; ++j) {
    const uint32_t ci = slot * BB_MAX_CONTACTS + j;
    float3 rr1, rr2;
    float C = avbd_contact_C(d, p, cur, slot, ci, b, d1, d2, 1.0f, n, rr1, rr2);
    float4 lam = d.c_lam[cur][ci];
    float4 kt = d.c_kt[cur][ci];
    const float lam0 = lam.x, k = lam.w;
    float nl = fminf(k * C + lam0, 0.f);
    lam.x = nl;
    if (nl < 0.f) lam.w = fminf(k + p.avbd_beta * fabsf(C), p.avbd_k_max);
    const float bound = mu * fabsf(lam0);
    bool stick_ok = true;
    float drift2 = 0.f;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      float3 ar1, ar2;
      float C0t;
      float Ct = avbd_dir_C(d, p, cur, ci, b, d1, d2, 1.0f, td[t], ar1, ar2, C0t);
      float lt = t == 0 ? lam.y : lam.z;
      float ktt = t == 0 ? kt.x : kt.y;
      float nlt = fminf(fmaxf(ktt * Ct + lt, -bound), bound);
      if (t == 0) lam.y = nlt;
      else lam.z = nlt;
      if (nlt > -bound && nlt < bound) {
        float nk = fminf(ktt + p.avbd_beta * fabsf(Ct), p.avbd_k_max);
        if (t == 0) kt.x = nk;
        else kt.y = nk;
      } else {
        stick_ok = false;
      }
      drift2 += C0t * C0t;
    }
    uint32_t stick = (stick_ok && drift2 < p.avbd_stick_thresh * p.avbd_stick_thresh) ? 1u : 0u;
    d.c_lam[cur][ci] = lam;
    d.c_kt[cur][ci] = make_float4(kt.x, kt.y, __uint_as_float(stick), kt.w);
  }
}

// entry_avbd_finalize (avbd.slang:132-202)
__device__ void avbd_finalize(const DevState& d, int cur, uint32_t i, float dt) {
  const float inv_dt = dt > 0.f ? 1.0f / dt : 0.f;
  float4 v4 = d.vel[i];
  d.pvel[i] = v4;
  float3 v = (f3(d.pos[i]) - f3(d.a_pos_start[i])) * inv_dt;
  Quatf dq = q_mul(q_from(d.rot[i]), q_conj(q_from(d.a_rot_start[i])));
  float sg = dq.w < 0.f ? -1.f : 1.f;
  float3 w = make_float3(dq.x, dq.y, dq.z) * (2.0f * sg * inv_dt);
  if (dot3(v, v) < 0.09f && dot3(w, w) < 0.16f && d.csr_start[cur][i + 1] - d.csr_start[cur][i] >= 3u) {
    v = v * 0.9f;
    w = w * 0.9f;
  }
  d.vel[i] = f4(v, v4.w);
  d.omega[i] = f4(w, 0.f);
}

// persistent solve: main iterations (colour sweeps + dual), finalize, post-stabilisation
__global__ void __launch_bounds__(BB_COOP_THREADS, 1) k_avbd_solve(const DevState d, Params p, int cur, uint32_t n, float dt,
                                                           int phase) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  // primal sweeps: AVBD_GROUPS bodies per warp (AVBD_LANES lanes each), warp-uniform trips
  const uint32_t wid = tid >> 5, nwarps = stride >> 5, grp = (threadIdx.x & 31u) / AVBD_LANES;
  const uint32_t* list = d.a_bucket_vals[1];
  uint32_t* sync = &d.ctr->sync_count[3 + phase];
  uint32_t ep = 0;
  if (phase == 0) {
    const uint32_t C = d.ctr->avbd_colors;
    const uint32_t M = d.ctr->manifold_count;
    for (uint32_t it = 0; it < p.avbd_iterations; ++it) {
      for (uint32_t c = 0; c < C; ++c) {
        uint32_t s0 = d.a_bucket_start[c], s1 = d.a_bucket_start[c + 1];
        if (s0 == s1) continue;
        for (uint32_t kw = s0 + wid * AVBD_GROUPS; kw < s1; kw += nwarps * AVBD_GROUPS)
          avbd_primal(d, p, cur, kw + grp < s1 ? list[kw + grp] : BB_NONE, dt, 1.0f);
        grid_sync(d.ctr, sync, ep);
      }
      for (uint32_t m = tid; m < M; m += stride) avbd_dual(d, p, cur, m);
      grid_sync(d.ctr, sync, ep);
    }
    for (uint32_t i = tid; i < n; i += stride)
      if (awake(d.flags[i])) avbd_finalize(d, cur, i, dt);
  } else if (phase == 1) {
    const uint32_t nb = p.avbd_shock_layers * BB_MAX_COLORS;
    for (uint32_t key = 0; key < nb; ++key) {
      uint32_t s0 = d.a_bucket_start[key], s1 = d.a_bucket_start[key + 1];
      if (s0 == s1) continue;
      for (uint32_t kw = s0 + wid * AVBD_GROUPS; kw < s1; kw += nwarps * AVBD_GROUPS)
        avbd_primal(d, p, cur, kw + grp < s1 ? list[kw + grp] : BB_NONE, dt, 0.0f);
      grid_sync(d.ctr, sync, ep);
    }
  } else {
    const uint32_t C = d.ctr->avbd_colors;
    for (uint32_t sw = 1; sw < p.avbd_post_stab_sweeps; ++sw) {
      for (uint32_t c = 0; c < C; ++c) {
        uint32_t s0 = d.a_bucket_start[c], s1 = d.a_bucket_start[c + 1];
        if (s0 == s1) continue;
        for (uint32_t kw = s0 + wid * AVBD_GROUPS; kw < s1; kw += nwarps * AVBD_GROUPS)
          avbd_primal(d, p, cur, kw + grp < s1 ? list[kw + grp] : BB_NONE, dt, 0.0f);
        grid_sync(d.ctr, sync, ep);
      }
    }
  }
}

// Scratch of the body bucket sorts (every region is zeroed once per substep and used once):
// histogram region `region` (2048 words each), status / tile-counter slots from `slot`.
static void avbd_buckets(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, const StepScratch& sc,
                         int sms, int post, int region, int slot) {
  const int T = BB_THREADS;
  uint32_t blocks = (n + T - 1) / T;
  k_avbd_keys<<<blocks, T, 0, s>>>(d, p, n, post);
  uint32_t* keys[2] = {d.a_bucket_keys[0], d.a_bucket_keys[1]};
  uint32_t* vals[2] = {d.a_bucket_vals[0], d.a_bucket_vals[1]};
  uint32_t* hist = sc.sort_hist + size_t(region) * BB_HIST_REGION;
  // post keys need 9 bits; three 8-bit passes (the third sees only zero digits, so it keeps
  // the order) leave the result in buffer 1 like the one-pass colour sort
  bb_launch_sort(s, keys, vals, nullptr, n, post ? 3 : 1, 0, hist, sc.sort_status + size_t(slot) * sc.sort_tiles * 256,
                 sc.sort_tile_ctr + slot, d.ctr, sms);
  uint32_t nb = post ? p.avbd_shock_layers * BB_MAX_COLORS : BB_MAX_COLORS;
  k_lower_bounds<<<(nb + 1 + 127) / 128, 128, 0, s>>>(d.a_bucket_keys[1], n, d.a_bucket_start, nb);
}

int bb_avbd_blocks(int sms) {
  return std::min(bb_coop_blocks((const void*)k_avbd_color, BB_COOP_THREADS, sms),
                  bb_coop_blocks((const void*)k_avbd_solve, BB_COOP_THREADS, sms));
}

void bb_solve_avbd(cudaStream_t s, const DevState& d, const Params& p, uint32_t n, float h, const StepScratch& sc,
                   int sms, int cur, int coop_blocks) {
  if (n == 0) return;
  const int T = BB_THREADS;
  uint32_t blocks = (n + T - 1) / T;
  {
    DevState dd = d;
    Params pp = p;
    int cc = cur;
    uint32_t nn = n;
    void* args[] = {&dd, &pp, &cc, &nn};
    bb_launch_coop((const void*)k_avbd_color, coop_blocks, BB_COOP_THREADS, args, s);
  }
  k_avbd_prepare<<<blocks, T, 0, s>>>(d, p, n, h);
  k_avbd_warmstart<<<sms * 8, T, 0, s>>>(d, p, cur);
  k_avbd_depth_reset<<<blocks, T, 0, s>>>(d, n);
  for (uint32_t k = 0; k < p.avbd_shock_layers; ++k) k_avbd_depth_relax<<<sms * 8, T, 0, s>>>(d, cur);
  DevState dd = d;
  Params pp = p;
  int cc = cur;
  uint32_t nn = n;
  float hh = h;
  int phase = 0;
  void* args[] = {&dd, &pp, &cc, &nn, &hh, &phase};
  avbd_buckets(s, d, p, n, sc, sms, 0, 2, 7);
  bb_launch_coop((const void*)k_avbd_solve, coop_blocks, BB_COOP_THREADS, args, s);
  avbd_buckets(s, d, p, n, sc, sms, 1, 3, 8);  // slots 8, 9, 10
  int phase1 = 1;
  void* args1[] = {&dd, &pp, &cc, &nn, &hh, &phase1};
  bb_launch_coop((const void*)k_avbd_solve, coop_blocks, BB_COOP_THREADS, args1, s);
  if (p.avbd_post_stab_sweeps > 1) {
    avbd_buckets(s, d, p, n, sc, sms, 0, 4, 11);
    int phase2 = 2;
    void* args2[] = {&dd, &pp, &cc, &nn, &hh, &phase2};
    bb_launch_coop((const void*)k_avbd_solve, coop_blocks, BB_COOP_THREADS, args2, s);
  }
}
