// Per-pixel arithmetic of the half-storage fused iteration.
//
// The same update as tgv_pixel.cuh (updateDualVariables.cu:33-98, thresholdingL1.cu:45-115,
// updatePrimalVariables.cu:77-110, preconditioning.cu:18-20), evaluated with fused
// multiply-adds and with the PTX instructions rcp.approx.ftz.f32 and rsqrt.approx.ftz.f32
// (relative error below 2^-22) in place of IEEE division and square root.  On this path p,
// q and v-bar are stored in half precision (relative rounding 2^-11), which dominates the
// difference; the result is checked against the FP64 oracle with a tolerance.  The FP32
// fused path keeps the exact forms of tgv_pixel.cuh and stays bit-identical to the drop-in
// kernels.
#pragma once
#include <cuda_runtime.h>

namespace vfs {
namespace fast {

__device__ __forceinline__ float rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ float rsqrt(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Pairs of floats on the packed FP32 instructions of sm_100 (add / sub / mul / fma .rn.f32x2,
// no flush to zero): each lane is the IEEE single-precision operation of the scalar form, so
// a packed step gives the bits of the two scalar steps it replaces.
namespace x2 {
typedef unsigned long long f2;
__device__ __forceinline__ f2 pk(float x, float y) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ float2 upk(f2 r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}
__device__ __forceinline__ f2 add(f2 a, f2 b) {
  f2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2 sub(f2 a, f2 b) {
  f2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2 mul(f2 a, f2 b) {
  f2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2 fma(f2 a, f2 b, f2 c) {
  f2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
}  // namespace x2

// Dual update.  A forward difference (right / down neighbour) and a backward one (left /
// up) differ only in sign, so each is written as sgn * (neighbour - centre); the sign
// change is exact.  The projection onto the unit ball multiplies by 1 / |p| where |p| > 1
// (a NaN norm propagates, as max(rep, 1) does in the reference).
__device__ __forceinline__ void dual(bool useRight, bool useDown, float u_pos, float u_xn, float u_yn, float2 vp,
                                     float2 v_xn, float2 v_yn, float a, float b, float c, float sp, float sq,
                                     float2& p, float4& q) {
  const float sx = useRight ? 1.0f : -1.0f;
  const float sy = useDown ? 1.0f : -1.0f;
  float u_x = __fmaf_rn(sx, u_xn - u_pos, -vp.x);
  float u_y = __fmaf_rn(sy, u_yn - u_pos, -vp.y);
  float dtx = __fmaf_rn(a, u_x, c * u_y);
  float dty = __fmaf_rn(c, u_x, b * u_y);
  // p and the q lanes (x, w) / (z, y) in pairs on the packed instructions (namespace x2)
  float2 pp = x2::upk(x2::fma(x2::pk(sp, sp), x2::pk(dtx, dty), x2::pk(p.x, p.y)));
  float ppx = pp.x, ppy = pp.y;
  float n2 = __fmaf_rn(ppx, ppx, ppy * ppy);
  if (!(n2 <= 1.0f)) {
    float r = rsqrt(n2);
    ppx *= r;
    ppy *= r;
  }
  p = make_float2(ppx, ppy);
  const float qsx = sq * sx, qsy = sq * sy;  // exact: a sign change
  const x2::f2 vpp = x2::pk(vp.x, vp.y);
  const float2 qxw = x2::upk(x2::fma(x2::pk(qsx, qsx), x2::sub(x2::pk(v_xn.x, v_xn.y), vpp), x2::pk(q.x, q.w)));
  const float2 qzy = x2::upk(x2::fma(x2::pk(qsy, qsy), x2::sub(x2::pk(v_yn.x, v_yn.y), vpp), x2::pk(q.z, q.y)));
  float qx = qxw.x, qw = qxw.y, qz = qzy.x, qy = qzy.y;
  float m2 = __fmaf_rn(qx, qx, __fmaf_rn(qy, qy, __fmaf_rn(qz, qz, qw * qw)));
  if (!(m2 <= 1.0f)) {
    float r = rsqrt(m2);
    qx *= r;
    qy *= r;
    qz *= r;
    qw *= r;
  }
  q = make_float4(qx, qy, qz, qw);
}

// dual() at a pixel whose right and down neighbours are the ones used (sx = sy = 1), with the
// x / y and q lanes paired.  fma(1, d, -v) and d - v round the same exact value once, and
// sq * 1 is exact, so every lane is the scalar form's operation.
__device__ __forceinline__ void dual_interior(float u_pos, float u_xn, float u_yn, float2 vp, float2 v_xn,
                                              float2 v_yn, float a, float b, float c, float sp, float sq, float2& p,
                                              float4& q) {
  using namespace x2;
  const f2 vpp = pk(vp.x, vp.y);
  const float2 u = upk(sub(sub(pk(u_xn, u_yn), pk(u_pos, u_pos)), vpp));
  float dtx = __fmaf_rn(a, u.x, c * u.y);
  float dty = __fmaf_rn(c, u.x, b * u.y);
  float2 pp = upk(fma(pk(sp, sp), pk(dtx, dty), pk(p.x, p.y)));
  float n2 = __fmaf_rn(pp.x, pp.x, pp.y * pp.y);
  if (!(n2 <= 1.0f)) {
    float r = rsqrt(n2);
    pp.x *= r;
    pp.y *= r;
  }
  p = pp;
  const f2 s2 = pk(sq, sq);
  const float2 qxw = upk(fma(s2, sub(pk(v_xn.x, v_xn.y), vpp), pk(q.x, q.w)));
  const float2 qzy = upk(fma(s2, sub(pk(v_yn.x, v_yn.y), vpp), pk(q.z, q.y)));
  float qx = qxw.x, qw = qxw.y, qz = qzy.x, qy = qzy.y;
  float m2 = __fmaf_rn(qx, qx, __fmaf_rn(qy, qy, __fmaf_rn(qz, qz, qw * qw)));
  if (!(m2 <= 1.0f)) {
    float r = rsqrt(m2);
    qx *= r;
    qy *= r;
    qz *= r;
    qw *= r;
  }
  q = make_float4(qx, qy, qz, qw);
}

__device__ __forceinline__ float2 tp(float a, float b, float c, float2 p) {
  return make_float2(__fmaf_rn(a, p.x, c * p.y), __fmaf_rn(c, p.x, b * p.y));
}

// Preconditioners eta_u, eta_v1, eta_v2 (a1s = alpha1^2, a0s4 = 4 alpha0^2).
__device__ __forceinline__ float etau(float a, float b, float c, float a1s) {
  float ac = a + c, bc = b + c;
  float s = __fmaf_rn(a, a, b * b);
  s = __fmaf_rn(2.0f * c, c, s);
  s = __fmaf_rn(ac, ac, s);
  s = __fmaf_rn(bc, bc, s);
  return s * a1s;
}
__device__ __forceinline__ float etav(float x, float c, float a1s, float a0s4) {
  return __fmaf_rn(a1s, __fmaf_rn(x, x, c * c), a0s4);
}

// Reciprocal preconditioners, constant over a pyramid level (a, b, c are): the fused
// iteration takes them from a per-level record (k_level_tensor) instead of recomputing them
// every iteration.  Each is the value the step would form itself, so the result is the same
// bit for bit either way.
//   etau_rcp: 1 / eta_u, or 1 where eta_u = 0 (the step is then tau itself: tau * 1 = tau).
//   etav_rcp: (1 / eta_v1, or 1 where eta_v1 = 0; 1 / eta_v2, or -0 where eta_v2 = 0).  eta_v2
//   is a sum of non-negative terms (or NaN), so rcp never gives -0 for it and -0 marks the
//   eta_v2 = 0 branch of updatePrimalVariables.cu:103-105 unambiguously.
__device__ __forceinline__ float etau_rcp(float eu) { return (eu == 0.0f) ? 1.0f : rcp(eu); }
__device__ __forceinline__ float2 etav_rcp(float ev1, float ev2) {
  return make_float2(ev1 != 0.0f ? rcp(ev1) : 1.0f, ev2 != 0.0f ? rcp(ev2) : -0.0f);
}
__device__ __forceinline__ bool etav2_zero(float r2) { return __float_as_uint(r2) == 0x80000000u; }

// L1 thresholding (the three cases of the linearised data term); teu = tau / eta_u.
__device__ __forceinline__ float threshold_teu(float dxm, float dym, float teu, float u_bar, float upos, float Ius,
                                               float Iz, float lambda) {
  float div_p = dxm + dym;
  float dun = __fmaf_rn(teu, div_p, u_bar) - upos;
  float rho = __fmaf_rn(Ius, dun, Iz);
  float lt = lambda * teu;
  float upper = lt * (Ius * Ius);
  float d = 0.0f;
  if ((rho <= upper) && (rho >= -upper)) {
    d = (Ius == 0.0f) ? dun : __fmaf_rn(-rho, rcp(Ius), dun);
  } else if (rho < -upper) {
    d = __fmaf_rn(lt, Ius, dun);
  } else if (rho > upper) {
    d = __fmaf_rn(-lt, Ius, dun);
  }
  return upos + d;
}
__device__ __forceinline__ float threshold(float dxm, float dym, float eu, float tau, float u_bar, float upos,
                                           float Ius, float Iz, float lambda) {
  return threshold_teu(dxm, dym, tau * etau_rcp(eu), u_bar, upos, Ius, Iz, lambda);
}

// Primal update with the x / y lanes paired: dq = (q.x - ql.x) + (q.z - qu.z) and
// (q.w - ql.w) + (q.y - qu.y), g = alpha1 T p + alpha0 dq, v = v-bar + (tau / eta_v) g (the
// eta_v2 = 0 case of updatePrimalVariables.cu:103-105 writes .x again and keeps .y), then the
// over-relaxation.  qxw_l = (q.x, q.w) of the west neighbour, qzy_u = (q.z, q.y) of the north
// one (zero where absent).
// r12 = etav_rcp(eta_v1, eta_v2).
__device__ __forceinline__ void primal_interior_r(float4 qc, float2 qxw_l, float2 qzy_u, float2 tpp, float2 r12,
                                                  float tau, float alpha0, float alpha1, float mu, float2 vb,
                                                  float u_new, float u_bar, float& u_s, float2& v_s) {
  using namespace x2;
  const f2 dq = add(sub(pk(qc.x, qc.w), pk(qxw_l.x, qxw_l.y)), sub(pk(qc.z, qc.y), pk(qzy_u.x, qzy_u.y)));
  const f2 g = fma(pk(alpha1, alpha1), pk(tpp.x, tpp.y), mul(pk(alpha0, alpha0), dq));
  const f2 vbb = pk(vb.x, vb.y);
  f2 v;
  if (!etav2_zero(r12.y)) {
    v = fma(pk(tau * r12.x, tau * r12.y), g, vbb);
  } else {  // updatePrimalVariables.cu:103-105 writes .x again; .y keeps the previous value
    v = pk(__fmaf_rn(tau, upk(g).x, vb.x), vb.y);
  }
  u_s = __fmaf_rn(mu, u_new - u_bar, u_new);
  v_s = upk(fma(pk(mu, mu), sub(v, vbb), v));
}
__device__ __forceinline__ void primal_interior(float4 qc, float2 qxw_l, float2 qzy_u, float2 tpp, float ev1,
                                                float ev2, float tau, float alpha0, float alpha1, float mu, float2 vb,
                                                float u_new, float u_bar, float& u_s, float2& v_s) {
  primal_interior_r(qc, qxw_l, qzy_u, tpp, etav_rcp(ev1, ev2), tau, alpha0, alpha1, mu, vb, u_new, u_bar, u_s, v_s);
}


// Primal update of v and the over-relaxation of u and v; tpp = T p at this pixel; ql / qu: q
// of the west / north neighbour (zero where absent), of which the step reads (x, w) / (z, y).
__device__ __forceinline__ void primal_r(float4 qc, float4 ql, float4 qu, float2 tpp, float2 r12, float tau,
                                         float alpha0, float alpha1, float mu, float2 vb, float u_new, float u_bar,
                                         float& u_s, float2& v_s) {
  primal_interior_r(qc, make_float2(ql.x, ql.w), make_float2(qu.z, qu.y), tpp, r12, tau, alpha0, alpha1, mu, vb,
                    u_new, u_bar, u_s, v_s);
}
__device__ __forceinline__ void primal(float4 qc, float4 ql, float4 qu, float2 tpp, float ev1, float ev2, float tau,
                                       float alpha0, float alpha1, float mu, float2 vb, float u_new, float u_bar,
                                       float& u_s, float2& v_s) {
  primal_r(qc, ql, qu, tpp, etav_rcp(ev1, ev2), tau, alpha0, alpha1, mu, vb, u_new, u_bar, u_s, v_s);
}

}  // namespace fast
}  // namespace vfs
