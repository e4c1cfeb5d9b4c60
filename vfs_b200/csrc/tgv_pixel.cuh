// Per-pixel arithmetic of the inner primal-dual iteration, shared by the drop-in
// kernels and the fused kernels so that both evaluate the same operations in the
// same order (the library is built with -fmad=false).
#pragma once
#include <cuda_runtime.h>

namespace vfs {

// updateDualVariables.cu:33-98.  u_xn / v_xn: the neighbour the reference uses for the
// x difference (right if useRight, else left); u_yn / v_yn likewise (down / up).
// sp = alpha1 * sigma / eta_p and sq = alpha0 * sigma / eta_q are the same for every
// pixel of a launch and are evaluated once by the caller (IEEE float division gives the
// same bits wherever it is evaluated).  A projection norm clamped to 1 divides by 1,
// which is exact, so that division is skipped.
__device__ __forceinline__ void dual_math(bool useRight, bool useDown, float u_pos, float u_xn, float u_yn,
                                          float2 vp, float2 v_xn, float2 v_yn, float a, float b, float c,
                                          float sp, float sq, float2& p, float4& q) {
  float u_x = useRight ? u_xn - u_pos - vp.x : u_pos - u_xn - vp.x;
  float u_y = useDown ? u_yn - u_pos - vp.y : u_pos - u_yn - vp.y;
  float dtx = a * u_x + c * u_y;
  float dty = c * u_x + b * u_y;
  float ppx = p.x + sp * dtx;
  float ppy = p.y + sp * dty;
  float rep = sqrtf(ppx * ppx + ppy * ppy);
  if (!(rep <= 1.0f)) {  // max(rep, 1) in the reference; NaN propagates as there
    ppx = ppx / rep;
    ppy = ppy / rep;
  }
  p = make_float2(ppx, ppy);
  float gvx = useRight ? v_xn.x - vp.x : vp.x - v_xn.x;
  float gvy = useDown ? v_yn.y - vp.y : vp.y - v_yn.y;
  float gvz = useDown ? v_yn.x - vp.x : vp.x - v_yn.x;
  float gvw = useRight ? v_xn.y - vp.y : vp.y - v_xn.y;
  float qx = q.x + sq * gvx;
  float qy = q.y + sq * gvy;
  float qz = q.z + sq * gvz;
  float qw = q.w + sq * gvw;
  float reproj = sqrtf(qx * qx + qy * qy + qz * qz + qw * qw);
  if (!(reproj <= 1.0f)) {
    qx = qx / reproj;
    qy = qy / reproj;
    qz = qz / reproj;
    qw = qw / reproj;
  }
  q = make_float4(qx, qy, qz, qw);
}

// thresholdingL1.cu:104-115
__device__ __forceinline__ float2 tp_math(float a, float b, float c, float2 p) {
  return make_float2(a * p.x + c * p.y, c * p.x + b * p.y);
}

// preconditioning.cu:18-20
__device__ __forceinline__ float etau_math(float a, float b, float c, float alpha1) {
  return (a * a + b * b + 2 * c * c + (a + c) * (a + c) + (b + c) * (b + c)) * (alpha1 * alpha1);
}
__device__ __forceinline__ float etav1_math(float b, float c, float alpha0, float alpha1) {
  return (alpha1 * alpha1) * (b * b + c * c) + 4 * alpha0 * alpha0;
}
__device__ __forceinline__ float etav2_math(float a, float c, float alpha0, float alpha1) {
  return (alpha1 * alpha1) * (a * a + c * c) + 4 * alpha0 * alpha0;
}

// thresholdingL1.cu:45-83 given the divergence terms dxm, dym
__device__ __forceinline__ float threshold_math(float dxm, float dym, float eu, float tau, float u_bar, float upos,
                                                float Ius, float Iz, float lambda) {
  float div_p = dxm + dym;
  float tau_eta_u = (eu == 0.0f) ? tau : tau / eu;
  float uhat = u_bar + tau_eta_u * div_p;
  float dun = uhat - upos;
  float rho = Ius * dun + Iz;
  float upper = lambda * tau_eta_u * (Ius * Ius);
  float lower = -lambda * tau_eta_u * (Ius * Ius);
  float d = 0.0f;
  if ((rho <= upper) && (rho >= lower)) {
    if (Ius == 0.0f) d = dun;
    else d = dun - rho / Ius;
  } else if (rho < lower) {
    d = dun + lambda * tau_eta_u * Ius;
  } else if (rho > upper) {
    d = dun - lambda * tau_eta_u * Ius;
  }
  return upos + d;
}

// updatePrimalVariables.cu:77-110 given qc (already zeroed at the right / lower
// edge), the west and north q (zero when absent), p, the tensor and preconditioners.
__device__ __forceinline__ void primal_math(float4 qc, float4 ql, float4 qu, float2 pp, float a, float b, float c,
                                            float ev1, float ev2, float tau, float alpha0, float alpha1, float mu,
                                            float2 vb, float u_new, float u_bar, float& u_s, float2& v_s,
                                            float2& v_out) {
  float dqx = (qc.x - ql.x) + (qc.z - qu.z);
  float dqy = (qc.w - ql.w) + (qc.y - qu.y);
  float dtx = a * pp.x + c * pp.y;
  float dty = c * pp.x + b * pp.y;
  float vx, vy;
  if (ev1 != 0.0f) vx = vb.x + (tau / ev1) * (alpha1 * dtx + alpha0 * dqx);
  else vx = vb.x + (tau) * (alpha1 * dtx + alpha0 * dqx);
  if (ev2 != 0.0f) {
    vy = vb.y + (tau / ev2) * (alpha1 * dty + alpha0 * dqy);
  } else {  // updatePrimalVariables.cu:103-105 writes .x again; .y keeps the previous value
    vx = vb.x + (tau) * (alpha1 * dtx + alpha0 * dqx);
    vy = vb.y;
  }
  v_out = make_float2(vx, vy);
  u_s = u_new + mu * (u_new - u_bar);
  v_s = make_float2(vx + mu * (vx - vb.x), vy + mu * (vy - vb.y));
}

// updateDualVariables.cu:13-16: the plain kernels' fixed circular domain
__device__ __forceinline__ bool outside_circle(int ix, int iy, int w, int h) {
  float desiredRadius = (float)w / 2.20f;
  float halfWidth = (float)w / 2.0f;
  float halfHeight = (float)h / 2.0f;
  float radius = sqrtf((iy - halfHeight) * (iy - halfHeight) + (ix - halfWidth) * (ix - halfWidth));
  return radius >= desiredRadius;
}

// One round of the forgetful selection below on the values s[0..K-1]: their minimum ends in
// s[0], their maximum in s[K-1], the other K-2 values in s[1..K-2].  Pairs (i, K-1-i) are
// ordered first; the minimum is then among the low members (and, K odd, the middle value),
// the maximum among the high members and the middle value.
__device__ __forceinline__ void order2(float& lo, float& hi) {
  const float a = fminf(lo, hi), b = fmaxf(lo, hi);
  lo = a;
  hi = b;
}
template <int K>
__device__ __forceinline__ void minmax_round(float* s) {
  constexpr int H = K / 2;
#pragma unroll
  for (int i = 0; i < H; i++) order2(s[i], s[K - 1 - i]);
#pragma unroll
  for (int i = 1; i < (K + 1) / 2; i++) order2(s[0], s[i]);
#pragma unroll
  for (int i = K - 2; i >= H; i--) order2(s[i], s[K - 1]);
}

// 13th smallest of m[0..24] by forgetful selection: the minimum and the maximum of 14 of the
// values are each beyond the median's rank (one is below 13 others, the other above 13), so
// both are dropped and the median of the 23 that remain is the same value; the next value
// joins the 12 kept, and so on down to three values, whose middle one is the median.  About
// 150 min / max pairs, against 234 for 13 passes of selection sort.
__device__ __forceinline__ float median25(float* m) {
  minmax_round<14>(m);
  m[0] = m[14];
  minmax_round<13>(m);
  m[0] = m[15];
  minmax_round<12>(m);
  m[0] = m[16];
  minmax_round<11>(m);
  m[0] = m[17];
  minmax_round<10>(m);
  m[0] = m[18];
  minmax_round<9>(m);
  m[0] = m[19];
  minmax_round<8>(m);
  m[0] = m[20];
  minmax_round<7>(m);
  m[0] = m[21];
  minmax_round<6>(m);
  m[0] = m[22];
  minmax_round<5>(m);
  m[0] = m[23];
  minmax_round<4>(m);
  m[0] = m[24];
  minmax_round<3>(m);
  return m[1];
}

// 5x5 median with the reference's border rule (medianFilter.cu:282-318): a tap
// outside the image in one direction is clamped to the edge, a corner tap outside
// in both directions is 0; result = 13th smallest of the 25 taps.
__device__ __forceinline__ float median5_at(const float* __restrict__ in, int ix, int iy, int w, int h, int s) {
  float m[25];
  if (ix >= 2 && iy >= 2 && ix + 2 < w && iy + 2 < h) {  // every tap inside the image
    const float* r0 = in + (ix - 2) + (long long)(iy - 2) * s;
#pragma unroll
    for (int j = 0; j < 5; j++) {
#pragma unroll
      for (int i = 0; i < 5; i++) m[j * 5 + i] = r0[i + (long long)j * s];
    }
  } else {
#pragma unroll
    for (int j = 0; j < 5; j++) {
#pragma unroll
      for (int i = 0; i < 5; i++) {
        int col = ix + i - 2, row = iy + j - 2;
        bool cin = col >= 0 && col < w, rin = row >= 0 && row < h;
        float v = 0.0f;
        if (cin || rin) {
          int cc = min(max(col, 0), w - 1), rr = min(max(row, 0), h - 1);
          v = in[cc + rr * s];
        }
        m[j * 5 + i] = v;
      }
    }
  }
  return median25(m);
}

}  // namespace vfs
