// Per-pixel steps of the fused primal-dual iteration on a region of the state held in shared
// memory, shared by the kernels that run several iterations per launch: the temporally
// blocked tiles (kernels_tb.cu) and the cluster-resident level (kernels_cluster.cu).
//
// The operations, their order and the storage rounding between iterations are those of
// k_fused_iter (dual step, then T p, then threshold and primal step), so every kernel built on
// them gives the bits of the one-iteration launches.  Region pixel i has its east / west
// neighbours at i +- 1 and its south / north neighbours at i +- RX.
#pragma once
#include "fused.cuh"
#include "tgv_pixel.cuh"
#include "tgv_pixel_fast.cuh"

#include <type_traits>

namespace vfs {

// The state of a region of N pixels in shared memory.  float arrays: u-bar, the other
// ping-pong buffer's u-bar, u, the tensor a / b / c, Iu, Iz; T2 (storage type): v-bar, the
// other buffer's v-bar, p; float4: q, kept unrounded (within an iteration the threshold and
// primal steps read this iteration's q at full precision, as the one-iteration kernel does from
// registers and shared memory; the next iteration's dual step reads it in the stored
// precision); float2: T p; u8: the edge code.
template <class ST>
struct RegionState {
  typedef typename Store2<ST>::T2 T2;
  float *ub, *uba, *u, *a, *b, *c, *Iu, *Iz;
  T2 *v, *va, *p;
  float4* q;
  float2* tp;
  uint8_t* code;

  // bytes per region pixel; N a multiple of 4 keeps every array 16-byte aligned
  static constexpr size_t kBytesPerPixel = 8 * sizeof(float) + 3 * sizeof(T2) + sizeof(float4) + sizeof(float2) + 1;

  __device__ __forceinline__ void carve(unsigned char* smem, int N) {
    ub = reinterpret_cast<float*>(smem);
    uba = ub + N;
    u = uba + N;
    a = u + N;
    b = a + N;
    c = b + N;
    Iu = c + N;
    Iz = Iu + N;
    v = reinterpret_cast<T2*>(Iz + N);
    va = v + N;
    p = va + N;
    q = reinterpret_cast<float4*>(p + N);
    tp = reinterpret_cast<float2*>(q + N);
    code = reinterpret_cast<uint8_t*>(tp + N);
  }

  // Load region pixel i from image position (gx, gy) at flat index pos = gx + gy s.
  // Column -1 is the flat position before column 0 (the previous row's last padding element),
  // which the reference reads as the west neighbour of column 0.
  template <bool MASKED>
  __device__ __forceinline__ void load(const IterPair& P, const T2* pin, const typename Store2<ST>::T4* qin, int i,
                                       int gx, int gy) {
    typedef Store2<ST> S;
    const int w = P.w, h = P.h, pos = gx + gy * P.s;
    const bool in = gx >= 0 && gx < w && gy >= 0 && gy < h;
    // flat positions the reference may read: columns [-1, w) of rows < h, at or after the
    // buffer start
    const bool flat = gx >= -1 && gx < w && gy < h && pos >= 0;
    const uint8_t cd = in ? P.code[pos] : (uint8_t)0;
    const bool act = MASKED ? (in && (cd & kOn)) : in;  // written by every iteration
    code[i] = cd;
    ub[i] = flat ? P.u_[pos] : 0.0f;
    v[i] = flat ? ((const T2*)P.v_)[pos] : S::ld2z();
    if (MASKED) {
      uba[i] = (flat && !act) ? P.u_s[pos] : 0.0f;
      va[i] = (flat && !act) ? ((const T2*)P.v_s)[pos] : S::ld2z();
    }
    u[i] = act ? P.u[pos] : 0.0f;
    p[i] = act ? pin[pos] : S::ld2z();
    q[i] = act ? S::cvt4(qin[pos]) : make_float4(0.f, 0.f, 0.f, 0.f);
    a[i] = in ? P.a[pos] : 0.0f;
    b[i] = in ? P.b[pos] : 0.0f;
    c[i] = in ? P.c[pos] : 0.0f;
    Iu[i] = act ? P.Iu[pos] : 0.0f;
    Iz[i] = act ? P.Iz[pos] : 0.0f;
    // stored T p: read where a pixel keeps its values (masked form) and west of column 0
    const bool tps = (MASKED && in && !act) || (gx == -1 && gy >= 1 && gy < h);
    tp[i] = tps ? P.Tp[pos] : make_float2(0.f, 0.f);
  }

  // A pixel that no iteration writes (masked form): its u-bar and v-bar alternate between
  // the values the two ping-pong buffers hold.
  __device__ __forceinline__ void keep(int i) {
    const float t = ub[i];
    ub[i] = uba[i];
    uba[i] = t;
    const T2 tv = v[i];
    v[i] = va[i];
    va[i] = tv;
  }

  // Dual step and T p at region pixel i of image pixel (gx, gy) inside the image.  Returns
  // false for a masked-out pixel of the masked form (it keeps its values; its stored T p is
  // in tp).
  template <bool MASKED>
  __device__ __forceinline__ bool dual(int i, int RX, int gx, int gy, int w, int h, float sp, float sq) {
    typedef Store2<ST> S;
    constexpr bool kFast = !std::is_same<ST, float>::value;
    const uint8_t cd = code[i];
    bool useRight, useDown;
    const float a_ = a[i], b_ = b[i], c_ = c[i];
    if (MASKED) {
      if (!(cd & kOn)) return false;
      useRight = cd & kR;
      useDown = cd & kD;
    } else {
      if (!(cd & kOn)) {  // outside the circle: p = q = 0, T p = T 0
        const float2 z = make_float2(0.f, 0.f);
        p[i] = S::ld2z();
        q[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        tp[i] = kFast ? fast::tp(a_, b_, c_, z) : tp_math(a_, b_, c_, z);
        return true;
      }
      useRight = (gx + 1) < w;
      useDown = (gy + 1) < h;
    }
    const float ubar = ub[i];
    const float2 vb = S::cvt2(v[i]);
    const float u_xn = useRight ? ub[i + 1] : ub[i - 1];
    const float u_yn = useDown ? ub[i + RX] : ub[i - RX];
    const float2 v_xn = S::cvt2(useRight ? v[i + 1] : v[i - 1]);
    const float2 v_yn = S::cvt2(useDown ? v[i + RX] : v[i - RX]);
    float2 pp = S::cvt2(p[i]);
    float4 qq = S::cvt4(S::rnd4(q[i]));  // the stored (rounded) q of the last iteration
    float2 t;
    if (kFast) {
      fast::dual(useRight, useDown, ubar, u_xn, u_yn, vb, v_xn, v_yn, a_, b_, c_, sp, sq, pp, qq);
      t = fast::tp(a_, b_, c_, pp);
    } else {
      dual_math(useRight, useDown, ubar, u_xn, u_yn, vb, v_xn, v_yn, a_, b_, c_, sp, sq, pp, qq);
      t = tp_math(a_, b_, c_, pp);
    }
    p[i] = S::rnd2(pp);
    q[i] = qq;
    tp[i] = t;
    return true;
  }

  // Threshold and primal steps at region pixel i of an active pixel (gx, gy): every pixel of
  // the plain form inside the image, the on pixels of the masked form.
  template <bool MASKED>
  __device__ __forceinline__ void primal(const IterPair& P, int i, int RX, int gx, int gy, float tau, float mu) {
    typedef Store2<ST> S;
    constexpr bool kFast = !std::is_same<ST, float>::value;
    const int w = P.w, h = P.h;
    const uint8_t cd = code[i];
    float dxm, dym;
    bool zR, zD, hasL, hasU;
    const float2 t = tp[i], tpW = tp[i - 1], tpN = tp[i - RX];
    if (MASKED) {
      const bool mR = cd & kR, mL = cd & kL, mD = cd & kD, mU = cd & kU;
      if (mL && mR) dxm = t.x - tpW.x;
      else if (!mR) dxm = -tpW.x;
      else dxm = t.x;
      if (mU && mD) dym = t.y - tpN.y;
      else if (!mD) dym = -tpN.y;
      else dym = t.y;
      zR = !mR;
      zD = !mD;
      hasL = mL;
      hasU = mU;
    } else {
      if (!(cd & kOn)) {
        u[i] = 0.0f;
        ub[i] = 0.0f;
        v[i] = S::rnd2(make_float2(0.f, 0.f));
        return;
      }
      if ((gx - 1) >= 0) dxm = t.x - tpW.x;
      else if (gx == w - 1) dxm = -tpW.x;
      else dxm = t.x;
      if ((gy - 1) >= 0) dym = t.y - tpN.y;
      else if (gy == h - 1) dym = -tpN.y;
      else dym = t.y;
      zR = gx == w - 1;
      zD = gy == h - 1;
      hasL = (gx - 1) >= 0;
      hasU = (gy - 1) >= 0;
    }
    const float a_ = a[i], b_ = b[i], c_ = c[i];
    const float ubar = ub[i];
    const float2 vb = S::cvt2(v[i]);
    float unew;
    if (kFast) {
      float eu = fast::etau(a_, b_, c_, P.alpha1 * P.alpha1);
      unew = fast::threshold(dxm, dym, eu, tau, ubar, u[i], Iu[i], Iz[i], P.lambda);
    } else {
      float eu = etau_math(a_, b_, c_, P.alpha1);
      unew = threshold_math(dxm, dym, eu, tau, ubar, u[i], Iu[i], Iz[i], P.lambda);
    }
    float4 qc = q[i];
    if (zR) qc.x = qc.w = 0.0f;
    if (zD) qc.y = qc.z = 0.0f;
    const float4 ql = hasL ? q[i - 1] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 qu = hasU ? q[i - RX] : make_float4(0.f, 0.f, 0.f, 0.f);
    float us_;
    float2 vs;
    if (kFast) {
      const float a1s = P.alpha1 * P.alpha1, a0s4 = 4.0f * P.alpha0 * P.alpha0;
      float ev1 = fast::etav(b_, c_, a1s, a0s4), ev2 = fast::etav(a_, c_, a1s, a0s4);
      fast::primal(qc, ql, qu, t, ev1, ev2, tau, P.alpha0, P.alpha1, mu, vb, unew, ubar, us_, vs);
    } else {
      float ev1 = etav1_math(b_, c_, P.alpha0, P.alpha1), ev2 = etav2_math(a_, c_, P.alpha0, P.alpha1);
      float2 vo;
      const float2 pp = S::cvt2(p[i]);
      primal_math(qc, ql, qu, pp, a_, b_, c_, ev1, ev2, tau, P.alpha0, P.alpha1, mu, vb, unew, ubar, us_, vs, vo);
    }
    u[i] = unew;
    ub[i] = us_;
    v[i] = S::rnd2(vs);
  }
};

}  // namespace vfs
