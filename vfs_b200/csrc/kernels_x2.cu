// Fused primal-dual iteration with two horizontally adjacent pixels per thread.
//
// The same per-pixel operations, in the same order, as k_fused_iter (kernels_fused.cu), so
// results are bit-identical; the work per pixel is smaller.
//
// Block layout. A block is 32 x (TH + 1) threads over a 64 x (TH + 1) region. Region
// columns 0 and 1 are west halo and column 1 is the only one whose dual step is needed;
// row 0 is the north halo. The tile is 62 x TH pixels. Lane L owns region columns 2L
// (pixel A) and 2L + 1 (pixel B). Tiles start at even columns, so the pair sits at an even
// element position (rows are pitched to 32 elements), and one load or store of twice the
// element size covers both pixels.
//
// Neighbours.
//   * A's east neighbour and B's west neighbour are the thread's own pixels.
//   * A's west (the previous lane's B) and B's east (the next lane's A) come by warp shuffle;
//     lane 31 loads its east neighbour itself.
//   * North and south neighbours are pair loads of the adjacent rows.
//   * After the dual step, the west and north T p and q of the threshold and primal steps
//     come from shared memory (for B's west, from registers).
#include "common.cuh"
#include "fused.cuh"
#include "tgv_pixel.cuh"
#include "tgv_pixel_fast.cuh"

#include <type_traits>

namespace vfs {

namespace {

template <class T>
struct alignas(2 * sizeof(T)) Pair2 {
  T a, b;
};

// base[pos] and base[pos + 1] (pos even, so the pair is aligned to twice the element size);
// a pixel whose predicate is off reads z
template <class T>
__device__ __forceinline__ void ld_pair(const T* base, int pos, bool okA, bool okB, T z, T& a, T& b) {
  if (okA && okB) {
    const Pair2<T> v = *reinterpret_cast<const Pair2<T>*>(base + pos);
    a = v.a;
    b = v.b;
  } else {
    a = okA ? base[pos] : z;
    b = okB ? base[pos + 1] : z;
  }
}

template <class T>
__device__ __forceinline__ void st_pair(T* base, int pos, bool okA, bool okB, T a, T b) {
  if (okA && okB) {
    Pair2<T> v;
    v.a = a;
    v.b = b;
    *reinterpret_cast<Pair2<T>*>(base + pos) = v;
  } else {
    if (okA) base[pos] = a;
    if (okB) base[pos + 1] = b;
  }
}

template <class ST>
struct X2Raw;
template <>
struct X2Raw<float> {
  static __device__ __forceinline__ float2 up(float2 v) {
    return make_float2(__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1));
  }
  static __device__ __forceinline__ float2 down(float2 v) {
    return make_float2(__shfl_down_sync(0xffffffffu, v.x, 1), __shfl_down_sync(0xffffffffu, v.y, 1));
  }
};
template <>
struct X2Raw<__half> {
  static __device__ __forceinline__ __half2 up(__half2 v) { return __shfl_up_sync(0xffffffffu, v, 1); }
  static __device__ __forceinline__ __half2 down(__half2 v) { return __shfl_down_sync(0xffffffffu, v, 1); }
};

// One pixel's values between the dual step and the threshold / primal steps.
struct X2Px {
  float2 pp, tp, vb;
  float4 qq;
  float ubar;
};

// Dual step of one pixel given its neighbours' u-bar / v-bar (zero where the reference
// reads before the buffer start).  Returns whether the pixel stores p and q (false where a
// masked-out pixel keeps its values; its T p is then the stored one).
template <bool MASKED, class ST>
__device__ __forceinline__ bool x2_dual(uint8_t code, int x, int y, int w, int h, float a, float b, float c, float sp,
                                        float sq, float ub, float uW, float uE, float uU, float uD,
                                        typename Store2<ST>::T2 vc, typename Store2<ST>::T2 vW,
                                        typename Store2<ST>::T2 vE, typename Store2<ST>::T2 vU,
                                        typename Store2<ST>::T2 vD, typename Store2<ST>::T2 praw,
                                        typename Store2<ST>::T4 qraw, float2 tps, X2Px& o) {
  typedef Store2<ST> S;
  constexpr bool kFast = !std::is_same<ST, float>::value;
  bool useRight, useDown;
  if (MASKED) {
    if (!(code & kOn)) {
      o.tp = tps;
      return false;
    }
    useRight = code & kR;
    useDown = code & kD;
  } else {
    if (!(code & kOn)) {  // outside the circle: p = q = 0, T p = T 0
      o.pp = make_float2(0.f, 0.f);
      o.qq = make_float4(0.f, 0.f, 0.f, 0.f);
      o.tp = tp_math(a, b, c, o.pp);
      return true;
    }
    useRight = (x + 1) < w;
    useDown = (y + 1) < h;
  }
  o.ubar = ub;
  o.vb = S::cvt2(vc);
  const float u_xn = useRight ? uE : uW;
  const float u_yn = useDown ? uD : uU;
  const float2 v_xn = S::cvt2(useRight ? vE : vW);
  const float2 v_yn = S::cvt2(useDown ? vD : vU);
  o.pp = S::cvt2(praw);
  o.qq = S::cvt4(qraw);
  if (kFast) {
    fast::dual(useRight, useDown, o.ubar, u_xn, u_yn, o.vb, v_xn, v_yn, a, b, c, sp, sq, o.pp, o.qq);
    o.tp = fast::tp(a, b, c, o.pp);
  } else {
    dual_math(useRight, useDown, o.ubar, u_xn, u_yn, o.vb, v_xn, v_yn, a, b, c, sp, sq, o.pp, o.qq);
    o.tp = tp_math(a, b, c, o.pp);
  }
  return true;
}

// Threshold and primal steps of one tile pixel; returns whether it stores u, u-bar, v-bar.
template <bool MASKED, class ST>
__device__ __forceinline__ bool x2_primal(const IterArgs& A, const IterPair& P, uint8_t code, int x, int y, float a,
                                          float b, float c, const X2Px& o, float2 tpW, float4 qW, float2 tpN,
                                          float4 qN, float u, float Iu, float Iz, float& unew, float& us_,
                                          float2& vs) {
  constexpr bool kFast = !std::is_same<ST, float>::value;
  float dxm, dym;
  bool zR, zD, hasL, hasU;
  const float2 tp = o.tp;
  if (MASKED) {
    if (!(code & kOn)) return false;
    const bool mR = code & kR, mL = code & kL, mD = code & kD, mU = code & kU;
    if (mL && mR) dxm = tp.x - tpW.x;
    else if (!mR) dxm = -tpW.x;
    else dxm = tp.x;
    if (mU && mD) dym = tp.y - tpN.y;
    else if (!mD) dym = -tpN.y;
    else dym = tp.y;
    zR = !mR;
    zD = !mD;
    hasL = mL;
    hasU = mU;
  } else {
    if (!(code & kOn)) {
      unew = 0.0f;
      us_ = 0.0f;
      vs = make_float2(0.f, 0.f);
      return true;
    }
    if ((x - 1) >= 0) dxm = tp.x - tpW.x;
    else if (x == P.w - 1) dxm = -tpW.x;
    else dxm = tp.x;
    if ((y - 1) >= 0) dym = tp.y - tpN.y;
    else if (y == P.h - 1) dym = -tpN.y;
    else dym = tp.y;
    zR = x == P.w - 1;
    zD = y == P.h - 1;
    hasL = (x - 1) >= 0;
    hasU = (y - 1) >= 0;
  }
  if (kFast) {
    float eu = fast::etau(a, b, c, P.alpha1 * P.alpha1);
    unew = fast::threshold(dxm, dym, eu, A.tau, o.ubar, u, Iu, Iz, P.lambda);
  } else {
    float eu = etau_math(a, b, c, P.alpha1);
    unew = threshold_math(dxm, dym, eu, A.tau, o.ubar, u, Iu, Iz, P.lambda);
  }
  float4 qc = o.qq;
  if (zR) qc.x = qc.w = 0.0f;
  if (zD) qc.y = qc.z = 0.0f;
  const float4 ql = hasL ? qW : make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 qu = hasU ? qN : make_float4(0.f, 0.f, 0.f, 0.f);
  if (kFast) {
    const float a1s = P.alpha1 * P.alpha1, a0s4 = 4.0f * P.alpha0 * P.alpha0;
    float ev1 = fast::etav(b, c, a1s, a0s4), ev2 = fast::etav(a, c, a1s, a0s4);
    fast::primal(qc, ql, qu, tp, ev1, ev2, A.tau, P.alpha0, P.alpha1, A.mu, o.vb, unew, o.ubar, us_, vs);
  } else {
    float ev1 = etav1_math(b, c, P.alpha0, P.alpha1), ev2 = etav2_math(a, c, P.alpha0, P.alpha1);
    float2 vo;
    primal_math(qc, ql, qu, o.pp, a, b, c, ev1, ev2, A.tau, P.alpha0, P.alpha1, A.mu, o.vb, unew, o.ubar, us_, vs,
                vo);
  }
  return true;
}

}  // namespace

template <bool MASKED, class ST, int TH, int MINB>
__global__ void __launch_bounds__(32 * (TH + 1), MINB) k_fused_iter_x2(const __grid_constant__ IterArgs A, int parity) {
  typedef Store2<ST> S;
  typedef typename S::T2 T2;
  typedef typename S::T4 T4;
  typedef X2Raw<ST> RW;
  __shared__ __align__(16) float2 sTp[TH + 1][64];
  __shared__ __align__(16) float4 sQ[TH + 1][64];
  const IterPair& P = A.pr[0];
  const int w = P.w, h = P.h, s = P.s;
  const int L = threadIdx.x, ry = threadIdx.y;
  const int xa = (int)blockIdx.x * 62 - 2 + 2 * L, xb = xa + 1;
  const int iy = (int)blockIdx.y * TH - 1 + ry;
  const int plane = s * h;
  const T2* pin = (const T2*)P.p + (parity ? plane : 0);
  const T4* qin = (const T4*)P.q + (parity ? plane : 0);
  T2* pout = (T2*)P.p + (parity ? 0 : plane);
  T4* qout = (T4*)P.q + (parity ? 0 : plane);
  const T2* vbar = (const T2*)P.v_;
  const bool rowin = iy >= 0 && iy < h;
  const bool inA = rowin && xa >= 0 && xa < w, inB = rowin && xb >= 0 && xb < w;
  const int pos = xa + iy * s;  // A's position (even); B is at pos + 1
  const bool tile = L >= 1 && ry >= 1;
  griddep_wait();  // the previous iteration's outputs are this one's inputs
  griddep_launch_dependents();

  // ---- first load round: edge codes and tensor ----------------------------------------------
  uint8_t cA, cB;
  float aA, aB, bA, bB, ccA, ccB;
  ld_pair(P.code, pos, inA, inB, (uint8_t)0, cA, cB);
  ld_pair(P.a, pos, inA, inB, 0.0f, aA, aB);
  ld_pair(P.b, pos, inA, inB, 0.0f, bA, bB);
  ld_pair(P.c, pos, inA, inB, 0.0f, ccA, ccB);
  // masked form: a block with no pixel on in its region writes nothing and reads nothing
  // another block needs, so it leaves here
  if (MASKED && !__syncthreads_or((inA && (cA & kOn)) || (inB && (cB & kOn)))) return;

  // ---- second load round --------------------------------------------------------------------
  // the dual step runs at A for lanes >= 1 (region column >= 2) and at B for every lane
  const bool dA = inA && L >= 1, dB = inB;
  const bool fullA = dA && (cA & kOn), fullB = dB && (cB & kOn);  // the full dual update
  const bool thA = fullA && tile, thB = fullB && tile;             // the threshold step
  // u-bar / v-bar at flat positions: columns [-1, w) of rows < h, positions >= 0
  auto flat = [&](int x, int y, int p) { return x >= -1 && x < w && y < h && p >= 0; };
  const bool fA = flat(xa, iy, pos), fB = flat(xb, iy, pos + 1);
  const bool fAu = flat(xa, iy - 1, pos - s), fBu = flat(xb, iy - 1, pos + 1 - s);
  const bool fAd = flat(xa, iy + 1, pos + s), fBd = flat(xb, iy + 1, pos + 1 + s);
  float ubA, ubB, uuA, uuB, udA, udB;
  ld_pair(P.u_, pos, fA, fB, 0.0f, ubA, ubB);
  ld_pair(P.u_, pos - s, fAu, fBu, 0.0f, uuA, uuB);
  ld_pair(P.u_, pos + s, fAd, fBd, 0.0f, udA, udB);
  T2 vA, vB, vuA, vuB, vdA, vdB;
  ld_pair(vbar, pos, fA, fB, S::ld2z(), vA, vB);
  ld_pair(vbar, pos - s, fAu, fBu, S::ld2z(), vuA, vuB);
  ld_pair(vbar, pos + s, fAd, fBd, S::ld2z(), vdA, vdB);
  float ueE = 0.0f;  // lane 31: B's east neighbour
  T2 veE = S::ld2z();
  if (L == 31 && flat(xb + 1, iy, pos + 2)) {
    ueE = P.u_[pos + 2];
    veE = vbar[pos + 2];
  }
  T2 pA, pB;
  T4 qA, qB;
  ld_pair(pin, pos, fullA, fullB, S::ld2z(), pA, pB);
  ld_pair(qin, pos, fullA, fullB, S::ld4z(), qA, qB);
  float uA, uB, IuA, IuB, IzA, IzB;
  ld_pair(P.u, pos, thA, thB, 0.0f, uA, uB);
  ld_pair(P.Iu, pos, thA, thB, 0.0f, IuA, IuB);
  ld_pair(P.Iz, pos, thA, thB, 0.0f, IzA, IzB);
  // stored T p: masked-out pixels (masked form) and the flat position west of column 0
  const bool tsA = MASKED && dA && !(cA & kOn);
  const bool tsB = (MASKED && dB && !(cB & kOn)) || (xb == -1 && iy >= 1 && iy < h);
  float2 tsvA, tsvB;
  ld_pair(P.Tp, pos, tsA, tsB, make_float2(0.f, 0.f), tsvA, tsvB);

  // west / east neighbours across lanes (every lane takes part in every shuffle)
  const float uWs = __shfl_up_sync(0xffffffffu, ubB, 1);
  const float uEs = __shfl_down_sync(0xffffffffu, ubA, 1);
  const T2 vWs = RW::up(vB), vEs = RW::down(vA);
  const float uE_B = L == 31 ? ueE : uEs;
  const T2 vE_B = L == 31 ? veE : vEs;

  // ---- dual step at A and B ----------------------------------------------------------------
  X2Px oA, oB;
  oA.pp = oA.tp = oA.vb = oB.pp = oB.tp = oB.vb = make_float2(0.f, 0.f);
  oA.qq = oB.qq = make_float4(0.f, 0.f, 0.f, 0.f);
  oA.ubar = oB.ubar = 0.0f;
  const float sp = A.sp[0], sq = A.sq[0];
  bool ownA = false, ownB = false;
  if (dA)
    ownA = x2_dual<MASKED, ST>(cA, xa, iy, w, h, aA, bA, ccA, sp, sq, ubA, uWs, ubB, uuA, udA, vA, vWs, vB, vuA, vdA,
                               pA, qA, tsvA, oA);
  if (dB)
    ownB = x2_dual<MASKED, ST>(cB, xb, iy, w, h, aB, bB, ccB, sp, sq, ubB, ubA, uE_B, uuB, udB, vB, vA, vE_B, vuB, vdB,
                               pB, qB, tsvB, oB);
  else if (xb == -1 && iy >= 1 && iy < h)
    oB.tp = tsvB;  // west of column 0: the previous row's last padding element
  {
    const bool sA = ownA && tile, sB = ownB && tile;
    st_pair(pout, pos, sA, sB, S::rnd2(oA.pp), S::rnd2(oB.pp));
    st_pair(qout, pos, sA, sB, S::rnd4(oA.qq), S::rnd4(oB.qq));
    if (A.write_tp) st_pair(P.Tp, pos, sA, sB, oA.tp, oB.tp);
  }
  *reinterpret_cast<float4*>(&sTp[ry][2 * L]) = make_float4(oA.tp.x, oA.tp.y, oB.tp.x, oB.tp.y);
  sQ[ry][2 * L] = oA.qq;
  sQ[ry][2 * L + 1] = oB.qq;
  __syncthreads();
  if (!tile) return;

  // ---- threshold and primal steps at the tile pixels -----------------------------------------
  float unA = 0.f, unB = 0.f, usA = 0.f, usB = 0.f;
  float2 vsA = make_float2(0.f, 0.f), vsB = make_float2(0.f, 0.f);
  bool wA = false, wB = false;
  const float4 tpN = *reinterpret_cast<const float4*>(&sTp[ry - 1][2 * L]);
  if (inA)
    wA = x2_primal<MASKED, ST>(A, P, cA, xa, iy, aA, bA, ccA, oA, sTp[ry][2 * L - 1], sQ[ry][2 * L - 1],
                               make_float2(tpN.x, tpN.y), sQ[ry - 1][2 * L], uA, IuA, IzA, unA, usA, vsA);
  if (inB)
    wB = x2_primal<MASKED, ST>(A, P, cB, xb, iy, aB, bB, ccB, oB, oA.tp, oA.qq, make_float2(tpN.z, tpN.w),
                               sQ[ry - 1][2 * L + 1], uB, IuB, IzB, unB, usB, vsB);
  st_pair(P.us, pos, wA, wB, unA, unB);
  st_pair(P.u_s, pos, wA, wB, usA, usB);
  st_pair((T2*)P.v_s, pos, wA, wB, S::rnd2(vsA), S::rnd2(vsB));
}

namespace {

template <int TH, int MINB>
void launch_x2_th(const IterArgs& A, bool masked, bool half_storage, cudaStream_t st, int parity) {
  const dim3 blk(32, TH + 1), grid((A.pr[0].w + 61) / 62, (A.pr[0].h + TH - 1) / TH);
  if (masked) {
    if (half_storage) launch_overlapped(k_fused_iter_x2<true, __half, TH, MINB>, grid, blk, st, A, parity);
    else launch_overlapped(k_fused_iter_x2<true, float, TH, MINB>, grid, blk, st, A, parity);
  } else {
    if (half_storage) launch_overlapped(k_fused_iter_x2<false, __half, TH, MINB>, grid, blk, st, A, parity);
    else launch_overlapped(k_fused_iter_x2<false, float, TH, MINB>, grid, blk, st, A, parity);
  }
}

template <int TH, int MINB>
int x2_blocks_per_sm(bool masked, bool half) {
  int n = 0;
  const int threads = 32 * (TH + 1);
  if (masked) {
    if (half) VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_x2<true, __half, TH, MINB>, threads, 0));
    else VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_x2<true, float, TH, MINB>, threads, 0));
  } else {
    if (half) VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_x2<false, __half, TH, MINB>, threads, 0));
    else VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_x2<false, float, TH, MINB>, threads, 0));
  }
  return n;
}

}  // namespace

void launch_fused_iteration_x2(const IterArgs& A, bool masked, bool half_storage, cudaStream_t st, int parity,
                               int variant) {
  if (A.npairs != 1) throw ArgError{"the two-pixel iteration form takes one pair per launch"};
  if (A.pr[0].w <= 0 || A.pr[0].h <= 0) return;
  if (variant == kIterFirstX2Variant) launch_x2_th<8, 3>(A, masked, half_storage, st, parity);
  else launch_x2_th<4, 6>(A, masked, half_storage, st, parity);
  VFS_LAUNCH_CHECK();
}

double x2_gpu_share(int variant, bool masked, bool half, int w, int h) {
  const int TH = variant == kIterFirstX2Variant ? 8 : 4;
  const int per_sm = variant == kIterFirstX2Variant ? x2_blocks_per_sm<8, 3>(masked, half)
                                                    : x2_blocks_per_sm<4, 6>(masked, half);
  const long long blocks = (long long)((w + 61) / 62) * ((h + TH - 1) / TH);
  int dev = 0, sms = 1;
  VFS_CUDA(cudaGetDevice(&dev));
  VFS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const double cap = (double)sms * (per_sm > 0 ? per_sm : 1);
  return blocks >= cap ? 1.0 : (double)blocks / cap;
}

}  // namespace vfs
