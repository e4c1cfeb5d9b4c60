// Row-streaming form of the fused primal-dual iteration.
//
// The same per-pixel operations, in the same order, as k_fused_iter (kernels_fused.cu),
// so the two forms give bit-identical results; only the way a block reaches its
// neighbours differs.  A warp owns a strip of 31 columns (its lane 0 is the west halo
// column) and walks down R rows plus one north halo row:
//   * west / east neighbours of u-bar and v-bar come from the adjacent lanes by warp
//     shuffle (the two strip-edge lanes load their outer neighbour themselves);
//   * north / south neighbours stay in registers from the previous / next row;
//   * T p and q of the west neighbour come by shuffle after the dual step, those of the
//     north neighbour from the previous row's registers;
//   * every global load is issued one row before it is used (u-bar, v-bar and the edge
//     codes two rows before), so the loads of the next row are in flight while the
//     current row computes.
// There is no shared memory and no barrier; warps are independent.
#include "common.cuh"
#include "fused.cuh"
#include "tgv_pixel.cuh"
#include "tgv_pixel_fast.cuh"

#include <type_traits>

namespace vfs {

namespace {

constexpr int kRowWarps = 4;  // warps (independent strips) per block

// raw storage registers of a 2-vector and a 4-vector, and their shuffles / widening
template <class ST>
struct Raw;
template <>
struct Raw<float> {
  typedef float2 T2;
  typedef float4 T4;
  static __device__ __forceinline__ float2 zero2() { return make_float2(0.f, 0.f); }
  static __device__ __forceinline__ float4 zero4() { return make_float4(0.f, 0.f, 0.f, 0.f); }
  static __device__ __forceinline__ float2 f2(float2 v) { return v; }
  static __device__ __forceinline__ float4 f4(float4 v) { return v; }
  static __device__ __forceinline__ float2 up(float2 v) {
    return make_float2(__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1));
  }
  static __device__ __forceinline__ float2 down(float2 v) {
    return make_float2(__shfl_down_sync(0xffffffffu, v.x, 1), __shfl_down_sync(0xffffffffu, v.y, 1));
  }
};
template <>
struct Raw<__half> {
  typedef __half2 T2;
  typedef Store2<__half>::T4 T4;
  static __device__ __forceinline__ __half2 zero2() { return __floats2half2_rn(0.f, 0.f); }
  static __device__ __forceinline__ T4 zero4() {
    T4 t;
    t.a = zero2();
    t.b = zero2();
    return t;
  }
  static __device__ __forceinline__ float2 f2(__half2 v) { return __half22float2(v); }
  static __device__ __forceinline__ float4 f4(T4 v) {
    float2 x = __half22float2(v.a), y = __half22float2(v.b);
    return make_float4(x.x, x.y, y.x, y.y);
  }
  static __device__ __forceinline__ __half2 up(__half2 v) { return __shfl_up_sync(0xffffffffu, v, 1); }
  static __device__ __forceinline__ __half2 down(__half2 v) { return __shfl_down_sync(0xffffffffu, v, 1); }
};

__device__ __forceinline__ float2 shfl_up2(float2 v) {
  return make_float2(__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1));
}
__device__ __forceinline__ float4 shfl_up4(float4 v) {
  return make_float4(__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1),
                     __shfl_up_sync(0xffffffffu, v.z, 1), __shfl_up_sync(0xffffffffu, v.w, 1));
}

// values of one row at one lane's column, loaded a row ahead
template <class ST>
struct RowVals {
  typename Raw<ST>::T2 p;
  typename Raw<ST>::T4 q;
  float a, b, c, u, Iu, Iz;
  float2 tps;  // stored T p (read where the pixel keeps its values, and west of column 0)
};

}  // namespace

// R: output rows per warp.  SINGLE: the launch carries one pair.
template <bool MASKED, class ST, int R, bool SINGLE>
__global__ void __launch_bounds__(32 * kRowWarps) k_fused_iter_rows(const __grid_constant__ IterArgs A, int parity) {
  typedef Raw<ST> RW;
  typedef typename RW::T2 T2;
  typedef typename RW::T4 T4;
  typedef Store2<ST> S;
  constexpr bool kFast = !std::is_same<ST, float>::value;
  const int lane = threadIdx.x & 31;
  const int unit = blockIdx.x * kRowWarps + (int)(threadIdx.x >> 5);
  if (unit >= A.ntiles) return;  // whole warps leave together
  const int pi = SINGLE ? 0 : find_pair(A.pr, A.npairs, unit);
  const IterPair& P = A.pr[pi];
  const int lu = unit - P.tile0;
  const int x0 = (lu % P.tiles_x) * 31;
  const int y0 = (lu / P.tiles_x) * R;
  const int w = P.w, h = P.h, s = P.s;
  const int x = x0 - 1 + lane;
  const int plane = s * h;
  const T2* pin = (const T2*)P.p + (parity ? plane : 0);
  const T4* qin = (const T4*)P.q + (parity ? plane : 0);
  T2* pout = (T2*)P.p + (parity ? 0 : plane);
  T4* qout = (T4*)P.q + (parity ? 0 : plane);
  const T2* vbar = (const T2*)P.v_;
  const float sp = A.sp[pi], sq = A.sq[pi];
  // the column whose value this lane loads for its strip-edge neighbour (lane 0: west,
  // lane 31: east); other lanes load nothing extra
  const bool edge = lane == 0 || lane == 31;
  const int xe = lane == 0 ? x - 1 : x + 1;
  const bool xin = x >= 0 && x < w;
  griddep_wait();  // the previous iteration's outputs are this one's inputs
  griddep_launch_dependents();

  // A flat position is loaded when its column is in [-1, w) and it lies in [0, s * h):
  // the reference reads the flat neighbour before column 0 (the previous row's last
  // padding element) and treats positions before the buffer start as 0.
  auto okpos = [&](int xx, int r) { return xx >= -1 && xx < w && r < h && xx + r * s >= 0; };
  auto ld_ubar = [&](int xx, int r) { return okpos(xx, r) ? P.u_[xx + r * s] : 0.0f; };
  auto ld_vbar = [&](int xx, int r) { return okpos(xx, r) ? vbar[xx + r * s] : RW::zero2(); };
  auto ld_code = [&](int r) -> int { return (xin && r >= 0 && r < h) ? (int)P.code[x + r * s] : 0; };
  auto ld_row = [&](int r, int code, RowVals<ST>& v) {
    const bool in = xin && r >= 0 && r < h;
    const int pos = x + r * s;
    v.p = in ? pin[pos] : RW::zero2();
    v.q = in ? qin[pos] : RW::zero4();
    v.a = in ? P.a[pos] : 0.0f;
    v.b = in ? P.b[pos] : 0.0f;
    v.c = in ? P.c[pos] : 0.0f;
    v.u = in ? P.u[pos] : 0.0f;
    v.Iu = in ? P.Iu[pos] : 0.0f;
    v.Iz = in ? P.Iz[pos] : 0.0f;
    // stored T p: at masked-out pixels (masked form), and west of column 0 (rows >= 1)
    const bool tps = (MASKED && in && !(code & kOn)) || (x == -1 && r >= 1 && r < h);
    v.tps = tps ? P.Tp[pos] : make_float2(0.f, 0.f);
  };

  // ---- prologue: rows y0-2 .. y0 of u-bar / v-bar, codes of rows y0-1 and y0, the
  // other values of row y0-1 --------------------------------------------------------
  int r = y0 - 1;
  float um = ld_ubar(x, r - 1), uc = ld_ubar(x, r), ud = ld_ubar(x, r + 1);
  T2 vm = ld_vbar(x, r - 1), vc = ld_vbar(x, r), vd = ld_vbar(x, r + 1);
  float ue = 0.0f;
  T2 ve = RW::zero2();
  if (edge) {
    ue = ld_ubar(xe, r);
    ve = ld_vbar(xe, r);
  }
  int code = ld_code(r), code1 = ld_code(r + 1);
  RowVals<ST> cur;
  ld_row(r, code, cur);
  float2 tpU = make_float2(0.f, 0.f);
  float4 qU = make_float4(0.f, 0.f, 0.f, 0.f);

  const int rend = min(y0 + R, h);  // rows below the image are never read
  for (; r < rend; r++) {
    // ---- loads for the next rows ----------------------------------------------------
    const float un2 = ld_ubar(x, r + 2);
    const T2 vn2 = ld_vbar(x, r + 2);
    const int code2 = ld_code(r + 2);
    float ue1 = 0.0f;
    T2 ve1 = RW::zero2();
    if (edge) {
      ue1 = ld_ubar(xe, r + 1);
      ve1 = ld_vbar(xe, r + 1);
    }
    RowVals<ST> nxt;
    ld_row(r + 1, code1, nxt);

    // ---- dual step at (x, r) (lane 0 and row y0 - 1 are halo) ----------------------
    const bool in_img = xin && r >= 0;
    const int pos = x + r * s;
    // every shuffle is executed by all 32 lanes (full mask); the strip-edge lanes then
    // replace the value with the one they loaded
    const float uWs = __shfl_up_sync(0xffffffffu, uc, 1);
    const float uEs = __shfl_down_sync(0xffffffffu, uc, 1);
    const T2 vWs = RW::up(vc), vEs = RW::down(vc);
    const float uW = lane == 0 ? ue : uWs;
    const float uE = lane == 31 ? ue : uEs;
    const T2 vW = lane == 0 ? ve : vWs;
    const T2 vE = lane == 31 ? ve : vEs;
    const bool tile = lane >= 1 && r >= y0;

    float2 pp = make_float2(0.f, 0.f), tp = make_float2(0.f, 0.f), vb = make_float2(0.f, 0.f);
    float4 qq = make_float4(0.f, 0.f, 0.f, 0.f);
    float ubar = 0.0f;
    if (in_img) {
      bool own = true, compute = true;
      bool useRight = false, useDown = false;
      if (MASKED) {
        if (!(code & kOn)) {
          tp = cur.tps;
          own = compute = false;
        } else {
          useRight = code & kR;
          useDown = code & kD;
        }
      } else {
        if (!(code & kOn)) {  // outside the circle: p = q = 0, T p = T 0
          tp = tp_math(cur.a, cur.b, cur.c, pp);
          compute = false;
        } else {
          useRight = (x + 1) < w;
          useDown = (r + 1) < h;
        }
      }
      if (compute) {
        ubar = uc;
        vb = RW::f2(vc);
        const float u_xn = useRight ? uE : uW;
        const float u_yn = useDown ? ud : um;
        const float2 v_xn = RW::f2(useRight ? vE : vW);
        const float2 v_yn = RW::f2(useDown ? vd : vm);
        pp = RW::f2(cur.p);
        qq = RW::f4(cur.q);
        if (kFast) {
          fast::dual(useRight, useDown, ubar, u_xn, u_yn, vb, v_xn, v_yn, cur.a, cur.b, cur.c, sp, sq, pp, qq);
          tp = fast::tp(cur.a, cur.b, cur.c, pp);
        } else {
          dual_math(useRight, useDown, ubar, u_xn, u_yn, vb, v_xn, v_yn, cur.a, cur.b, cur.c, sp, sq, pp, qq);
          tp = tp_math(cur.a, cur.b, cur.c, pp);
        }
      }
      if (own && tile) {
        S::st2(pout, pos, pp);
        S::st4(qout, pos, qq);
        if (A.write_tp) P.Tp[pos] = tp;
      }
    } else if (x == -1 && r >= 1) {
      tp = cur.tps;  // west neighbour of column 0: the previous row's last padding element
    }
    const float2 tpW = shfl_up2(tp);
    const float4 qW = shfl_up4(qq);

    // ---- threshold and primal steps at the tile pixels ----------------------------
    if (tile && in_img) {
      float dxm = 0.f, dym = 0.f;
      bool zR = false, zD = false, hasL = false, hasU = false, go = true;
      if (MASKED) {
        if (!(code & kOn)) {
          go = false;
        } else {
          const bool mR = code & kR, mL = code & kL, mD = code & kD, mU = code & kU;
          if (mL && mR) dxm = tp.x - tpW.x;
          else if (!mR) dxm = -tpW.x;
          else dxm = tp.x;
          if (mU && mD) dym = tp.y - tpU.y;
          else if (!mD) dym = -tpU.y;
          else dym = tp.y;
          zR = !mR;
          zD = !mD;
          hasL = mL;
          hasU = mU;
        }
      } else {
        if (!(code & kOn)) {
          P.us[pos] = 0.0f;
          P.u_s[pos] = 0.0f;
          S::st2((T2*)P.v_s, pos, make_float2(0.f, 0.f));
          go = false;
        } else {
          if ((x - 1) >= 0) dxm = tp.x - tpW.x;
          else if (x == w - 1) dxm = -tpW.x;
          else dxm = tp.x;
          if ((r - 1) >= 0) dym = tp.y - tpU.y;
          else if (r == h - 1) dym = -tpU.y;
          else dym = tp.y;
          zR = x == w - 1;
          zD = r == h - 1;
          hasL = (x - 1) >= 0;
          hasU = (r - 1) >= 0;
        }
      }
      if (go) {
        const float a = cur.a, b = cur.b, c = cur.c;
        float unew;
        if (kFast) {
          float eu = fast::etau(a, b, c, P.alpha1 * P.alpha1);
          unew = fast::threshold(dxm, dym, eu, A.tau, ubar, cur.u, cur.Iu, cur.Iz, P.lambda);
        } else {
          float eu = etau_math(a, b, c, P.alpha1);
          unew = threshold_math(dxm, dym, eu, A.tau, ubar, cur.u, cur.Iu, cur.Iz, P.lambda);
        }
        P.us[pos] = unew;
        float4 qc = qq;
        if (zR) qc.x = qc.w = 0.0f;
        if (zD) qc.y = qc.z = 0.0f;
        const float4 ql = hasL ? qW : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 qu = hasU ? qU : make_float4(0.f, 0.f, 0.f, 0.f);
        float us_;
        float2 vs;
        if (kFast) {
          const float a1s = P.alpha1 * P.alpha1, a0s4 = 4.0f * P.alpha0 * P.alpha0;
          float ev1 = fast::etav(b, c, a1s, a0s4), ev2 = fast::etav(a, c, a1s, a0s4);
          fast::primal(qc, ql, qu, tp, ev1, ev2, A.tau, P.alpha0, P.alpha1, A.mu, vb, unew, ubar, us_, vs);
        } else {
          float ev1 = etav1_math(b, c, P.alpha0, P.alpha1), ev2 = etav2_math(a, c, P.alpha0, P.alpha1);
          float2 vo;
          primal_math(qc, ql, qu, pp, a, b, c, ev1, ev2, A.tau, P.alpha0, P.alpha1, A.mu, vb, unew, ubar, us_, vs,
                      vo);
        }
        P.u_s[pos] = us_;
        S::st2((T2*)P.v_s, pos, vs);
      }
    }

    // ---- advance one row ---------------------------------------------------------------
    tpU = tp;
    qU = qq;
    um = uc;
    uc = ud;
    ud = un2;
    vm = vc;
    vc = vd;
    vd = vn2;
    ue = ue1;
    ve = ve1;
    code = code1;
    code1 = code2;
    cur = nxt;
  }
}

template <int R, bool SINGLE>
static void launch_rows2(const IterArgs& A, bool masked, bool half_storage, cudaStream_t st, int parity) {
  const dim3 grid((A.ntiles + kRowWarps - 1) / kRowWarps), blk(32 * kRowWarps);
  if (masked) {
    if (half_storage) launch_overlapped(k_fused_iter_rows<true, __half, R, SINGLE>, grid, blk, st, A, parity);
    else launch_overlapped(k_fused_iter_rows<true, float, R, SINGLE>, grid, blk, st, A, parity);
  } else {
    if (half_storage) launch_overlapped(k_fused_iter_rows<false, __half, R, SINGLE>, grid, blk, st, A, parity);
    else launch_overlapped(k_fused_iter_rows<false, float, R, SINGLE>, grid, blk, st, A, parity);
  }
}

template <int R>
static void launch_rows(const IterArgs& A, bool masked, bool half_storage, cudaStream_t st, int parity) {
  if (A.npairs == 1) launch_rows2<R, true>(A, masked, half_storage, st, parity);
  else launch_rows2<R, false>(A, masked, half_storage, st, parity);
}

namespace {
template <int R>
int rows_blocks_per_sm(bool masked, bool half) {
  int n = 0;
  const int threads = 32 * kRowWarps;
  if (masked) {
    if (half) VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_rows<true, __half, R, true>, threads, 0));
    else VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_rows<true, float, R, true>, threads, 0));
  } else {
    if (half) VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_rows<false, __half, R, true>, threads, 0));
    else VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_rows<false, float, R, true>, threads, 0));
  }
  return n;
}
}  // namespace

double rows_gpu_share(int variant, bool masked, bool half, int w, int h) {
  const int R = kIterVariantRows[variant];
  const long long blocks = ((long long)iter_tiles_of(w, h, R) + kRowWarps - 1) / kRowWarps;
  int per_sm = R == 8 ? rows_blocks_per_sm<8>(masked, half) : R == 32 ? rows_blocks_per_sm<32>(masked, half)
                                                                     : rows_blocks_per_sm<16>(masked, half);
  int dev = 0, sms = 1;
  VFS_CUDA(cudaGetDevice(&dev));
  VFS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const double cap = (double)sms * (per_sm > 0 ? per_sm : 1);
  return blocks >= cap ? 1.0 : (double)blocks / cap;
}

void launch_fused_iteration_rows(const IterArgs& A, bool masked, bool half_storage, cudaStream_t st, int parity,
                                 int rows) {
  if (A.ntiles <= 0) return;
  switch (rows) {
    case 8: launch_rows<8>(A, masked, half_storage, st, parity); break;
    case 32: launch_rows<32>(A, masked, half_storage, st, parity); break;
    default: launch_rows<16>(A, masked, half_storage, st, parity); break;
  }
  VFS_LAUNCH_CHECK();
}

}  // namespace vfs
