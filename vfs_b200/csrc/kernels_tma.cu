// Persistent, TMA-pipelined form of the one-iteration fused primal-dual kernel (iteration
// variant 18).
//
// Geometry.  Tiles are those of k_fused_iter with 8-row tiles (variant 1): 31 columns by 8 rows,
// x0 = 31 * tile column, y0 = 8 * tile row.  A block of 256 threads (32 x 8) runs the dual step
// (updateDualVariables.cu:122-237) at the tile's 8 rows plus the west halo column x0 - 1, then,
// after a barrier, the threshold and primal steps (thresholdingL1.cu:128-228,
// updatePrimalVariables.cu:139-245) at the tile pixels with the west / north T p and q from
// shared memory.  The per-pixel arithmetic is the code of tgv_pixel.cuh / tgv_pixel_fast.cuh,
// so the results are bit-identical to the other variants.
//
// Work.  The host cuts every column of active tiles into segments of consecutive tile rows
// (tma_segments).  Each block is persistent over the segments blockIdx.x, blockIdx.x + gridDim.x,
// ..., and walks each segment downwards.  The north halo row of a tile (row y0 - 1) is the last
// row of the tile above, whose dual results (T p, q) the block still holds in shared memory; it
// is recomputed (by one warp) only for the first tile of a segment.
//
// Staging.  One thread brings the region of every input plane that a tile needs into shared
// memory with eleven 2-D bulk tensor copies (cp.async.bulk.tensor, TMA) completing on an
// mbarrier.  There are two stages: while the block computes one tile from one stage, the copies
// of its next tile fill the other.  The threads sleep on the mbarrier (try_wait with a suspend
// hint) instead of spinning, and every wait is bounded: if the copies have not landed after
// kMaxWaits waits, the block records it in g_tma_status (vfs_device_status), waits once more
// for copies still in flight, and leaves.
//
// Copy boxes (x in pixels; a box starts on a 16-byte boundary, as TMA requires, so its start is
// rounded down and the box is wider than the region):
//   u-bar, v-bar        x from (x0 - 2) & ~3, 40 wide, rows y0 - 2 .. y0 + 8
//   tensor a b c, p, q  x from (x0 - 2) & ~3, 40 wide, rows y0 - 1 .. y0 + 7
//   u, Iu, Iz           x from (x0 - 2) & ~3, 40 wide, rows y0 .. y0 + 7
//   edge codes (bytes)  x from (x0 - 1) & ~15, 48 wide, rows y0 - 1 .. y0 + 7
// Coordinates outside the image read 0 (the tensor maps' out-of-bounds fill), which is also
// what the drop-in kernels read before a buffer's start (row -1).  West of column 0 the
// reference reads the flat position before it (the previous row's last element); the caller
// uses this kernel on a masked level only when no pixel of column 0 is on
// (StereoTgvImpl::tma_ok), so no pixel reads there.  The stale T p of masked-out pixels is read
// from global memory, as in k_fused_iter.
//
// The tensor maps describe this GPU's own buffers only; no copy uses cluster multicast.
#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "fused.cuh"
#include "tgv_pixel.cuh"
#include "tgv_pixel_fast.cuh"

namespace vfs {

namespace {

constexpr int kTH = 8;           // tile rows (the geometry of variant 1)
constexpr int kThreads = 32 * kTH;
constexpr int kBW = 40;          // pixels per box row of the 4-, 8- and 16-byte planes
constexpr int kCodeW = 48;       // bytes per box row of the edge codes
constexpr int kMaxWaits = 4096;  // bounded mbarrier waits (each sleeps up to kSuspendNs)
constexpr uint32_t kSuspendNs = 1000000;

__device__ int g_tma_status;  // 0 = fine; 1 = an mbarrier wait ran out

// One stage: the regions of every input plane of one tile, as the copies lay them out (rows of
// the box width, no padding).
template <class ST>
struct TmaStage {
  typedef typename Store2<ST>::T2 T2;
  typedef typename Store2<ST>::T4 T4;
  alignas(128) uint8_t code[kTH + 1][kCodeW];
  alignas(128) float a[kTH + 1][kBW];
  alignas(128) float b[kTH + 1][kBW];
  alignas(128) float c[kTH + 1][kBW];
  alignas(128) T2 p[kTH + 1][kBW];
  alignas(128) T4 q[kTH + 1][kBW];
  alignas(128) float ub[kTH + 3][kBW];  // u-bar
  alignas(128) T2 vb[kTH + 3][kBW];     // v-bar
  alignas(128) float u[kTH][kBW];
  alignas(128) float Iu[kTH][kBW];
  alignas(128) float Iz[kTH][kBW];
  static constexpr uint32_t kBytes =
      (uint32_t)(sizeof(code) + sizeof(a) + sizeof(b) + sizeof(c) + sizeof(p) + sizeof(q) + sizeof(ub) +
                 sizeof(vb) + sizeof(u) + sizeof(Iu) + sizeof(Iz));
};

// Shared memory of a block: two stages, the dual results of the north halo row (row 0) and of
// the tile rows (rows 1 .. kTH) for the west / north exchange, and the stages' mbarriers.
template <class ST>
struct TmaSmem {
  TmaStage<ST> st[2];
  float2 sTp[kTH + 1][32];
  float4 sQ[kTH + 1][32];
  alignas(8) unsigned long long bar[2];
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_load_2d(const void* dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// Sleeps until the phase of the given parity has completed or the suspend hint has elapsed.
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(kSuspendNs)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < kMaxWaits; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// segment descriptor: tile column (bits 0-11), first tile row (12-23), tile rows (24-31)
__device__ __forceinline__ int seg_tx(uint32_t s) { return (int)(s & 0xfffu); }
__device__ __forceinline__ int seg_ty(uint32_t s) { return (int)((s >> 12) & 0xfffu); }
__device__ __forceinline__ int seg_len(uint32_t s) { return (int)(s >> 24); }

}  // namespace

// Kernel parameters: the launch's tensor maps (the current ping-pong buffers and p / q
// planes), the pair's pointers for the stores, the segment list and the iteration's scalars.
struct IterTmaArgs {
  CUtensorMap m_code, m_a, m_b, m_c, m_p, m_q, m_ub, m_vb, m_u, m_Iu, m_Iz;
  IterPair P;
  const uint32_t* seg;
  int nseg;
  float sp, sq, tau, mu;
  int parity, write_tp;
};

namespace {

// Thread 0: arm the stage's mbarrier with the bytes of one tile and issue the tile's copies.
template <class ST>
__device__ __forceinline__ void issue_tile(TmaStage<ST>& S, const IterTmaArgs& A, int tx, int ty, uint32_t bar) {
  typedef typename Store2<ST>::T2 T2;
  typedef typename Store2<ST>::T4 T4;
  constexpr int c2 = (int)(sizeof(T2) / 4), c4 = (int)(sizeof(T4) / 4);  // 32-bit words per element
  const int x0 = tx * 31, y0 = ty * kTH;
  // box origins (see the file comment): multiples of 4 pixels, and of 16 for the edge codes
  const int xs = (x0 - 2) & ~3, xc = (x0 - 1) & ~15;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(TmaStage<ST>::kBytes)
               : "memory");
  tma_load_2d(S.code, &A.m_code, xc, y0 - 1, bar);
  tma_load_2d(S.a, &A.m_a, xs, y0 - 1, bar);
  tma_load_2d(S.b, &A.m_b, xs, y0 - 1, bar);
  tma_load_2d(S.c, &A.m_c, xs, y0 - 1, bar);
  tma_load_2d(S.p, &A.m_p, xs * c2, y0 - 1, bar);
  tma_load_2d(S.q, &A.m_q, xs * c4, y0 - 1, bar);
  tma_load_2d(S.ub, &A.m_ub, xs, y0 - 2, bar);
  tma_load_2d(S.vb, &A.m_vb, xs * c2, y0 - 2, bar);
  tma_load_2d(S.u, &A.m_u, xs, y0, bar);
  tma_load_2d(S.Iu, &A.m_Iu, xs, y0, bar);
  tma_load_2d(S.Iz, &A.m_Iz, xs, y0, bar);
}

// What the threshold and primal steps of a tile pixel take from its dual step.
struct PixelState {
  uint8_t code;
  bool in_img, own;
  float a, b, c, ubar, u, Iu, Iz;
  float2 vb, pp, tp;
  float4 qq;
};

// Dual step at the region pixel of column rx (image column x0 - 1 + rx) and region row r (image
// row y0 - 1 + r; r = 0 is the north halo row), from the stage.  The same operations as
// FusedIter::dual_at of k_fused_iter, with every operand read from shared memory.
template <bool MASKED, class ST>
__device__ __forceinline__ void dual_pixel(const IterTmaArgs& A, const TmaStage<ST>& S, int x0, int y0, int rx,
                                           int r, PixelState& o) {
  typedef Store2<ST> St;
  constexpr bool kFast = !std::is_same<ST, float>::value;
  const IterPair& P = A.P;
  const int ix = x0 - 1 + rx, iy = y0 - 1 + r;
  const int lx = ix - ((x0 - 2) & ~3), lc = ix - ((x0 - 1) & ~15);
  o.code = 0;
  o.own = false;
  o.a = o.b = o.c = o.ubar = o.u = o.Iu = o.Iz = 0.f;
  o.vb = o.pp = o.tp = make_float2(0.f, 0.f);
  o.qq = make_float4(0.f, 0.f, 0.f, 0.f);
  o.in_img = ix >= 0 && iy >= 0 && ix < P.w && iy < P.h;
  const int pos = ix + iy * P.s;
  if (o.in_img) {
    o.code = S.code[r][lc];
    o.a = S.a[r][lx];
    o.b = S.b[r][lx];
    o.c = S.c[r][lx];
    bool useRight, useDown, active = true;
    if (MASKED) {
      active = o.code & kOn;
      useRight = o.code & kR;
      useDown = o.code & kD;
    } else {
      useRight = (ix + 1) < P.w;
      useDown = (iy + 1) < P.h;
    }
    if (!active) {
      o.tp = P.Tp[pos];  // masked out: the stale T p
    } else if (!MASKED && !(o.code & kOn)) {  // plain form, outside the circle: p = q = 0
      o.own = true;
      o.tp = tp_math(o.a, o.b, o.c, o.pp);
    } else {
      o.own = true;
      const int yb = r + 1;  // u-bar / v-bar row of the pixel
      o.ubar = S.ub[yb][lx];
      o.vb = St::cvt2(S.vb[yb][lx]);
      const float u_xn = useRight ? S.ub[yb][lx + 1] : S.ub[yb][lx - 1];
      const float u_yn = useDown ? S.ub[yb + 1][lx] : S.ub[yb - 1][lx];
      const float2 v_xn = St::cvt2(useRight ? S.vb[yb][lx + 1] : S.vb[yb][lx - 1]);
      const float2 v_yn = St::cvt2(useDown ? S.vb[yb + 1][lx] : S.vb[yb - 1][lx]);
      o.pp = St::cvt2(S.p[r][lx]);
      o.qq = St::cvt4(S.q[r][lx]);
      if (r >= 1 && rx >= 1) {
        o.u = S.u[r - 1][lx];
        o.Iu = S.Iu[r - 1][lx];
        o.Iz = S.Iz[r - 1][lx];
      }
      if (kFast) {
        fast::dual(useRight, useDown, o.ubar, u_xn, u_yn, o.vb, v_xn, v_yn, o.a, o.b, o.c, A.sp, A.sq, o.pp, o.qq);
        o.tp = fast::tp(o.a, o.b, o.c, o.pp);
      } else {
        dual_math(useRight, useDown, o.ubar, u_xn, u_yn, o.vb, v_xn, v_yn, o.a, o.b, o.c, A.sp, A.sq, o.pp, o.qq);
        o.tp = tp_math(o.a, o.b, o.c, o.pp);
      }
    }
  } else if (ix < 0 && iy >= 1 && iy < P.h) {
    // left of the image: the reference's west neighbour of column 0 is the flat position
    // before it, the last padding element of the previous row
    o.tp = P.Tp[pos];
  }
}

// Threshold and primal steps of the tile pixel at region column rx >= 1, region row r >= 1,
// with the west / north T p and q from the exchange rows; the same operations as phases 2 and 3
// of k_fused_iter.
template <bool MASKED, class ST>
__device__ __forceinline__ void finish_pixel(const IterTmaArgs& A, const TmaSmem<ST>& sm, int x0, int y0, int rx,
                                             int r, const PixelState& o) {
  typedef Store2<ST> St;
  typedef typename St::T2 T2;
  constexpr bool kFast = !std::is_same<ST, float>::value;
  const IterPair& P = A.P;
  const int ix = x0 - 1 + rx, iy = y0 - 1 + r;
  const int pos = ix + iy * P.s;
  const float2 tp = o.tp;
  float dxm, dym;
  bool zR, zD, hasL, hasU;
  if (MASKED) {
    if (!(o.code & kOn)) return;
    bool mR = o.code & kR, mL = o.code & kL, mD = o.code & kD, mU = o.code & kU;
    if (mL && mR) dxm = tp.x - sm.sTp[r][rx - 1].x;
    else if (!mR) dxm = -sm.sTp[r][rx - 1].x;
    else dxm = tp.x;
    if (mU && mD) dym = tp.y - sm.sTp[r - 1][rx].y;
    else if (!mD) dym = -sm.sTp[r - 1][rx].y;
    else dym = tp.y;
    zR = !mR;
    zD = !mD;
    hasL = mL;
    hasU = mU;
  } else {
    if (!(o.code & kOn)) {
      P.us[pos] = 0.0f;
      P.u_s[pos] = 0.0f;
      St::st2((T2*)P.v_s, pos, make_float2(0.f, 0.f));
      return;
    }
    if ((ix - 1) >= 0) dxm = tp.x - sm.sTp[r][rx - 1].x;
    else if (ix == P.w - 1) dxm = -sm.sTp[r][rx - 1].x;
    else dxm = tp.x;
    if ((iy - 1) >= 0) dym = tp.y - sm.sTp[r - 1][rx].y;
    else if (iy == P.h - 1) dym = -sm.sTp[r - 1][rx].y;
    else dym = tp.y;
    zR = ix == P.w - 1;
    zD = iy == P.h - 1;
    hasL = (ix - 1) >= 0;
    hasU = (iy - 1) >= 0;
  }
  float unew;
  if (kFast) {
    float eu = fast::etau(o.a, o.b, o.c, P.alpha1 * P.alpha1);
    unew = fast::threshold(dxm, dym, eu, A.tau, o.ubar, o.u, o.Iu, o.Iz, P.lambda);
  } else {
    float eu = etau_math(o.a, o.b, o.c, P.alpha1);
    unew = threshold_math(dxm, dym, eu, A.tau, o.ubar, o.u, o.Iu, o.Iz, P.lambda);
  }
  P.us[pos] = unew;
  float4 qc = o.qq;
  if (zR) qc.x = qc.w = 0.0f;
  if (zD) qc.y = qc.z = 0.0f;
  float4 ql = hasL ? sm.sQ[r][rx - 1] : make_float4(0.f, 0.f, 0.f, 0.f);
  float4 qu = hasU ? sm.sQ[r - 1][rx] : make_float4(0.f, 0.f, 0.f, 0.f);
  float us_;
  float2 vs;
  if (kFast) {
    const float a1s = P.alpha1 * P.alpha1, a0s4 = 4.0f * P.alpha0 * P.alpha0;
    float ev1 = fast::etav(o.b, o.c, a1s, a0s4), ev2 = fast::etav(o.a, o.c, a1s, a0s4);
    fast::primal(qc, ql, qu, tp, ev1, ev2, A.tau, P.alpha0, P.alpha1, A.mu, o.vb, unew, o.ubar, us_, vs);
  } else {
    float ev1 = etav1_math(o.b, o.c, P.alpha0, P.alpha1), ev2 = etav2_math(o.a, o.c, P.alpha0, P.alpha1);
    float2 vo;
    primal_math(qc, ql, qu, o.pp, o.a, o.b, o.c, ev1, ev2, A.tau, P.alpha0, P.alpha1, A.mu, o.vb, unew, o.ubar, us_,
                vs, vo);
  }
  P.u_s[pos] = us_;
  St::st2((T2*)P.v_s, pos, vs);
}

}  // namespace

template <bool MASKED, class ST>
__global__ void __launch_bounds__(kThreads, 4) k_fused_iter_tma(const __grid_constant__ IterTmaArgs A) {
  typedef Store2<ST> St;
  typedef typename St::T2 T2;
  typedef typename St::T4 T4;
  extern __shared__ unsigned char smem_raw[];
  TmaSmem<ST>& sm = *reinterpret_cast<TmaSmem<ST>*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
  if ((int)blockIdx.x >= A.nseg) return;
  const IterPair& P = A.P;
  const int tid = (int)threadIdx.x, rx = tid & 31, ry = tid >> 5;
  const int plane = P.s * P.h;
  T2* pout = (T2*)P.p + (A.parity ? 0 : plane);
  T4* qout = (T4*)P.q + (A.parity ? 0 : plane);
  const uint32_t bar0 = smem_addr(&sm.bar[0]);  // bar[1] follows at + 8
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  griddep_wait();  // the previous iteration's outputs are this one's inputs
  griddep_launch_dependents();
  int si = (int)blockIdx.x, k = 0;
  uint32_t sv = A.seg[si];
  if (tid == 0) issue_tile<ST>(sm.st[0], A, seg_tx(sv), seg_ty(sv), bar0);
  for (int n = 0;; n++) {
    const int stage = n & 1;
    const int x0 = seg_tx(sv) * 31, y0 = (seg_ty(sv) + k) * kTH;
    // the block's next tile: further down the segment, or the first tile of its next segment
    int nsi = si, nk = k + 1;
    uint32_t nsv = sv;
    if (nk >= seg_len(sv)) {
      nsi = si + (int)gridDim.x;
      nk = 0;
      if (nsi < A.nseg) nsv = A.seg[nsi];
    }
    const bool has_next = nsi < A.nseg;
    // The other stage was last read by the previous tile, which every thread has finished.
    const uint32_t bar = bar0 + 8u * (uint32_t)stage, bar_next = bar0 + 8u * (uint32_t)(stage ^ 1);
    if (tid == 0 && has_next) issue_tile<ST>(sm.st[stage ^ 1], A, seg_tx(nsv), seg_ty(nsv) + nk, bar_next);
    const bool ok = mbar_wait_bounded(bar, (uint32_t)(n >> 1) & 1u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicExch(&g_tma_status, 1);
      // the copies still in flight (this tile's, the next tile's) get a last bounded wait
      (void)mbar_wait_bounded(bar, (uint32_t)(n >> 1) & 1u);
      if (has_next) (void)mbar_wait_bounded(bar_next, (uint32_t)((n + 1) >> 1) & 1u);
      return;
    }
    const TmaStage<ST>& S = sm.st[stage];
    // north halo row: carried over from the tile above, or recomputed at a segment's first tile
    if (k == 0 && ry == 0) {
      PixelState h;
      dual_pixel<MASKED, ST>(A, S, x0, y0, rx, 0, h);
      sm.sTp[0][rx] = h.tp;
      sm.sQ[0][rx] = h.qq;
    }
    PixelState o;
    dual_pixel<MASKED, ST>(A, S, x0, y0, rx, ry + 1, o);
    if (o.own && rx >= 1) {
      const int pos = (x0 - 1 + rx) + (y0 + ry) * P.s;
      St::st2(pout, pos, o.pp);
      St::st4(qout, pos, o.qq);
      if (A.write_tp) P.Tp[pos] = o.tp;
    }
    sm.sTp[ry + 1][rx] = o.tp;
    sm.sQ[ry + 1][rx] = o.qq;
    __syncthreads();
    if (rx >= 1 && o.in_img) finish_pixel<MASKED, ST>(A, sm, x0, y0, rx, ry + 1, o);
    __syncthreads();  // the stage and the exchange rows are read
    if (!has_next) break;
    // the last row's dual results are the next tile's north halo when it is the tile below
    if (nk > 0 && ry == kTH - 1) {
      sm.sTp[0][rx] = sm.sTp[kTH][rx];
      sm.sQ[0][rx] = sm.sQ[kTH][rx];
    }
    si = nsi;
    k = nk;
    sv = nsv;
  }
}

// ---------------------------------------------------------------------------------------
// Host side.
namespace {

// Tensor maps.  A map only describes an address and a layout (no resource is held), so maps
// are cached process-wide by everything that defines them.
typedef CUresult (*PfnEncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

PfnEncodeTiled encode_fn() {
  static PfnEncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PfnEncodeTiled)f;
    (void)cudaGetLastError();
  });
  if (!fn) throw ArgError{"cuTensorMapEncodeTiled is not available from the driver"};
  return fn;
}

// units: 0 = bytes (edge codes), else the number of 32-bit words per pixel (1, 2 or 4);
// is_float: the words are float32 (else raw 32-bit words)
typedef std::tuple<uintptr_t, int, int, int, int, int, int> MapKey;  // ptr, units, float, w, h, s, rows

const CUtensorMap& tensor_map(const void* ptr, int units, bool is_float, int w, int h, int s, int box_rows) {
  static std::mutex mu;
  static std::map<MapKey, CUtensorMap> cache;
  const MapKey key{(uintptr_t)ptr, units, is_float ? 1 : 0, w, h, s, box_rows};
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  if (((uintptr_t)ptr & 15) != 0) throw ArgError{"TMA iteration: buffer not 16-byte aligned"};
  CUtensorMap m;
  cuuint64_t dims[2], strides[1];
  cuuint32_t box[2], estr[2] = {1, 1};
  CUtensorMapDataType dt;
  if (units == 0) {
    dt = CU_TENSOR_MAP_DATA_TYPE_UINT8;
    dims[0] = (cuuint64_t)w;
    strides[0] = (cuuint64_t)s;
    box[0] = kCodeW;
  } else {
    dt = is_float ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT32;
    dims[0] = (cuuint64_t)w * units;
    strides[0] = (cuuint64_t)s * units * 4;
    box[0] = (cuuint32_t)(kBW * units);
  }
  dims[1] = (cuuint64_t)h;
  box[1] = (cuuint32_t)box_rows;
  if (strides[0] % 16 != 0) throw ArgError{"TMA iteration: row pitch not a multiple of 16 bytes"};
  CUresult r = encode_fn()(&m, dt, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw ArgError{"TMA iteration: cuTensorMapEncodeTiled failed"};
  return cache.emplace(key, m).first->second;
}

typedef void (*TmaKernel)(IterTmaArgs);

template <bool MASKED, class ST>
TmaKernel tma_kernel() {
  return k_fused_iter_tma<MASKED, ST>;
}

size_t tma_smem_bytes(bool half) {
  return (half ? sizeof(TmaSmem<__half>) : sizeof(TmaSmem<float>)) + 128;  // + the base alignment
}

TmaKernel pick(bool masked, bool half) {
  if (masked) return half ? tma_kernel<true, __half>() : tma_kernel<true, float>();
  return half ? tma_kernel<false, __half>() : tma_kernel<false, float>();
}

// The kernel's dynamic shared-memory limit and its resident blocks per SM, once per device.
int tma_blocks_per_sm(bool masked, bool half) {
  static std::mutex mu;
  static std::map<std::tuple<int, bool, bool>, int> known;
  int dev = 0;
  VFS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_tuple(dev, masked, half);
  auto it = known.find(key);
  if (it != known.end()) return it->second;
  const TmaKernel k = pick(masked, half);
  const size_t smem = tma_smem_bytes(half);
  VFS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int n = 0;
  VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kThreads, smem));
  known[key] = n;
  return n;
}

int sm_count() {
  int dev = 0, sms = 1;
  VFS_CUDA(cudaGetDevice(&dev));
  VFS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return sms;
}

}  // namespace

std::vector<uint32_t> tma_segments(int w, int h, const uint16_t* lo, const uint16_t* hi) {
  const int tiles_x = iter_tiles_x_of(w), rows = (h + kTH - 1) / kTH;
  if (tiles_x > 4095 || rows > 4095) throw ArgError{"TMA iteration: level too large for the segment list"};
  auto active = [&](int tx, int ty) { return !lo || (tx >= (int)lo[ty] && tx <= (int)hi[ty]); };
  int tiles = 0;
  for (int ty = 0; ty < rows; ty++)
    for (int tx = 0; tx < tiles_x; tx++) tiles += active(tx, ty) ? 1 : 0;
  // about as many segments as the GPU holds resident blocks (4 per SM with 256 threads)
  const int target = std::max(1, sm_count() * 4);
  const int len = std::min(255, std::max(1, (tiles + target - 1) / target));
  std::vector<uint32_t> seg;
  for (int tx = 0; tx < tiles_x; tx++) {
    int ty = 0;
    while (ty < rows) {
      if (!active(tx, ty)) {
        ty++;
        continue;
      }
      int run = 0;
      while (ty + run < rows && active(tx, ty + run) && run < len) run++;
      seg.push_back((uint32_t)tx | ((uint32_t)ty << 12) | ((uint32_t)run << 24));
      ty += run;
    }
  }
  return seg;
}

size_t tma_segment_capacity(int s, int h) {
  return (size_t)iter_tiles_x_of(s) * (size_t)((h + kTH - 1) / kTH);
}

void launch_fused_iteration_tma(const IterArgs& I, const uint32_t* seg, int nseg, bool masked, bool half_storage,
                                cudaStream_t st, int parity) {
  if (I.npairs != 1) throw ArgError{"TMA iteration: one pair per launch"};
  if (nseg <= 0) return;
  if (!seg) throw ArgError{"TMA iteration: no segment list"};
  const IterPair& P = I.pr[0];
  if (P.w < 2 || P.h < 2 || P.w > 65535 || P.h > 32767) throw ArgError{"TMA iteration: unsupported level size"};
  IterTmaArgs A;
  A.P = P;
  A.seg = seg;
  A.nseg = nseg;
  A.sp = I.sp[0];
  A.sq = I.sq[0];
  A.tau = I.tau;
  A.mu = I.mu;
  A.parity = parity;
  A.write_tp = I.write_tp;
  const int w = P.w, h = P.h, s = P.s;
  const int u2 = half_storage ? 1 : 2, u4 = half_storage ? 2 : 4;  // 32-bit words per T2 / T4
  const size_t plane = (size_t)s * h;
  const char* pin = (const char*)P.p + (parity ? plane * u2 * 4 : 0);
  const char* qin = (const char*)P.q + (parity ? plane * u4 * 4 : 0);
  A.m_code = tensor_map(P.code, 0, false, w, h, s, kTH + 1);
  A.m_a = tensor_map(P.a, 1, true, w, h, s, kTH + 1);
  A.m_b = tensor_map(P.b, 1, true, w, h, s, kTH + 1);
  A.m_c = tensor_map(P.c, 1, true, w, h, s, kTH + 1);
  A.m_p = tensor_map(pin, u2, !half_storage, w, h, s, kTH + 1);
  A.m_q = tensor_map(qin, u4, !half_storage, w, h, s, kTH + 1);
  A.m_ub = tensor_map(P.u_, 1, true, w, h, s, kTH + 3);
  A.m_vb = tensor_map(P.v_, u2, !half_storage, w, h, s, kTH + 3);
  A.m_u = tensor_map(P.u, 1, true, w, h, s, kTH);
  A.m_Iu = tensor_map(P.Iu, 1, true, w, h, s, kTH);
  A.m_Iz = tensor_map(P.Iz, 1, true, w, h, s, kTH);
  const int per_sm = std::max(1, tma_blocks_per_sm(masked, half_storage));
  const int grid = std::min(nseg, per_sm * sm_count());
  launch_overlapped_smem(pick(masked, half_storage), dim3(grid), dim3(kThreads), tma_smem_bytes(half_storage), st, A);
  VFS_LAUNCH_CHECK();
}

double tma_gpu_share(bool masked, bool half, int nseg) {
  const double cap = (double)sm_count() * std::max(1, tma_blocks_per_sm(masked, half));
  return nseg >= cap ? 1.0 : (double)nseg / cap;
}

int tma_status_take() {
  int v = 0, zero = 0;
  VFS_CUDA(cudaMemcpyFromSymbol(&v, g_tma_status, sizeof(int)));
  VFS_CUDA(cudaMemcpyToSymbol(g_tma_status, &zero, sizeof(int)));
  return v;
}

}  // namespace vfs
