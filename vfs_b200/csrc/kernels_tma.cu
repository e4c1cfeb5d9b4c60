// TMA-staged form of the one-iteration fused primal-dual kernel (iteration variant 18).
//
// The block and tile geometry are those of k_fused_iter with 8-row tiles (variant 1): a
// 32 x 9 block covers a 31 x 8 tile plus a one-pixel west / north halo, every thread runs the
// dual step (updateDualVariables.cu:122-237) at its region pixel, and after a barrier the
// tile threads run the threshold and primal steps (thresholdingL1.cu:128-228,
// updatePrimalVariables.cu:139-245) with the west / north T p and q from shared memory.  The
// per-pixel arithmetic is the same code (tgv_pixel.cuh / tgv_pixel_fast.cuh), so the results
// are bit-identical to the other variants.
//
// What differs is how the inputs arrive.  k_fused_iter issues per-thread global loads in two
// dependent rounds: the edge code and tensor first, then the neighbours the code selects,
// p, q, u, Iu and Iz.  Here one thread issues eleven bulk tensor copies
// (cp.async.bulk.tensor.2d, TMA) that bring the block's whole region of every input plane
// into shared memory, completing on one mbarrier; the threads then read everything,
// neighbours included, from shared memory.  One round trip, no per-thread address arithmetic
// for the loads, and no load whose address depends on another load.
//
// Copy boxes (x in pixels; a box starts on a 16-byte boundary, as TMA requires, so its start
// is rounded down and the box is wider than the region):
//   u-bar, v-bar        x from (x0 - 2) & ~3, 40 wide, rows y0 - 2 .. y0 + 8
//   tensor a b c, p, q  x from (x0 - 2) & ~3, 40 wide, rows y0 - 1 .. y0 + 7
//   u, Iu, Iz           x from (x0 - 2) & ~3, 40 wide, rows y0 .. y0 + 7
//   edge codes (bytes)  x from (x0 - 1) & ~15, 48 wide, rows y0 - 1 .. y0 + 7
// with x0 = 31 * tile column, y0 = 8 * tile row.  Coordinates outside the image read 0
// (the tensor maps' out-of-bounds fill), which is also what the drop-in kernels read before
// a buffer's start (row -1).  West of column 0 the reference reads the flat position before
// it (the previous row's last element); the caller uses this kernel on a masked level only
// when no pixel of column 0 is on (StereoTgvImpl::tma_ok), so no pixel reads there.  The
// stale T p of masked-out pixels is still read from global memory, as in k_fused_iter.
//
// The tensor maps describe this GPU's own buffers only; no copy uses cluster multicast.
// The wait on the mbarrier is bounded: if the copies have not landed after kTmaMaxPolls polls
// the block records an error in g_tma_status (vfs_device_status) and leaves.
#include <cuda.h>

#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "common.cuh"
#include "fused.cuh"
#include "tgv_pixel.cuh"
#include "tgv_pixel_fast.cuh"

namespace vfs {

namespace {

constexpr int kTH = 8;        // tile rows (the geometry of variant 1)
constexpr int kBW = 40;       // pixels per box row of the 4-, 8- and 16-byte planes
constexpr int kCodeW = 48;    // bytes per box row of the edge codes
constexpr long long kTmaMaxPolls = 1ll << 24;

__device__ int g_tma_status;  // 0 = fine; 1 = an mbarrier wait ran out

template <class ST>
struct TmaTile {
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
  float2 sTp[kTH + 1][32];
  float4 sQ[kTH + 1][32];
  alignas(8) unsigned long long bar;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_load_2d(const void* dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(phase)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase 0 of the block's mbarrier (all copies landed).
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar) {
  for (long long i = 0; i < kTmaMaxPolls; i++)
    if (mbar_try_wait(bar, 0)) return true;
  return false;
}

}  // namespace

// Kernel parameters: the launch's tensor maps (the current ping-pong buffers and p / q
// planes), the pair's pointers for the stores, and the iteration's scalars.
struct IterTmaArgs {
  CUtensorMap m_code, m_a, m_b, m_c, m_p, m_q, m_ub, m_vb, m_u, m_Iu, m_Iz;
  IterPair P;
  float sp, sq, tau, mu;
  int parity, write_tp;
  int span_rows, span_max;
  uint16_t span_lo[kMaxSpanRows], span_hi[kMaxSpanRows];
};

template <bool MASKED, class ST>
__global__ void __launch_bounds__(32 * (kTH + 1), 6) k_fused_iter_tma(const __grid_constant__ IterTmaArgs A) {
  typedef Store2<ST> S;
  typedef typename S::T2 T2;
  typedef typename S::T4 T4;
  constexpr bool kFast = !std::is_same<ST, float>::value;
  __shared__ TmaTile<ST> sm;
  const IterPair& P = A.P;
  int tx = (int)blockIdx.x;
  if (MASKED && A.span_rows > 0) {  // only the tiles of this row that hold a pixel that is on
    tx += A.span_lo[blockIdx.y];
    if (tx > (int)A.span_hi[blockIdx.y]) return;
  }
  const int x0 = tx * 31, y0 = (int)blockIdx.y * kTH;
  const int rx = threadIdx.x, ry = threadIdx.y;
  const int tid = ry * 32 + rx;
  const int ix = x0 - 1 + rx, iy = y0 - 1 + ry;
  const int plane = P.s * P.h;
  T2* pout = (T2*)P.p + (A.parity ? 0 : plane);
  T4* qout = (T4*)P.q + (A.parity ? 0 : plane);
  const bool tile = rx >= 1 && ry >= 1;
  const bool in_img = ix >= 0 && iy >= 0 && ix < P.w && iy < P.h;
  const int pos = ix + iy * P.s;
  // box origins (see the file comment); xs and xc are multiples of 4 and 16 pixels
  const int xs = (x0 - 2) & ~3, xc = (x0 - 1) & ~15;
  const uint32_t bar = smem_addr(&sm.bar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  griddep_wait();  // the previous iteration's outputs are this one's inputs
  griddep_launch_dependents();
  if (tid == 0) {
    constexpr uint32_t kBytes = (uint32_t)(sizeof(sm.code) + sizeof(sm.a) + sizeof(sm.b) + sizeof(sm.c) +
                                           sizeof(sm.p) + sizeof(sm.q) + sizeof(sm.ub) + sizeof(sm.vb) +
                                           sizeof(sm.u) + sizeof(sm.Iu) + sizeof(sm.Iz));
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kBytes) : "memory");
    constexpr int c2 = (int)(sizeof(T2) / 4), c4 = (int)(sizeof(T4) / 4);  // 4-byte units per element
    tma_load_2d(sm.code, &A.m_code, xc, y0 - 1, bar);
    tma_load_2d(sm.a, &A.m_a, xs, y0 - 1, bar);
    tma_load_2d(sm.b, &A.m_b, xs, y0 - 1, bar);
    tma_load_2d(sm.c, &A.m_c, xs, y0 - 1, bar);
    tma_load_2d(sm.p, &A.m_p, xs * c2, y0 - 1, bar);
    tma_load_2d(sm.q, &A.m_q, xs * c4, y0 - 1, bar);
    tma_load_2d(sm.ub, &A.m_ub, xs, y0 - 2, bar);
    tma_load_2d(sm.vb, &A.m_vb, xs * c2, y0 - 2, bar);
    tma_load_2d(sm.u, &A.m_u, xs, y0, bar);
    tma_load_2d(sm.Iu, &A.m_Iu, xs, y0, bar);
    tma_load_2d(sm.Iz, &A.m_Iz, xs, y0, bar);
  }
  // the block decides together whether the copies landed (a block barrier follows later)
  if (__syncthreads_or(!mbar_wait_bounded(bar))) {
    if (tid == 0) atomicExch(&g_tma_status, 1);
    (void)mbar_wait_bounded(bar);  // give copies still in flight a last bounded chance to land
    return;
  }

  // shared-memory coordinates of this thread's region pixel
  const int lx = ix - xs;        // 4-byte planes: 1 .. 35
  const int lc = ix - xc;        // edge codes: 0 .. 45
  // ---- phase 1: dual update at every region pixel ------------------------------------
  float2 pp = make_float2(0.f, 0.f), tp = make_float2(0.f, 0.f), vb = make_float2(0.f, 0.f);
  float4 qq = make_float4(0.f, 0.f, 0.f, 0.f);
  uint8_t code = 0;
  float a = 0.f, b = 0.f, c = 0.f, ubar = 0.f;
  float u_th = 0.f, Iu_th = 0.f, Iz_th = 0.f;
  bool own = false;
  if (in_img) {
    code = sm.code[ry][lc];
    a = sm.a[ry][lx];
    b = sm.b[ry][lx];
    c = sm.c[ry][lx];
    bool useRight = false, useDown = false, active = true;
    if (MASKED) {
      active = code & kOn;
      useRight = code & kR;
      useDown = code & kD;
    } else {
      useRight = (ix + 1) < P.w;
      useDown = (iy + 1) < P.h;
    }
    if (!active) {
      tp = P.Tp[pos];  // masked out: the stale T p
    } else if (!MASKED && !(code & kOn)) {  // plain form, outside the circle: p = q = 0
      own = true;
      tp = tp_math(a, b, c, pp);
    } else {
      own = true;
      const int yb = ry + 1;  // u-bar / v-bar row of the pixel
      ubar = sm.ub[yb][lx];
      vb = S::cvt2(sm.vb[yb][lx]);
      const float u_xn = useRight ? sm.ub[yb][lx + 1] : sm.ub[yb][lx - 1];
      const float u_yn = useDown ? sm.ub[yb + 1][lx] : sm.ub[yb - 1][lx];
      const float2 v_xn = S::cvt2(useRight ? sm.vb[yb][lx + 1] : sm.vb[yb][lx - 1]);
      const float2 v_yn = S::cvt2(useDown ? sm.vb[yb + 1][lx] : sm.vb[yb - 1][lx]);
      pp = S::cvt2(sm.p[ry][lx]);
      qq = S::cvt4(sm.q[ry][lx]);
      if (tile) {
        u_th = sm.u[ry - 1][lx];
        Iu_th = sm.Iu[ry - 1][lx];
        Iz_th = sm.Iz[ry - 1][lx];
      }
      if (kFast) {
        fast::dual(useRight, useDown, ubar, u_xn, u_yn, vb, v_xn, v_yn, a, b, c, A.sp, A.sq, pp, qq);
        tp = fast::tp(a, b, c, pp);
      } else {
        dual_math(useRight, useDown, ubar, u_xn, u_yn, vb, v_xn, v_yn, a, b, c, A.sp, A.sq, pp, qq);
        tp = tp_math(a, b, c, pp);
      }
    }
    if (own && tile) {
      S::st2(pout, pos, pp);
      S::st4(qout, pos, qq);
      if (A.write_tp) P.Tp[pos] = tp;
    }
  } else if (ix < 0 && iy >= 1 && iy < P.h) {
    // left of the image: the reference's west neighbour of column 0 is the flat position
    // before it, the last padding element of the previous row
    tp = P.Tp[pos];
  }
  sm.sTp[ry][rx] = tp;
  sm.sQ[ry][rx] = qq;
  __syncthreads();
  if (!tile || !in_img) return;

  // ---- phase 2: thresholding --------------------------------------------------------
  float dxm, dym;
  bool zR, zD, hasL, hasU;
  if (MASKED) {
    if (!(code & kOn)) return;
    bool mR = code & kR, mL = code & kL, mD = code & kD, mU = code & kU;
    if (mL && mR) dxm = tp.x - sm.sTp[ry][rx - 1].x;
    else if (!mR) dxm = -sm.sTp[ry][rx - 1].x;
    else dxm = tp.x;
    if (mU && mD) dym = tp.y - sm.sTp[ry - 1][rx].y;
    else if (!mD) dym = -sm.sTp[ry - 1][rx].y;
    else dym = tp.y;
    zR = !mR;
    zD = !mD;
    hasL = mL;
    hasU = mU;
  } else {
    if (!(code & kOn)) {
      P.us[pos] = 0.0f;
      P.u_s[pos] = 0.0f;
      S::st2((T2*)P.v_s, pos, make_float2(0.f, 0.f));
      return;
    }
    if ((ix - 1) >= 0) dxm = tp.x - sm.sTp[ry][rx - 1].x;
    else if (ix == P.w - 1) dxm = -sm.sTp[ry][rx - 1].x;
    else dxm = tp.x;
    if ((iy - 1) >= 0) dym = tp.y - sm.sTp[ry - 1][rx].y;
    else if (iy == P.h - 1) dym = -sm.sTp[ry - 1][rx].y;
    else dym = tp.y;
    zR = ix == P.w - 1;
    zD = iy == P.h - 1;
    hasL = (ix - 1) >= 0;
    hasU = (iy - 1) >= 0;
  }
  float unew;
  if (kFast) {
    float eu = fast::etau(a, b, c, P.alpha1 * P.alpha1);
    unew = fast::threshold(dxm, dym, eu, A.tau, ubar, u_th, Iu_th, Iz_th, P.lambda);
  } else {
    float eu = etau_math(a, b, c, P.alpha1);
    unew = threshold_math(dxm, dym, eu, A.tau, ubar, u_th, Iu_th, Iz_th, P.lambda);
  }
  P.us[pos] = unew;

  // ---- phase 3: primal update ------------------------------------------------------
  float4 qc = qq;
  if (zR) qc.x = qc.w = 0.0f;
  if (zD) qc.y = qc.z = 0.0f;
  float4 ql = hasL ? sm.sQ[ry][rx - 1] : make_float4(0.f, 0.f, 0.f, 0.f);
  float4 qu = hasU ? sm.sQ[ry - 1][rx] : make_float4(0.f, 0.f, 0.f, 0.f);
  float us_;
  float2 vs;
  if (kFast) {
    const float a1s = P.alpha1 * P.alpha1, a0s4 = 4.0f * P.alpha0 * P.alpha0;
    float ev1 = fast::etav(b, c, a1s, a0s4), ev2 = fast::etav(a, c, a1s, a0s4);
    fast::primal(qc, ql, qu, tp, ev1, ev2, A.tau, P.alpha0, P.alpha1, A.mu, vb, unew, ubar, us_, vs);
  } else {
    float ev1 = etav1_math(b, c, P.alpha0, P.alpha1), ev2 = etav2_math(a, c, P.alpha0, P.alpha1);
    float2 vo;
    primal_math(qc, ql, qu, pp, a, b, c, ev1, ev2, A.tau, P.alpha0, P.alpha1, A.mu, vb, unew, ubar, us_, vs, vo);
  }
  P.u_s[pos] = us_;
  S::st2((T2*)P.v_s, pos, vs);
}

// ---------------------------------------------------------------------------------------
// Host side: tensor maps.  A map only describes an address and a layout (no resource is held),
// so maps are cached process-wide by everything that defines them.
namespace {

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
// float: the words are float32 (else raw 32-bit words)
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

}  // namespace

void launch_fused_iteration_tma(const IterArgs& I, bool masked, bool half_storage, cudaStream_t st, int parity) {
  if (I.npairs != 1) throw ArgError{"TMA iteration: one pair per launch"};
  const IterPair& P = I.pr[0];
  if (P.w < 2 || P.h < 2 || P.w > 65535 || P.h > 65535) throw ArgError{"TMA iteration: unsupported level size"};
  IterTmaArgs A;
  A.P = P;
  A.sp = I.sp[0];
  A.sq = I.sq[0];
  A.tau = I.tau;
  A.mu = I.mu;
  A.parity = parity;
  A.write_tp = I.write_tp;
  A.span_rows = I.span_rows;
  A.span_max = I.span_max;
  for (int r = 0; r < kMaxSpanRows; r++) {
    A.span_lo[r] = I.span_lo[r];
    A.span_hi[r] = I.span_hi[r];
  }
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
  dim3 grid(P.tiles_x, (h + kTH - 1) / kTH), blk(32, kTH + 1);
  if (masked && A.span_rows > 0) {
    if (A.span_rows != (int)grid.y) throw ArgError{"tile spans do not match the launch"};
    grid.x = A.span_max > 0 ? A.span_max : 1;
  }
  if (masked) {
    if (half_storage) launch_overlapped(k_fused_iter_tma<true, __half>, grid, blk, st, A);
    else launch_overlapped(k_fused_iter_tma<true, float>, grid, blk, st, A);
  } else {
    if (half_storage) launch_overlapped(k_fused_iter_tma<false, __half>, grid, blk, st, A);
    else launch_overlapped(k_fused_iter_tma<false, float>, grid, blk, st, A);
  }
  VFS_LAUNCH_CHECK();
}

double tma_gpu_share(bool masked, bool half, int w, int h) {
  int n = 0, dev = 0, sms = 1;
  const int threads = 32 * (kTH + 1);
  if (masked) {
    if (half) VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_tma<true, __half>, threads, 0));
    else VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_tma<true, float>, threads, 0));
  } else {
    if (half) VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_tma<false, __half>, threads, 0));
    else VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter_tma<false, float>, threads, 0));
  }
  VFS_CUDA(cudaGetDevice(&dev));
  VFS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const double blocks = (double)iter_tiles_of(w, h, kTH);
  const double cap = (double)sms * (n > 0 ? n : 1);
  return blocks >= cap ? 1.0 : blocks / cap;
}

int tma_status_take() {
  int v = 0, zero = 0;
  VFS_CUDA(cudaMemcpyFromSymbol(&v, g_tma_status, sizeof(int)));
  VFS_CUDA(cudaMemcpyToSymbol(g_tma_status, &zero, sizeof(int)));
  return v;
}

}  // namespace vfs
