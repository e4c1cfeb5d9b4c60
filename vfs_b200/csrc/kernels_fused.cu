// Fused, batched kernels of the fast solve path (see fused.cuh).
#include "common.cuh"
#include "fused.cuh"
#include "tgv_math.cuh"
#include "tgv_pixel.cuh"
#include "tgv_pixel_fast.cuh"

#include <type_traits>

namespace vfs {

#define TILE_SETUP(ARGS)                                        \
  const int t_ = blockIdx.x;                                    \
  const int pi_ = find_pair(ARGS.pr, ARGS.npairs, t_);          \
  const auto& P = ARGS.pr[pi_];                                 \
  const int lt_ = t_ - P.tile0;                                 \
  const int x0 = (lt_ % P.tiles_x) * kFTW;                      \
  const int y0 = (lt_ / P.tiles_x) * kFTH;                      \
  const int ix = x0 + (int)threadIdx.x;                         \
  const int iy = y0 + (int)threadIdx.y;

// ---------------------------------------------------------------------------
// One primal-dual iteration (updateDualVariables + solveTp + thresholdingL1 +
// updatePrimalVariables).  The dual update is also evaluated on a one-pixel halo to
// the left and top of the tile (the threshold and primal steps read T p and q of the
// west and north neighbours), so p and q are read from one buffer and written to
// another (the caller ping-pongs them).
// ---------------------------------------------------------------------------
template <bool MASKED, class ST>
struct FusedIter {
  typedef Store2<ST> S;
  typedef typename S::T2 T2;
  typedef typename S::T4 T4;
  // Half storage takes the fused multiply-add / approximate reciprocal arithmetic of
  // tgv_pixel_fast.cuh; float storage the exact forms of tgv_pixel.cuh.
  static constexpr bool kFast = !std::is_same<ST, float>::value;

  // dual update at an in-image pixel whose code and tensor are given; returns false where
  // the pixel keeps its values (masked out), in which case tp is the stored (stale) T p.
  // u_pos and vp (u-bar and v-bar here) are returned for the threshold and primal steps.
  // With want_th, also loads u, Iu and Iz of the pixel (read by the threshold step after the
  // barrier) together with the dual step's loads, so they travel in the same round trip.
  static __device__ __forceinline__ bool dual_at(const IterPair& P, const T2* pin, const T4* qin, int ix, int iy,
                                                 int pos, uint8_t code, float a, float b, float c, float sp, float sq,
                                                 float& u_pos, float2& vp, float2& p, float4& q, float2& tp,
                                                 bool want_th, float& u_th, float& Iu_th, float& Iz_th) {
    int right = pos + 1, down = pos + P.s, left = pos - 1, up = pos - P.s;
    bool useRight, useDown;
    if (MASKED) {
      if (!(code & kOn)) {
        tp = P.Tp[pos];
        return false;
      }
      useRight = code & kR;
      useDown = code & kD;
    } else {
      if (!(code & kOn)) {  // outside the circle: p = q = 0, T p = T 0
        p = make_float2(0.f, 0.f);
        q = make_float4(0.f, 0.f, 0.f, 0.f);
        tp = tp_math(a, b, c, p);
        return true;
      }
      useRight = (ix + 1) < P.w;
      useDown = (iy + 1) < P.h;
    }
    const T2* v_ = (const T2*)P.v_;
    u_pos = P.u_[pos];
    vp = S::ld2(v_, pos);
    float u_xn = useRight ? P.u_[right] : (left < 0 ? 0.0f : P.u_[left]);
    float u_yn = useDown ? P.u_[down] : (up < 0 ? 0.0f : P.u_[up]);
    float2 v_xn = useRight ? S::ld2(v_, right) : (left < 0 ? make_float2(0.f, 0.f) : S::ld2(v_, left));
    float2 v_yn = useDown ? S::ld2(v_, down) : (up < 0 ? make_float2(0.f, 0.f) : S::ld2(v_, up));
    p = S::ld2(pin, pos);
    q = S::ld4(qin, pos);
    if (want_th) {
      u_th = P.u[pos];
      Iu_th = P.Iu[pos];
      Iz_th = P.Iz[pos];
    }
    if (kFast) {
      fast::dual(useRight, useDown, u_pos, u_xn, u_yn, vp, v_xn, v_yn, a, b, c, sp, sq, p, q);
      tp = fast::tp(a, b, c, p);
    } else {
      dual_math(useRight, useDown, u_pos, u_xn, u_yn, vp, v_xn, v_yn, a, b, c, sp, sq, p, q);
      tp = tp_math(a, b, c, p);
    }
    return true;
  }

  // dual_at for a pixel that is on and whose four neighbours are in the image (and, masked,
  // on): the right and down neighbours are the ones used, and nothing depends on the code.
  static __device__ __forceinline__ void dual_interior(const IterPair& P, const T2* pin, const T4* qin, int pos,
                                                       float a, float b, float c, float sp, float sq, float& u_pos,
                                                       float2& vp, float2& p, float4& q, float2& tp, bool want_th,
                                                       float& u_th, float& Iu_th, float& Iz_th) {
    const T2* v_ = (const T2*)P.v_;
    u_pos = P.u_[pos];
    vp = S::ld2(v_, pos);
    float u_xn = P.u_[pos + 1];
    float u_yn = P.u_[pos + P.s];
    float2 v_xn = S::ld2(v_, pos + 1);
    float2 v_yn = S::ld2(v_, pos + P.s);
    p = S::ld2(pin, pos);
    q = S::ld4(qin, pos);
    if (want_th) {
      u_th = P.u[pos];
      Iu_th = P.Iu[pos];
      Iz_th = P.Iz[pos];
    }
    if (kFast) {
      fast::dual_interior(u_pos, u_xn, u_yn, vp, v_xn, v_yn, a, b, c, sp, sq, p, q);
      tp = fast::tp(a, b, c, p);
    } else {
      dual_math(true, true, u_pos, u_xn, u_yn, vp, v_xn, v_yn, a, b, c, sp, sq, p, q);
      tp = tp_math(a, b, c, p);
    }
  }

  // a pixel whose code (and, for the plain form, position) makes every edge rule of the
  // threshold and primal steps take its interior branch
  static __device__ __forceinline__ bool interior(uint8_t code, int ix, int iy, int w, int h) {
    if (MASKED) return code == (kOn | kR | kL | kD | kU);
    return (code & kOn) && ix >= 1 && iy >= 1 && ix + 1 < w && iy + 1 < h;
  }
};

// The block is a 32 x (TH + 1) region: one image row segment per warp, the first
// column and the first row being the halo of the 31 x TH tile.  Every thread
// evaluates the dual update at its region pixel; after a barrier the tile threads
// finish the threshold and primal steps with the west / north values from shared
// memory.  The pixel's code, tensor, u-bar and v-bar stay in registers across the
// barrier (no buffer the launch writes aliases them).
// SINGLE: the launch carries one pair, whose descriptor fields then sit at fixed
// parameter offsets (no per-block indexing of the parameter array).
template <bool MASKED, class ST, int TH, int MINB, bool SINGLE>
__global__ void __launch_bounds__(32 * (TH + 1), MINB) k_fused_iter(const __grid_constant__ IterArgs A, int parity) {
  typedef FusedIter<MASKED, ST> F;
  typedef typename F::T2 T2;
  typedef typename F::T4 T4;
  typedef Store2<ST> S;
  constexpr bool kFast = F::kFast;
  __shared__ float2 sTp[TH + 1][32];
  // q of the region: the primal step reads (q.x, q.w) of the west and (q.z, q.y) of the north
  // neighbour only
  __shared__ float2 sQxw[TH + 1][32], sQzy[TH + 1][32];
  // one pair: a 2-D grid of tiles; several pairs: a 1-D grid over the pairs' tile ranges
  const int t_ = blockIdx.x;
  const int pi_ = SINGLE ? 0 : find_pair(A.pr, A.npairs, t_);
  const IterPair& P = A.pr[pi_];
  int x0, y0;
  bool blk_inner = false;  // every pixel of the block's region is interior (host-computed)
  if (SINGLE) {
    int tx = (int)blockIdx.x;
    if (MASKED && A.span_rows > 0) {  // only the tiles of this row that hold a pixel that is on
      tx += A.span_lo[blockIdx.y];
      if (tx > (int)A.span_hi[blockIdx.y]) return;
      blk_inner = tx >= (int)A.in_lo[blockIdx.y] && tx <= (int)A.in_hi[blockIdx.y];
    }
    x0 = tx * 31;
    y0 = (int)blockIdx.y * TH;
  } else {
    const int lt_ = t_ - P.tile0;
    x0 = (lt_ % P.tiles_x) * 31;
    y0 = (lt_ / P.tiles_x) * TH;
  }
  const int rx = threadIdx.x, ry = threadIdx.y;
  const int ix = x0 - 1 + rx, iy = y0 - 1 + ry;
  const int plane = P.s * P.h;
  const T2* pin = (const T2*)P.p + (parity ? plane : 0);
  const T4* qin = (const T4*)P.q + (parity ? plane : 0);
  T2* pout = (T2*)P.p + (parity ? 0 : plane);
  T4* qout = (T4*)P.q + (parity ? 0 : plane);
  const bool tile = rx >= 1 && ry >= 1;
  const bool in_img = ix >= 0 && iy >= 0 && ix < P.w && iy < P.h;
  const int pos = ix + iy * P.s;
  griddep_wait();  // the previous iteration's outputs are this one's inputs
  griddep_launch_dependents();

  // ---- phase 1: dual update at every region pixel ------------------------------------
  float2 pp = make_float2(0.f, 0.f), tp = make_float2(0.f, 0.f), vb = make_float2(0.f, 0.f);
  float4 qq = make_float4(0.f, 0.f, 0.f, 0.f);
  uint8_t code = 0;
  float a = 0.f, b = 0.f, c = 0.f, ubar = 0.f;
  float u_th = 0.f, Iu_th = 0.f, Iz_th = 0.f;
  // half storage: the reciprocal preconditioners come with a, b, c from the level's records
  float r_eu = 0.f;
  float2 r_ev = make_float2(0.f, 0.f);
  if (in_img) {
    if (!blk_inner) code = P.code[pos];
    if (kFast) {
      const float4 r = P.abce[pos];
      a = r.x;
      b = r.y;
      c = r.z;
      r_eu = r.w;
    } else {
      a = P.a[pos];
      b = P.b[pos];
      c = P.c[pos];
    }
  }
  // masked form: a block with no pixel on in its region writes nothing and reads nothing
  // another block needs, so it leaves here.  With tile spans the grid holds only tiles
  // between a row's first and last tile with a pixel on, which for the fisheye circle all
  // have one; there the block-wide vote would only make every warp wait for the first load
  // round before any issues the second, so it is skipped (a tile without a pixel on then
  // does its few loads and writes nothing, as before).
  if (MASKED && A.span_rows == 0 && !__syncthreads_or(in_img && (code & kOn))) return;
  // A warp whose 32 pixels are all interior (on, with the four neighbours in the image and,
  // masked, on) takes the same operations without any of the edge rules' selections; the
  // fisheye mask's inside is most of the warps.  In a block known to be interior nothing
  // waits for the edge codes: its loads go out in one round.
  const bool inner = blk_inner || __all_sync(0xffffffffu, in_img && F::interior(code, ix, iy, P.w, P.h));
  if (inner) {
    F::dual_interior(P, pin, qin, pos, a, b, c, A.sp[pi_], A.sq[pi_], ubar, vb, pp, qq, tp, tile, u_th, Iu_th, Iz_th);
    if (tile) {
      S::st2(pout, pos, pp);
      S::st4(qout, pos, qq);
      if (A.write_tp) P.Tp[pos] = tp;
    }
  } else if (in_img) {
    bool own = F::dual_at(P, pin, qin, ix, iy, pos, code, a, b, c, A.sp[pi_], A.sq[pi_], ubar, vb, pp, qq, tp, tile,
                          u_th, Iu_th, Iz_th);
    if (own && tile) {
      S::st2(pout, pos, pp);
      S::st4(qout, pos, qq);
      if (A.write_tp) P.Tp[pos] = tp;
    }
  } else if (ix < 0 && iy >= 1 && iy < P.h) {
    // left of the image: the reference's west neighbour of column 0 is the flat
    // position before it, the last padding element of the previous row (row 0 has
    // none; positions before the buffer start read 0).  Halo pixels right of or
    // below the image are never read.
    tp = P.Tp[pos];
  }
  sTp[ry][rx] = tp;
  sQxw[ry][rx] = make_float2(qq.x, qq.w);
  sQzy[ry][rx] = make_float2(qq.z, qq.y);
  __syncthreads();
  if (!tile || !in_img) return;
  // read here rather than with the phase-1 loads, where holding it across the barrier costs
  // registers; its latency overlaps the threshold step
  if (kFast) r_ev = P.rv[pos];

  // ---- phase 2: thresholding --------------------------------------------------------
  float dxm, dym;
  bool zR, zD, hasL, hasU;
  if (inner) {  // both neighbours of each difference exist: the central forms
    dxm = tp.x - sTp[ry][rx - 1].x;
    dym = tp.y - sTp[ry - 1][rx].y;
    zR = zD = false;
    hasL = hasU = true;
  } else if (MASKED) {
    if (!(code & kOn)) return;
    bool mR = code & kR, mL = code & kL, mD = code & kD, mU = code & kU;
    if (mL && mR) dxm = tp.x - sTp[ry][rx - 1].x;
    else if (!mR) dxm = -sTp[ry][rx - 1].x;
    else dxm = tp.x;
    if (mU && mD) dym = tp.y - sTp[ry - 1][rx].y;
    else if (!mD) dym = -sTp[ry - 1][rx].y;
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
    if ((ix - 1) >= 0) dxm = tp.x - sTp[ry][rx - 1].x;
    else if (ix == P.w - 1) dxm = -sTp[ry][rx - 1].x;
    else dxm = tp.x;
    if ((iy - 1) >= 0) dym = tp.y - sTp[ry - 1][rx].y;
    else if (iy == P.h - 1) dym = -sTp[ry - 1][rx].y;
    else dym = tp.y;
    zR = ix == P.w - 1;
    zD = iy == P.h - 1;
    hasL = (ix - 1) >= 0;
    hasU = (iy - 1) >= 0;
  }
  float unew;
  if (kFast) {
    unew = fast::threshold_teu(dxm, dym, A.tau * r_eu, ubar, u_th, Iu_th, Iz_th, P.lambda);
  } else {
    float eu = etau_math(a, b, c, P.alpha1);
    unew = threshold_math(dxm, dym, eu, A.tau, ubar, u_th, Iu_th, Iz_th, P.lambda);
  }
  P.us[pos] = unew;

  // ---- phase 3: primal update ------------------------------------------------------
  float4 qc = qq;
  if (zR) qc.x = qc.w = 0.0f;
  if (zD) qc.y = qc.z = 0.0f;
  const float2 qxw_l = hasL ? sQxw[ry][rx - 1] : make_float2(0.f, 0.f);
  const float2 qzy_u = hasU ? sQzy[ry - 1][rx] : make_float2(0.f, 0.f);
  const float4 ql = make_float4(qxw_l.x, 0.f, 0.f, qxw_l.y), qu = make_float4(0.f, qzy_u.y, qzy_u.x, 0.f);
  float us_;
  float2 vs;
  if (kFast) {
    if (inner)
      fast::primal_interior_r(qq, qxw_l, qzy_u, tp, r_ev, A.tau, P.alpha0, P.alpha1, A.mu, vb, unew, ubar, us_, vs);
    else
      fast::primal_r(qc, ql, qu, tp, r_ev, A.tau, P.alpha0, P.alpha1, A.mu, vb, unew, ubar, us_, vs);
  } else {
    float ev1 = etav1_math(b, c, P.alpha0, P.alpha1), ev2 = etav2_math(a, c, P.alpha0, P.alpha1);
    float2 vo;
    primal_math(qc, ql, qu, pp, a, b, c, ev1, ev2, A.tau, P.alpha0, P.alpha1, A.mu, vb, unew, ubar, us_, vs, vo);
  }
  P.u_s[pos] = us_;
  S::st2((T2*)P.v_s, pos, vs);
}

template <int TH, int MINB, bool SINGLE>
static void launch_iter_th2(const IterArgs& A, bool masked, bool half_storage, cudaStream_t st, int parity) {
  dim3 blk(32, TH + 1), grid(A.ntiles);
  if (SINGLE) {
    grid = dim3(A.pr[0].tiles_x, (A.pr[0].h + TH - 1) / TH);
    if (masked && A.span_rows > 0) {
      if (A.span_rows != (int)grid.y) throw ArgError{"tile spans do not match the launch"};
      grid.x = A.span_max > 0 ? A.span_max : 1;
    }
  }
  if (masked) {
    if (half_storage) launch_overlapped(k_fused_iter<true, __half, TH, MINB, SINGLE>, grid, blk, st, A, parity);
    else launch_overlapped(k_fused_iter<true, float, TH, MINB, SINGLE>, grid, blk, st, A, parity);
  } else {
    if (half_storage) launch_overlapped(k_fused_iter<false, __half, TH, MINB, SINGLE>, grid, blk, st, A, parity);
    else launch_overlapped(k_fused_iter<false, float, TH, MINB, SINGLE>, grid, blk, st, A, parity);
  }
}

template <int TH, int MINB>
static void launch_iter_th(const IterArgs& A, bool masked, bool half_storage, cudaStream_t st, int parity) {
  if (A.npairs == 1) launch_iter_th2<TH, MINB, true>(A, masked, half_storage, st, parity);
  else launch_iter_th2<TH, MINB, false>(A, masked, half_storage, st, parity);
}

namespace {
template <int TH, int MINB>
int blocks_per_sm_th(bool masked, bool half) {
  int n = 0;
  const int threads = 32 * (TH + 1);
  if (masked) {
    if (half) VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter<true, __half, TH, MINB, true>, threads, 0));
    else VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter<true, float, TH, MINB, true>, threads, 0));
  } else {
    if (half) VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter<false, __half, TH, MINB, true>, threads, 0));
    else VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused_iter<false, float, TH, MINB, true>, threads, 0));
  }
  return n;
}
}  // namespace

double iteration_gpu_share(int variant, bool masked, bool half, int w, int h) {
  // blocks of the launch and resident blocks per SM of the variant's kernel (one pair)
  long long blocks = 0;
  int per_sm = 0;
  if (iter_variant_cluster(variant)) {
    return cluster_gpu_share(variant, w, h);
  } else if (variant == kIterTmaVariant) {
    return tma_gpu_share(masked, half, w, h);
  } else if (variant >= kIterFirstTBVariant && !iter_variant_tiled(variant)) {
    return tb_gpu_share(variant, masked, half, w, h);
  } else {
    const int rows = kIterVariantRows[variant];
    blocks = (long long)iter_tiles_of(w, h, rows);
    switch (variant) {
      case 0: per_sm = blocks_per_sm_th<4, kIterVariantMinBlocks[0]>(masked, half); break;
      case 2: per_sm = blocks_per_sm_th<16, kIterVariantMinBlocks[2]>(masked, half); break;
      case 19: per_sm = blocks_per_sm_th<15, kIterVariantMinBlocks[19]>(masked, half); break;
      default: per_sm = blocks_per_sm_th<8, kIterVariantMinBlocks[1]>(masked, half); break;
    }
  }
  int dev = 0, sms = 1;
  VFS_CUDA(cudaGetDevice(&dev));
  VFS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const double cap = (double)sms * (per_sm > 0 ? per_sm : 1);
  return blocks >= cap ? 1.0 : (double)blocks / cap;
}

void launch_fused_iteration(const IterArgs& A, bool masked, bool half_storage, cudaStream_t st, int parity,
                            int variant) {
  if (A.ntiles <= 0) return;
  static_assert(kIterVariantRows[0] == 4 && kIterVariantRows[1] == 8 && kIterVariantRows[2] == 16 &&
                    kIterVariantRows[19] == 15,
                "variants");
  if (iter_variant_retired(variant) || variant == kIterTmaVariant) throw ArgError{"not a k_fused_iter variant"};
  switch (variant) {
    case 0: launch_iter_th<4, kIterVariantMinBlocks[0]>(A, masked, half_storage, st, parity); break;
    case 2: launch_iter_th<16, kIterVariantMinBlocks[2]>(A, masked, half_storage, st, parity); break;
    case 19: launch_iter_th<15, kIterVariantMinBlocks[19]>(A, masked, half_storage, st, parity); break;
    default: launch_iter_th<8, kIterVariantMinBlocks[1]>(A, masked, half_storage, st, parity); break;
  }
  VFS_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Per-warp prologue: zero p, q (both halves) and v-bar; tv2 = tv(x + warpUV);
// i1warp = I1(x + warpUV)  (stereotgv.cu:431-439; warpImage.cu:9-23, 96-111), stored in
// the storage type (rounded to half with half storage)
// ---------------------------------------------------------------------------
// the prologue at one pixel of a pair (pos = ix + iy * s; warpUV already read)
template <class ST>
__device__ __forceinline__ void warp_start_at(const WarpStartPair& P, int ix, int iy, long long pos, float2 wv) {
  typedef Store2<ST> S;
  long long plane = (long long)P.s * P.h;
  typename S::T2* p = (typename S::T2*)P.p;
  typename S::T4* q = (typename S::T4*)P.q;
  S::st2(p, pos, make_float2(0.f, 0.f));
  S::st2(p, pos + plane, make_float2(0.f, 0.f));
  S::st4(q, pos, make_float4(0.f, 0.f, 0.f, 0.f));
  S::st4(q, pos + plane, make_float4(0.f, 0.f, 0.f, 0.f));
  S::st2((typename S::T2*)P.v_, pos, make_float2(0.f, 0.f));
  float x = ((float)ix + wv.x + 0.5f) / (float)P.w;
  float y = ((float)iy + wv.y + 0.5f) / (float)P.h;
  P.tv2[pos] = tex2D<float2>(P.texTv, x, y);
  ((ST*)P.i1warp)[pos] = (ST)tex2D<float>(P.texI1, x, y);
}

template <class ST>
__global__ void __launch_bounds__(kFTW* kFTH) k_warp_start(const __grid_constant__ WarpStartArgs A) {
  TILE_SETUP(A)
  if (ix >= P.w || iy >= P.h) return;
  long long pos = ix + (long long)iy * P.s;
  warp_start_at<ST>(P, ix, iy, pos, P.warpUV[pos]);
}

void launch_warp_start(const WarpStartArgs& A, bool half_storage, cudaStream_t st) {
  if (A.ntiles <= 0) return;
  dim3 blk(kFTW, kFTH);
  if (half_storage) k_warp_start<__half><<<A.ntiles, blk, 0, st>>>(A);
  else k_warp_start<float><<<A.ntiles, blk, 0, st>>>(A);
  VFS_LAUNCH_CHECK();
}

// computeDerivatives.cu:89-129 and Clone(u_last, u) (stereotgv.cu:447)
__global__ void __launch_bounds__(kFTW* kFTH) k_derivatives_b(const __grid_constant__ DerivArgs A) {
  TILE_SETUP(A)
  if (ix >= P.w || iy >= P.h) return;
  long long pos = ix + (long long)iy * P.s;
  float2 vv = P.tv[pos];
  float r = sqrtf(vv.x * vv.x + vv.y * vv.y);
  float dx = (vv.x / r) / (float)P.w;
  float dy = (vv.y / r) / (float)P.h;
  float x = ((float)ix + 0.5f) / (float)P.w;
  float y = ((float)iy + 0.5f) / (float)P.h;
  cudaTextureObject_t I0 = P.texI0, I1 = P.texI1w;
  float t0 = tex2D<float>(I0, x - 2.0f * dx, y - 2.0f * dy);
  t0 -= tex2D<float>(I0, x - 1.0f * dx, y - 1.0f * dy) * 8.0f;
  t0 += tex2D<float>(I0, x + 1.0f * dx, y + 1.0f * dy) * 8.0f;
  t0 -= tex2D<float>(I0, x + 2.0f * dx, y + 2.0f * dy);
  t0 /= 12.0f;
  float t1 = tex2D<float>(I1, x - 2.0f * dx, y - 2.0f * dy);
  t1 -= tex2D<float>(I1, x - 1.0f * dx, y - 1.0f * dy) * 8.0f;
  t1 += tex2D<float>(I1, x + 1.0f * dx, y + 1.0f * dy) * 8.0f;
  t1 -= tex2D<float>(I1, x + 2.0f * dx, y + 2.0f * dy);
  t1 /= 12.0f;
  P.Iu[pos] = (t0 + t1) * 0.5f;
  P.Iz[pos] = tex2D<float>(I1, x, y) - tex2D<float>(I0, x, y);
  P.u_last[pos] = P.u[pos];
}

void launch_derivatives_batched(const DerivArgs& A, cudaStream_t st) {
  if (A.ntiles <= 0) return;
  k_derivatives_b<<<A.ntiles, dim3(kFTW, kFTH), 0, st>>>(A);
  VFS_LAUNCH_CHECK();
}

// stereotgv.cu:481-493: median (masked form), du = min(u - u_last, limit),
// u = u_last + du, u-bar = u, warpUV += du * tv2
// the epilogue at one pixel of a pair; returns the updated warpUV it stored
__device__ __forceinline__ float2 epilogue_at(const EpiPair& P, bool median, int ix, int iy, long long pos) {
  float m = median ? median5_at(P.u_in, ix, iy, P.w, P.h, P.s) : P.u_in[pos];
  float ul = P.u_last[pos];
  float d = m - ul;
  d = d > P.limitRange ? P.limitRange : d;
  float un = ul + d;
  P.u_out[pos] = un;
  P.u_bar[pos] = un;
  float2 t = P.tv2[pos];
  float2 dw = make_float2(d * t.x, d * t.y);
  float2 wv = P.warpUV[pos];
  wv = make_float2(wv.x + dw.x, wv.y + dw.y);
  P.warpUV[pos] = wv;
  return wv;
}

__global__ void __launch_bounds__(kFTW* kFTH) k_epilogue_b(const __grid_constant__ EpiArgs A) {
  TILE_SETUP(A)
  if (ix >= P.w || iy >= P.h) return;
  epilogue_at(P, A.median != 0, ix, iy, ix + (long long)iy * P.s);
}

// The epilogue of one warp and the prologue of the next in one launch: both touch only their
// own pixel's warpUV, tv2 and warped image (the epilogue reads tv2 before the prologue
// replaces it; the median reads u, which the prologue does not write), and the pairs' tiles
// are the same in both argument sets.
template <class ST>
__global__ void __launch_bounds__(kFTW* kFTH) k_epilogue_warp_start(const __grid_constant__ EpiArgs A,
                                                                   const __grid_constant__ WarpStartArgs B) {
  TILE_SETUP(A)
  if (ix >= P.w || iy >= P.h) return;
  const long long pos = ix + (long long)iy * P.s;
  const float2 wv = epilogue_at(P, A.median != 0, ix, iy, pos);
  warp_start_at<ST>(B.pr[pi_], ix, iy, pos, wv);
}

void launch_epilogue_warp_start(const EpiArgs& A, const WarpStartArgs& B, bool half_storage, cudaStream_t st) {
  if (A.ntiles <= 0) return;
  if (B.npairs != A.npairs || B.ntiles != A.ntiles) throw ArgError{"epilogue and warp start tiles differ"};
  dim3 blk(kFTW, kFTH);
  if (half_storage) k_epilogue_warp_start<__half><<<A.ntiles, blk, 0, st>>>(A, B);
  else k_epilogue_warp_start<float><<<A.ntiles, blk, 0, st>>>(A, B);
  VFS_LAUNCH_CHECK();
}

void launch_warp_epilogue_batched(const EpiArgs& A, cudaStream_t st) {
  if (A.ntiles <= 0) return;
  k_epilogue_b<<<A.ntiles, dim3(kFTW, kFTH), 0, st>>>(A);
  VFS_LAUNCH_CHECK();
}

// calcTensor.cu:99-128 / 245-273 with the per-level zeroing of stereotgv.cu:409-415:
// i0smooth = gaussian where computed, 0 elsewhere (level footprint); at a pair's
// coarsest level also warpUV = u * tv (stereotgv.cu:419-421).
__global__ void __launch_bounds__(kFTW* kFTH) k_level_gaussian(const __grid_constant__ LevelArgs A) {
  TILE_SETUP(A)
  if (ix >= P.w || iy >= P.h) return;
  long long pos = ix + (long long)iy * P.s;
  if (P.init_flow) {
    float us = P.u[pos];
    float2 t = P.tv[pos];
    P.warpUV[pos] = make_float2(us * t.x, us * t.y);
  }
  if (P.mask && P.mask[pos] == 0.0f) {
    P.i0smooth[pos] = 0.0f;
    return;
  }
  float dx = 1.0f / (float)P.w, dy = 1.0f / (float)P.h;
  float x = ((float)ix + 0.5f) * dx, y = ((float)iy + 0.5f) * dy;
  cudaTextureObject_t in = P.texI0;
  float t0 = (1 / 4.0f) * tex2D<float>(in, x, y);
  t0 += (1 / 16.0f) * tex2D<float>(in, x - 1.0f * dx, y - 1.0f * dy);
  t0 += (1 / 16.0f) * tex2D<float>(in, x - 1.0f * dx, y + 1.0f * dy);
  t0 += (1 / 16.0f) * tex2D<float>(in, x + 1.0f * dx, y - 1.0f * dy);
  t0 += (1 / 16.0f) * tex2D<float>(in, x + 1.0f * dx, y + 1.0f * dy);
  t0 += (1 / 8.0f) * tex2D<float>(in, x - 1.0f * dx, y);
  t0 += (1 / 8.0f) * tex2D<float>(in, x + 1.0f * dx, y);
  t0 += (1 / 8.0f) * tex2D<float>(in, x, y - 1.0f * dy);
  t0 += (1 / 8.0f) * tex2D<float>(in, x, y + 1.0f * dy);
  P.i0smooth[pos] = t0;
}

// The half-storage iteration's per-level records at one pixel: (a, b, c, 1 / eta_u) and
// (1 / eta_v1, 1 / eta_v2), formed by the same expressions the iteration kernels use
// (tgv_pixel_fast.cuh, a1s = alpha1^2, a0s4 = 4 alpha0^2), so reading them gives the bits of
// recomputing them.
__device__ __forceinline__ void level_records(const LevelPair& P, long long pos, float a, float b, float c) {
  const float a1s = P.alpha1 * P.alpha1, a0s4 = 4.0f * P.alpha0 * P.alpha0;
  P.abce[pos] = make_float4(a, b, c, fast::etau_rcp(fast::etau(a, b, c, a1s)));
  P.rv[pos] = fast::etav_rcp(fast::etav(b, c, a1s, a0s4), fast::etav(a, c, a1s, a0s4));
}

// calcTensor.cu:8-73 / 155-219; a = b = c = 0 where the reference does not compute
// (masked out, or columns >= xmax of its launch grid)
__global__ void __launch_bounds__(kFTW* kFTH) k_level_tensor(const __grid_constant__ LevelArgs A) {
  TILE_SETUP(A)
  if (ix >= P.w || iy >= P.h) return;
  long long pos = ix + (long long)iy * P.s;
  if (ix >= P.xmax || (P.mask && P.mask[pos] == 0.0f)) {
    P.a[pos] = 0.0f;
    P.b[pos] = 0.0f;
    P.c[pos] = 0.0f;
    if (P.abce) level_records(P, pos, 0.0f, 0.0f, 0.0f);
    return;
  }
  float dx = 1.0f / (float)P.w, dy = 1.0f / (float)P.h;
  float x = ((float)ix + 0.5f) * dx, y = ((float)iy + 0.5f) * dy;
  cudaTextureObject_t gray = P.texSmooth;
  float gx = tex2D<float>(gray, x + 1.0f * dx, y + 1.0f * dy) - tex2D<float>(gray, x, y + 1.0f * dy);
  float gy = tex2D<float>(gray, x + 1.0f * dx, y + 1.0f * dy) - tex2D<float>(gray, x + 1.0f * dx, y);
  float abs_img = sqrtf(gx * gx + gy * gy);
  float norm_n = abs_img;
  float nx = gx / norm_n, ny = gy / norm_n;
  if (norm_n < 1e-8f) {
    nx = 1.0f;
    ny = 0.0f;
  }
  float ntx = ny, nty = -nx;
  float wt = tensor_weight(abs_img, P.beta, P.gamma, P.cuda_math);
  if (!(wt > 1e-8f)) wt = 1e-8f;
  const float a = wt * nx * nx + ntx * ntx, c = wt * nx * ny + ntx * nty, b = wt * ny * ny + nty * nty;
  P.a[pos] = a;
  P.c[pos] = c;
  P.b[pos] = b;
  if (P.abce) level_records(P, pos, a, b, c);
}

void launch_level_gaussian(const LevelArgs& A, cudaStream_t st) {
  if (A.ntiles <= 0) return;
  k_level_gaussian<<<A.ntiles, dim3(kFTW, kFTH), 0, st>>>(A);
  VFS_LAUNCH_CHECK();
}
void launch_level_tensor(const LevelArgs& A, cudaStream_t st) {
  if (A.ntiles <= 0) return;
  k_level_tensor<<<A.ntiles, dim3(kFTW, kFTH), 0, st>>>(A);
  VFS_LAUNCH_CHECK();
}

// upscale.cu:8-21, 46-61 for u, u-bar and warpUV (stereotgv.cu:497-510)
__global__ void __launch_bounds__(kFTW* kFTH) k_upscale3(const __grid_constant__ UpArgs A) {
  TILE_SETUP(A)
  if (ix >= P.w || iy >= P.h) return;
  long long pos = ix + (long long)iy * P.s;
  float x = ((float)ix + 0.5f) / (float)P.w;
  float y = ((float)iy + 0.5f) / (float)P.h;
  P.u_out[pos] = tex2D<float>(P.texU, x, y) * P.scale;
  P.ubar_out[pos] = tex2D<float>(P.texUbar, x, y) * P.scale;
  float2 v = tex2D<float2>(P.texWarp, x, y);
  P.warp_out[pos] = make_float2(v.x * P.scale, v.y * P.scale);
}

void launch_upscale_batched(const UpArgs& A, cudaStream_t st) {
  if (A.ntiles <= 0) return;
  k_upscale3<<<A.ntiles, dim3(kFTW, kFTH), 0, st>>>(A);
  VFS_LAUNCH_CHECK();
}

// downscale.cu:10-30 for I0 and I1 (stereotgv.cu:400-405)
__global__ void __launch_bounds__(kFTW* kFTH) k_downscale2img(const __grid_constant__ DownArgs A) {
  TILE_SETUP(A)
  if (ix >= P.w || iy >= P.h) return;
  float dx = 1.0f / (float)P.w, dy = 1.0f / (float)P.h;
  float x = ((float)ix + 0.5f) * dx, y = ((float)iy + 0.5f) * dy;
  long long pos = ix + (long long)iy * P.s;
  {
    cudaTextureObject_t f = P.texI0;
    float t1 = tex2D<float>(f, x - dx * 0.25f, y);
    float t2 = tex2D<float>(f, x + dx * 0.25f, y);
    float t3 = tex2D<float>(f, x, y - dy * 0.25f);
    float t4 = tex2D<float>(f, x, y + dy * 0.25f);
    P.I0[pos] = 0.25f * (t1 + t2 + t3 + t4);
  }
  {
    cudaTextureObject_t f = P.texI1;
    float t1 = tex2D<float>(f, x - dx * 0.25f, y);
    float t2 = tex2D<float>(f, x + dx * 0.25f, y);
    float t3 = tex2D<float>(f, x, y - dy * 0.25f);
    float t4 = tex2D<float>(f, x, y + dy * 0.25f);
    P.I1[pos] = 0.25f * (t1 + t2 + t3 + t4);
  }
}

void launch_downscale_batched(const DownArgs& A, cudaStream_t st) {
  if (A.ntiles <= 0) return;
  k_downscale2img<<<A.ntiles, dim3(kFTW, kFTH), 0, st>>>(A);
  VFS_LAUNCH_CHECK();
}

// Edge codes: masked form from the level's mask (neighbours outside the image are
// off), plain form (mask == nullptr) flags the pixels inside the fixed circle.
__global__ void k_edge_codes(const float* __restrict__ mask, uint8_t* code, int w, int h, int s) {
  int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y;
  if (ix >= w || iy >= h) return;
  long long pos = ix + (long long)iy * s;
  uint8_t c = 0;
  if (mask) {
    if (mask[pos] != 0.0f) c |= kOn;
    if (ix + 1 < w && mask[pos + 1] != 0.0f) c |= kR;
    if (ix - 1 >= 0 && mask[pos - 1] != 0.0f) c |= kL;
    if (iy + 1 < h && mask[pos + s] != 0.0f) c |= kD;
    if (iy - 1 >= 0 && mask[pos - s] != 0.0f) c |= kU;
  } else {
    if (!outside_circle(ix, iy, w, h)) c |= kOn;
  }
  code[pos] = c;
}

void launch_edge_codes(const float* mask, uint8_t* code, int w, int h, int s, cudaStream_t st) {
  k_edge_codes<<<dim3((w + 31) / 32, (h + 7) / 8), dim3(32, 8), 0, st>>>(mask, code, w, h, s);
  VFS_LAUNCH_CHECK();
}

}  // namespace vfs
