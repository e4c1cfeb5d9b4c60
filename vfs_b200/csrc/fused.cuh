// Fused, batched kernels of the fast solve path.
//
// A launch covers one pair (the batch's concurrent mode, and single solves) or every pair
// of a batch at one pyramid level (its one-launch mode); pairs may differ in size.
// Per-pair state is passed by value in the kernel parameters (up to kMaxPairs pairs), with
// the pointers that are current at that launch, so a launch sequence can be captured once
// in a CUDA graph and replayed.
//
// With float storage the fused kernels compute bit-for-bit what the per-kernel
// drop-in path computes: the same operations in the same order on the same
// physical buffers (including the stale values that masked-out pixels keep), so
// the two paths agree exactly.  With half storage p, q and v-bar are kept as
// IEEE half in memory and widened to float for all arithmetic.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace vfs {

constexpr int kMaxPairs = 24;
constexpr int kFTW = 32;  // fused iteration tile: 32 x 8 pixels, one thread each
constexpr int kFTH = 8;

// per-level edge code of each pixel (computed once per mask upload):
//   bit0 mask(x) != 0, bit1 right neighbour on, bit2 left on, bit3 down on, bit4 up on
// (a neighbour outside the image counts as off, as in the reference's masked kernels)
enum : uint8_t { kOn = 1, kR = 2, kL = 4, kD = 8, kU = 16 };

template <class ST>
struct Store2;  // storage of a 2-vector (p, v-bar) and a 4-vector (q)
template <>
struct Store2<float> {
  typedef float2 T2;
  typedef float4 T4;
  static __device__ __forceinline__ float2 ld2(const T2* b, long long k) { return b[k]; }
  static __device__ __forceinline__ void st2(T2* b, long long k, float2 v) { b[k] = v; }
  static __device__ __forceinline__ float4 ld4(const T4* b, long long k) { return b[k]; }
  static __device__ __forceinline__ void st4(T4* b, long long k, float4 v) { b[k] = v; }
  // conversions between the stored form and float (identities here)
  static __device__ __forceinline__ T2 ld2z() { return make_float2(0.f, 0.f); }
  static __device__ __forceinline__ T4 ld4z() { return make_float4(0.f, 0.f, 0.f, 0.f); }
  static __device__ __forceinline__ float2 cvt2(T2 v) { return v; }
  static __device__ __forceinline__ float4 cvt4(T4 v) { return v; }
  static __device__ __forceinline__ T2 rnd2(float2 v) { return v; }
  static __device__ __forceinline__ T4 rnd4(float4 v) { return v; }
};
template <>
struct Store2<__half> {
  typedef __half2 T2;
  struct __align__(8) T4 { __half2 a, b; };
  static __device__ __forceinline__ float2 ld2(const T2* b, long long k) { return __half22float2(b[k]); }
  static __device__ __forceinline__ void st2(T2* b, long long k, float2 v) { b[k] = __float22half2_rn(v); }
  static __device__ __forceinline__ float4 ld4(const T4* b, long long k) {
    T4 t = b[k];
    float2 x = __half22float2(t.a), y = __half22float2(t.b);
    return make_float4(x.x, x.y, y.x, y.y);
  }
  static __device__ __forceinline__ void st4(T4* b, long long k, float4 v) { b[k] = rnd4(v); }
  // conversions between the stored form and float, the same roundings as ld / st above
  static __device__ __forceinline__ T2 ld2z() { return __floats2half2_rn(0.f, 0.f); }
  static __device__ __forceinline__ T4 ld4z() {
    T4 t;
    t.a = ld2z();
    t.b = ld2z();
    return t;
  }
  static __device__ __forceinline__ float2 cvt2(T2 v) { return __half22float2(v); }
  static __device__ __forceinline__ float4 cvt4(T4 t) {
    float2 x = __half22float2(t.a), y = __half22float2(t.b);
    return make_float4(x.x, x.y, y.x, y.y);
  }
  static __device__ __forceinline__ T2 rnd2(float2 v) { return __float22half2_rn(v); }
  static __device__ __forceinline__ T4 rnd4(float4 v) {
    T4 t;
    t.a = __float22half2_rn(make_float2(v.x, v.y));
    t.b = __float22half2_rn(make_float2(v.z, v.w));
    return t;
  }
};

// Locate the pair that owns tile t from the batch's tile ranges.
template <class PairT, int N>
__device__ __forceinline__ int find_pair(const PairT (&pr)[N], int npairs, int t) {
  int k = 0;
  while (k + 1 < npairs && t >= pr[k + 1].tile0) k++;
  return k;
}

// ---- one primal-dual iteration -------------------------------------------------
struct IterPair {
  const uint8_t* code;  // edge codes (masked form) or inside-circle flags (plain form)
  const float* u_;      // u-bar (current)
  const float* u;       // u (current)
  const void* v_;       // v-bar (current), Store2<ST>::T2
  void* p;              // T2, in place
  void* q;              // T4, in place
  float2* Tp;           // T p (float); read for masked-out neighbours, written when write_tp
  const float *a, *b, *c, *Iu, *Iz;
  // half storage: the level's coefficient records (k_level_tensor), read by k_fused_iter in
  // place of a, b, c: (a, b, c, etau_rcp) and etav_rcp (tgv_pixel_fast.cuh); null otherwise
  const float4* abce;
  const float2* rv;
  float* us;            // thresholded u (output)
  float* u_s;           // new u-bar (output)
  void* v_s;            // new v-bar (output), T2
  int w, h, s, tiles_x, tile0;
  float alpha0, alpha1, lambda;
};
constexpr int kMaxSpanRows = 256;
struct IterArgs {
  int npairs, ntiles;
  float sigma, tau, mu;
  float sp[kMaxPairs], sq[kMaxPairs];  // alpha1 sigma / 3 and alpha0 sigma / 2 per pair (host-evaluated)
  int write_tp;
  IterPair pr[kMaxPairs];
  // One-pair masked launches of k_fused_iter: with span_rows > 0 the grid covers, in tile row
  // r, only the tile columns span_lo[r] .. span_hi[r] (the tiles whose region holds a pixel
  // that is on); the others would write nothing.  span_max: the widest span (grid width).
  int span_rows, span_max;
  uint16_t span_lo[kMaxSpanRows], span_hi[kMaxSpanRows];
  // With tile spans, tiles in_lo[r] .. in_hi[r] of tile row r (none where in_lo > in_hi) have
  // a region whose every pixel is interior: on, with its four neighbours in the image and on.
  uint16_t in_lo[kMaxSpanRows], in_hi[kMaxSpanRows];
};
// parity selects which half of the p / q ping-pong buffers is read (the other is written);
// variant selects the tile height (kIterVariantRows[variant] rows of 31 pixels).
void launch_fused_iteration(const IterArgs& A, bool masked, bool half_storage, cudaStream_t st, int parity,
                            int variant);

// ---- K consecutive primal-dual iterations of one pair in one launch (kernels_tb.cu) ----
constexpr int kIterTBMax = 9;
struct IterTBArgs {
  IterPair P;  // pointers of the launch's first iteration (its outputs: us, u_s, v_s)
  float sp[kIterTBMax], sq[kIterTBMax], tau[kIterTBMax], mu[kIterTBMax];  // per iteration
  int parity;    // p / q plane read by the first iteration
  int write_tp;  // 1: the last iteration of the launch stores T p
};
// iterations per launch of an iteration-kernel variant (1 for the one-iteration forms)
int tb_iterations(int variant);

// ---- up to kCLMaxIters iterations of one small level in one launch of a thread-block
// cluster that holds the level in shared memory (kernels_cluster.cu) ----
constexpr int kCLMaxIters = 64;
struct IterCLArgs {
  IterPair P;  // pointers of the launch's first iteration
  float sp[kCLMaxIters], sq[kCLMaxIters], tau[kCLMaxIters], mu[kCLMaxIters];  // per iteration
  int n;         // iterations (1 .. kCLMaxIters)
  int parity;    // p / q plane read by the first iteration
  int write_tp;  // 1: the last iteration stores T p
  int rows;      // image rows per CTA (cluster_rows)
  int ctas;      // CTAs of the cluster (cluster_ctas); the grid is one cluster
};
// CTAs per cluster of a cluster-resident variant (0 for the other variants)
int cluster_ctas(int variant);
// image rows each CTA owns for a level of height h
int cluster_rows(int variant, int h);
// the level's state fits the cluster's shared memory and such a cluster can be resident
bool cluster_fits(int variant, bool masked, bool half, int w, int h);
// solves of the process that timed iteration-kernel variants (vfs_tuning_solves)
long long tuning_solve_count();
// owned pixels per thread of the cluster-resident kernel on a w x h level (0: not a cluster variant)
int cluster_pixels_per_thread(int variant, bool half, int w, int h);
double cluster_gpu_share(int variant, int w, int h);
void launch_fused_iteration_cluster(const IterCLArgs& A, bool masked, bool half_storage, cudaStream_t st,
                                    int variant);
// Fraction of the GPU's resident-block capacity that one launch of a variant for one pair of
// w x h pixels occupies (1 when it fills or exceeds a wave); the tuner's cost model.
double iteration_gpu_share(int variant, bool masked, bool half, int w, int h);
double tb_gpu_share(int variant, bool masked, bool half, int w, int h);
void launch_fused_iteration_tb(const IterTBArgs& A, bool masked, bool half_storage, cudaStream_t st, int variant);
// one iteration of one pair with its region staged by TMA (variant 18, kernels_tma.cu); A is
// laid out as for variant 1 (8-row tiles, tile spans)
void launch_fused_iteration_tma(const IterArgs& A, bool masked, bool half_storage, cudaStream_t st, int parity);
double tma_gpu_share(bool masked, bool half, int w, int h);
// reads and clears the device status of the TMA iteration kernel (1: a bounded wait ran out)
int tma_status_take();

// ---- per-warp prologue: zero p, q, v-bar; resample tv at x + warpUV; warp I1 ----
struct WarpStartPair {
  cudaTextureObject_t texI1, texTv;
  const float2* warpUV;
  float2* tv2;
  void* i1warp;  // warped image: float, or half with half_storage
  void *p, *q, *v_;  // zeroed (px < w); storage type by half_storage
  int w, h, s, tiles_x, tile0;
};
struct WarpStartArgs {
  int npairs, ntiles;
  WarpStartPair pr[kMaxPairs];
};
void launch_warp_start(const WarpStartArgs& A, bool half_storage, cudaStream_t st);

// ---- derivatives along the translation field + u_last = u -----------------------
struct DerivPair {
  cudaTextureObject_t texI0, texI1w;  // texI1w over the warped image as stored (float or half)
  const float2* tv;
  float *Iu, *Iz;
  const float* u;
  float* u_last;
  int w, h, s, tiles_x, tile0;
};
struct DerivArgs {
  int npairs, ntiles;
  DerivPair pr[kMaxPairs];
};
void launch_derivatives_batched(const DerivArgs& A, cudaStream_t st);

// ---- 5x5 median (masked form) + range limit + u / u-bar / warpUV update ----------
struct EpiPair {
  const float* u_in;   // u after the inner loop (median input)
  float* u_out;        // receives u_last + min(median - u_last, limit)
  float* u_bar;        // u-bar = u
  const float* u_last;
  const float2* tv2;
  float2* warpUV;      // += du * tv2
  int w, h, s, tiles_x, tile0;
  float limitRange;
};
struct EpiArgs {
  int npairs, ntiles;
  int median;  // 1: masked form applies the 5x5 median first
  EpiPair pr[kMaxPairs];
};
void launch_warp_epilogue_batched(const EpiArgs& A, cudaStream_t st);
// the epilogue (A) and the next warp's prologue (B, same pairs and tiles) in one launch
void launch_epilogue_warp_start(const EpiArgs& A, const WarpStartArgs& B, bool half_storage, cudaStream_t st);

// ---- per-level setup: gaussian (+ zero where not computed), tensor (+ zero) -------
struct LevelPair {
  cudaTextureObject_t texI0, texSmooth;
  const float* mask;  // nullptr: plain form
  float* i0smooth;
  float *a, *b, *c;
  float2* warpUV;        // coarsest level: warpUV = u * tv (u = 0)
  const float* u;
  const float2* tv;
  int init_flow;         // 1 at a pair's coarsest level
  int w, h, s, xmax, tiles_x, tile0;
  float beta, gamma;
  int cuda_math;  // tensor weight from CUDA's expf / powf (1) or the portable construction (0)
  // half storage: also write the coefficient records of the iteration (IterPair::abce / rv),
  // whose reciprocal preconditioners take alpha0 and alpha1; null otherwise
  float4* abce;
  float2* rv;
  float alpha0, alpha1;
};
struct LevelArgs {
  int npairs, ntiles;
  LevelPair pr[kMaxPairs];
};
void launch_level_gaussian(const LevelArgs& A, cudaStream_t st);
void launch_level_tensor(const LevelArgs& A, cudaStream_t st);

// ---- upscale u, u-bar and warpUV to the next finer level in one pass --------------
struct UpPair {
  cudaTextureObject_t texU, texUbar, texWarp;
  float *u_out, *ubar_out;
  float2* warp_out;
  int w, h, s, tiles_x, tile0;  // fine level
  float scale;
};
struct UpArgs {
  int npairs, ntiles;
  UpPair pr[kMaxPairs];
};
void launch_upscale_batched(const UpArgs& A, cudaStream_t st);

// ---- pyramid: downscale I0 and I1 of every pair to the next coarser level --------
struct DownPair {
  cudaTextureObject_t texI0, texI1;
  float *I0, *I1;
  int w, h, s, tiles_x, tile0;  // coarse level
};
struct DownArgs {
  int npairs, ntiles;
  DownPair pr[kMaxPairs];
};
void launch_downscale_batched(const DownArgs& A, cudaStream_t st);

// edge codes of one level from its mask (masked form) or the fixed circle (plain)
void launch_edge_codes(const float* mask, uint8_t* code, int w, int h, int s, cudaStream_t st);

// tile bookkeeping shared by the batched launches (32 x 8 tiles)
inline int tiles_x_of(int w) { return (w + kFTW - 1) / kFTW; }
inline int tiles_of(int w, int h) { return tiles_x_of(w) * ((h + kFTH - 1) / kFTH); }
// the iteration kernel's tiles: 31 x kIterTH pixels (a 32 x (kIterTH + 1) block with halo)
// Variants of the iteration kernel (chosen per level by the autotuner in FusedEngine): rows
// per tile and the minimum resident blocks per SM its launch bounds ask for (which caps
// registers at 32 or 40 per thread).  All give identical results.
// Variants 0-2: k_fused_iter (32 x (rows + 1) blocks, shared-memory west / north exchange).
// Variants 6-9: k_fused_iter_tb, several iterations per launch with the tile's region in
// shared memory (kernels_tb.cu), one pair per launch only: 3 iterations on 64 x 24 tiles,
// 5 on 32 x 24, and with one region pixel per thread 3 on 23 x 23 and 5 on 17 x 17 tiles.
// Variants 12-13: k_fused_iter_tb with one region pixel per thread, 7 iterations on 11 x 11
// tiles and 9 on 5 x 5 tiles (for the smallest levels, where the GPU is mostly idle).
// Variants 14-15: k_fused_iter_cluster, the whole level in the shared memory of a cluster of
// 16 / 8 CTAs, all iterations of a warp (up to kCLMaxIters) per launch, two cluster
// barriers per iteration.  Levels that do not fit use the default variant.
// Variant 18: k_fused_iter_tma (kernels_tma.cu), the 8-row tiles of variant 1 with every input
// plane of the block's region brought into shared memory by bulk tensor copies (TMA); one pair
// per launch, on levels where no pixel of column 0 is on (masked form).
// Variant 19: k_fused_iter with 15-row tiles (512 threads, 4 blocks per SM): 64 resident
// warps per SM, as against 63 with 8-row tiles, and 9 % of the threads on the halo, against
// 14 %.
// Numbers 3-5, 10-11 and 16-17 belonged to forms that never won on B200 (a warp streaming a
// row strip, two pixels per thread, one cluster barrier per iteration) and were removed;
// they are rejected, and the remaining numbers keep their meaning.
constexpr int kIterVariants = 20;
constexpr int kIterVariantRows[kIterVariants] = {4, 8, 16, 0, 0, 0, 24, 24, 23, 17, 0, 0, 11, 5, 0, 0, 0, 0, 8, 15};
constexpr int kIterVariantMinBlocks[kIterVariants] = {12, 7, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 4};
constexpr int kIterTmaVariant = 18;
constexpr int kIterFirstTBVariant = 6;
inline bool iter_variant_retired(int v) { return (v >= 3 && v <= 5) || v == 10 || v == 11 || v == 16 || v == 17; }
inline bool iter_variant_valid(int v) { return v >= 0 && v < kIterVariants && !iter_variant_retired(v); }
// the k_fused_iter variants (one iteration per launch, one or several pairs per launch)
inline bool iter_variant_tiled(int v) { return v == 0 || v == 1 || v == 2 || v == 19; }
// per-row tile spans are kept for each k_fused_iter tile height; the slot of a variant
constexpr int kIterSpanSlots = 4;
inline int iter_span_slot(int v) { return v <= 2 ? v : v == 19 ? 3 : -1; }
// variants whose launch carries one pair only (others fall back to the default there)
inline bool iter_variant_single_pair(int v) { return v >= kIterFirstTBVariant && !iter_variant_tiled(v); }
constexpr int kIterFirstDeepTBVariant = 12;
constexpr int kIterFirstClusterVariant = 14;
inline bool iter_variant_cluster(int v) { return v == kIterFirstClusterVariant || v == kIterFirstClusterVariant + 1; }
constexpr int kIterDefaultVariant = 1;
inline int iter_tiles_x_of(int w) { return (w + 30) / 31; }
inline int iter_tiles_of(int w, int h, int rows) { return iter_tiles_x_of(w) * ((h + rows - 1) / rows); }

}  // namespace vfs
