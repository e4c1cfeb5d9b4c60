// Launchers of the per-operation kernels of the drop-in solve path.  Each kernel
// computes exactly what the reference kernel named in its comment computes, on the
// same pixels, with the same floating-point operation order (the library is built
// with -fmad=false so that no multiply-add is contracted).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace vfs {

// Geometry of one pyramid level: logical size and row pitch (elements).
struct Geom {
  int w, h, s;
};

// imageConverter.cu:4-15 / :27-41
void launch_cv8u_to_gray(const uint8_t* src, float* dst, Geom g, cudaStream_t st);
void launch_cv8uc3_to_gray(const uchar3* src, float* dst, Geom g, cudaStream_t st);
void launch_cv8u_tight_to_gray2(const uint8_t* s0, const uint8_t* s1, float* d0, float* d1, Geom g, cudaStream_t st);
void launch_pack_tight(const float* src, float* dst, int comps, Geom g, cudaStream_t st);
void launch_pack_tight_half(const void* src, float* dst, Geom g, cudaStream_t st);
// downscale.cu:10-30 (float) / :98-122 (float2): mean of 4 taps at +-1/4 coarse px
void launch_downscale(cudaTextureObject_t fine, int comps, float* out, Geom coarse, cudaStream_t st);
// downscale.cu:52-73 point-sampled (mask pyramid)
// 2 x 2 box to the next coarser level with the values multiplied by `scale` (warm start)
void launch_downscale_scaled(cudaTextureObject_t fine, float* out, float scale, Geom g, cudaStream_t st);
void launch_downscale_nearest(cudaTextureObject_t fine, float* out, Geom coarse, cudaStream_t st);
// warpImage.cu:9-23
void launch_warp_image(cudaTextureObject_t src, const float2* warpUV, float* out, Geom g, cudaStream_t st);
// warpImage.cu:96-111
void launch_find_warping_vector(cudaTextureObject_t tv, const float2* warpUV, float2* tv2, Geom g,
                                cudaStream_t st);
// warpImage.cu:136-150
void launch_optical_flow_vector(const float* u, const float2* tv2, float2* warpUV, Geom g, cudaStream_t st);
// computeDerivatives.cu:89-129
void launch_derivatives_fisheye(cudaTextureObject_t i0, cudaTextureObject_t i1w, const float2* tv, float* Iu,
                                float* Iz, Geom g, cudaStream_t st);
// calcTensor.cu:99-128 (mask == nullptr) and :245-273
void launch_gaussian(cudaTextureObject_t in, const float* mask, float* out, Geom g, cudaStream_t st);
// calcTensor.cu:8-73 / :155-219; columns >= xmax are not computed
// cuda_math: tensor weight from CUDA's expf / powf (1, as the reference) or the portable
// construction of tgv_math.cuh (0)
void launch_calc_tensor(cudaTextureObject_t gray, const float* mask, float beta, float gamma, float* a, float* b,
                        float* c, Geom g, int xmax, int cuda_math, cudaStream_t st);
// preconditioning.cu:3-22 / :41-60
void launch_solve_eta(const float* mask, float alpha0, float alpha1, const float* a, const float* b,
                      const float* c, float* etau, float* etav1, float* etav2, Geom g, cudaStream_t st);

// Inner primal-dual iteration, one kernel per reference kernel.  mask == nullptr
// selects the plain form with the hard-coded circle.
struct DualArgs {
  const float* mask;
  const float* u_;
  const float2* v_;
  const float *a, *b, *c;
  float2* p;
  float4* q;
  float alpha0, alpha1, sigma, eta_p, eta_q;
  float sp, sq;  // alpha1 * sigma / eta_p and alpha0 * sigma / eta_q (set by the launcher)
};
// updateDualVariables.cu:4-101 / :122-237
void launch_update_dual(const DualArgs& A, Geom g, cudaStream_t st);
// thresholdingL1.cu:104-115 / :234-244
void launch_solve_tp(const float* mask, const float* a, const float* b, const float* c, const float2* p,
                     float2* Tp, Geom g, cudaStream_t st);
struct ThreshArgs {
  const float* mask;
  const float2* Tp;
  const float *u_, *Iu, *Iz, *etau, *u;
  float* us;
  float lambda, tau;
};
// thresholdingL1.cu:3-86 / :128-216
void launch_thresholding(const ThreshArgs& A, Geom g, cudaStream_t st);
struct PrimalArgs {
  const float* mask;
  const float* u_;
  const float2* v_;
  const float2* p;
  const float4* q;
  const float *a, *b, *c, *etav1, *etav2, *u;
  float2* v;
  float* u_s;
  float2* v_s;
  float tau, alpha0, alpha1, mu;
};
// updatePrimalVariables.cu:3-113 / :139-245
void launch_update_primal(const PrimalArgs& A, Geom g, cudaStream_t st);
// medianFilter.cu:264-319
void launch_median5(const float* in, float* out, Geom g, cudaStream_t st);
// stereotgv.cu:484-493: Subtract, LimitRange, Add, Clone, ComputeOpticalFlowVector,
// AddFloat2 applied in sequence (point-wise, all pixels of the level)
void launch_warp_epilogue(float* u, const float* u_last, float* du, float* u_, const float2* tv2, float2* dwarpUV,
                          float2* warpUV, float limitRange, Geom g, cudaStream_t st);
// copyClone.cu:3-12 / :21-30
void launch_clone(float* dst, const float* src, Geom g, cudaStream_t st);
void launch_clone2(float2* dst, const float2* src, Geom g, cudaStream_t st);
// upscale.cu:8-21 / :46-61
void launch_upscale(cudaTextureObject_t coarse, int comps, float* out, float scale, Geom fine, cudaStream_t st);
// conversion.cu:3-69
void launch_convert_kb(const float2* disparity, float focalx, float focaly, float cx, float cy, float d1, float d2,
                       float d3, float d4, float t1, float t2, float t3, float3* X, float* depth, Geom g,
                       cudaStream_t st);
// flowToHsv.cu:4-110
void launch_flow_to_hsv(const float2* uv, float3* rgb, float flowscale, Geom g, cudaStream_t st);

// Pitched <-> tight copies of W x H x comps float images (device to device).
void launch_pack(const float* src, int comps, float* dst, Geom g, cudaStream_t st);

}  // namespace vfs
