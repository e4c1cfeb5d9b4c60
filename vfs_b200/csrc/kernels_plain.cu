// Per-operation kernels of the drop-in solve path (see kernels.cuh).
//
// Addressing follows the reference: images are row-major and pitched by the level's
// stride s (elements); float2 / float4 fields are arrays of structures with the same
// pitch.  A kernel touches exactly the pixels the reference kernel touches: the
// unmasked kernels all ix < w, iy < h; the masked kernels the pixels whose mask is
// non-zero.
#include "common.cuh"
#include "kernels.cuh"
#include "tgv_math.cuh"
#include "tgv_pixel.cuh"

namespace vfs {

__device__ __forceinline__ bool pixel(int& ix, int& iy, int w, int h) {
  ix = blockIdx.x * blockDim.x + threadIdx.x;
  iy = blockIdx.y * blockDim.y + threadIdx.y;
  return ix < w && iy < h;
}

// A flat index before the start of a buffer reads 0.  Only the masked edge rules
// can form one (a mask that is on in row 0 or column 0 with its right / lower
// neighbour off); the reference reads out of bounds there.
__device__ __forceinline__ float rd1(const float* b, long long k) { return k < 0 ? 0.0f : b[k]; }
__device__ __forceinline__ float2 rd2(const float2* b, long long k) { return k < 0 ? make_float2(0.f, 0.f) : b[k]; }

// ---------------------------------------------------------------------------
__global__ void k_cv8u_to_gray(const uint8_t* src, float* dst, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int idx = ix + g.s * iy;
  dst[idx] = (float)src[idx] / 256.0f;
}

// Both images of a pair from tight (row length w) u8 buffers into the pitched float planes,
// with the same u8 / 256 conversion as k_cv8u_to_gray: a host upload is then one contiguous
// copy per image.
__global__ void k_cv8u_tight_to_gray2(const uint8_t* src0, const uint8_t* src1, float* dst0, float* dst1, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  const int si = ix + g.w * iy, di = ix + g.s * iy;
  dst0[di] = (float)src0[si] / 256.0f;
  dst1[di] = (float)src1[si] / 256.0f;
}

// A pitched plane of `comps` floats per pixel into a tight buffer (one contiguous download).
__global__ void k_pack_tight(const float* src, float* dst, int comps, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  const long long si = ((long long)ix + (long long)g.s * iy) * comps, di = ((long long)ix + (long long)g.w * iy) * comps;
  for (int c = 0; c < comps; c++) dst[di + c] = src[si + c];
}

// A pitched half plane (the FP16 form's warped image) widened to float into a tight buffer.
__global__ void k_pack_tight_half(const __half* src, float* dst, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  dst[(long long)ix + (long long)g.w * iy] = __half2float(src[(long long)ix + (long long)g.s * iy]);
}

__global__ void k_cv8uc3_to_gray(const uchar3* src, float* dst, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int idx = ix + g.s * iy;
  uchar3 px = src[idx];
  float v = ((float)px.x + (float)px.y + (float)px.z) / 3;
  dst[idx] = v / 256.0f;
}

// Warm start: the previous frame's disparity one level coarser, the same 2 x 2 box as
// k_downscale1, with the values scaled to the coarser level's pixels (x scale).
__global__ void k_downscale_scaled(cudaTextureObject_t fine, float* out, float scale, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  float dx = 1.0f / (float)g.w, dy = 1.0f / (float)g.h;
  float x = ((float)ix + 0.5f) * dx, y = ((float)iy + 0.5f) * dy;
  float t1 = tex2D<float>(fine, x - dx * 0.25f, y);
  float t2 = tex2D<float>(fine, x + dx * 0.25f, y);
  float t3 = tex2D<float>(fine, x, y - dy * 0.25f);
  float t4 = tex2D<float>(fine, x, y + dy * 0.25f);
  out[ix + iy * g.s] = 0.25f * (t1 + t2 + t3 + t4) * scale;
}

__global__ void k_downscale1(cudaTextureObject_t fine, float* out, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  float dx = 1.0f / (float)g.w, dy = 1.0f / (float)g.h;
  float x = ((float)ix + 0.5f) * dx, y = ((float)iy + 0.5f) * dy;
  float t1 = tex2D<float>(fine, x - dx * 0.25f, y);
  float t2 = tex2D<float>(fine, x + dx * 0.25f, y);
  float t3 = tex2D<float>(fine, x, y - dy * 0.25f);
  float t4 = tex2D<float>(fine, x, y + dy * 0.25f);
  out[ix + iy * g.s] = 0.25f * (t1 + t2 + t3 + t4);
}

__global__ void k_downscale2(cudaTextureObject_t fine, float2* out, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  float dx = 1.0f / (float)g.w, dy = 1.0f / (float)g.h;
  float x = ((float)ix + 0.5f) * dx, y = ((float)iy + 0.5f) * dy;
  float2 v00 = tex2D<float2>(fine, x - dx * 0.25f, y);
  float2 v01 = tex2D<float2>(fine, x + dx * 0.25f, y);
  float2 v10 = tex2D<float2>(fine, x, y - dy * 0.25f);
  float2 v11 = tex2D<float2>(fine, x, y + dy * 0.25f);
  out[ix + iy * g.s] = make_float2(0.25f * (v00.x + v01.x + v10.x + v11.x), 0.25f * (v00.y + v01.y + v10.y + v11.y));
}

__global__ void k_downscale_nearest(cudaTextureObject_t fine, float* out, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  float dx = 1.0f / (float)g.w, dy = 1.0f / (float)g.h;
  float x = ((float)ix + 0.5f) * dx, y = ((float)iy + 0.5f) * dy;
  out[ix + iy * g.s] = tex2D<float>(fine, x, y);
}

__global__ void k_warp_image(cudaTextureObject_t src, const float2* __restrict__ warpUV, float* out, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  float2 wv = warpUV[pos];
  float x = ((float)ix + wv.x + 0.5f) / (float)g.w;
  float y = ((float)iy + wv.y + 0.5f) / (float)g.h;
  out[pos] = tex2D<float>(src, x, y);
}

__global__ void k_find_warping_vector(cudaTextureObject_t tv, const float2* __restrict__ warpUV, float2* tv2,
                                      Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  float2 wv = warpUV[pos];
  float x = ((float)ix + wv.x + 0.5f) / (float)g.w;
  float y = ((float)iy + wv.y + 0.5f) / (float)g.h;
  tv2[pos] = tex2D<float2>(tv, x, y);
}

__global__ void k_optical_flow_vector(const float* __restrict__ u, const float2* __restrict__ tv2, float2* warpUV,
                                      Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  float us = u[pos];
  float2 t = tv2[pos];
  warpUV[pos] = make_float2(us * t.x, us * t.y);
}

__global__ void k_derivatives_fisheye(cudaTextureObject_t I0, cudaTextureObject_t I1, const float2* __restrict__ vec,
                                      float* Iw, float* Iz, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  float2 vv = vec[pos];
  float r = sqrtf(vv.x * vv.x + vv.y * vv.y);
  float dx = (vv.x / r) / (float)g.w;
  float dy = (vv.y / r) / (float)g.h;
  float x = ((float)ix + 0.5f) / (float)g.w;
  float y = ((float)iy + 0.5f) / (float)g.h;
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
  Iw[pos] = (t0 + t1) * 0.5f;
  Iz[pos] = tex2D<float>(I1, x, y) - tex2D<float>(I0, x, y);
}

__global__ void k_gaussian(cudaTextureObject_t in, const float* __restrict__ mask, float* out, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  if (mask && mask[pos] == 0.0f) return;
  float dx = 1.0f / (float)g.w, dy = 1.0f / (float)g.h;
  float x = ((float)ix + 0.5f) * dx, y = ((float)iy + 0.5f) * dy;
  float t0 = (1 / 4.0f) * tex2D<float>(in, x, y);
  t0 += (1 / 16.0f) * tex2D<float>(in, x - 1.0f * dx, y - 1.0f * dy);
  t0 += (1 / 16.0f) * tex2D<float>(in, x - 1.0f * dx, y + 1.0f * dy);
  t0 += (1 / 16.0f) * tex2D<float>(in, x + 1.0f * dx, y - 1.0f * dy);
  t0 += (1 / 16.0f) * tex2D<float>(in, x + 1.0f * dx, y + 1.0f * dy);
  t0 += (1 / 8.0f) * tex2D<float>(in, x - 1.0f * dx, y);
  t0 += (1 / 8.0f) * tex2D<float>(in, x + 1.0f * dx, y);
  t0 += (1 / 8.0f) * tex2D<float>(in, x, y - 1.0f * dy);
  t0 += (1 / 8.0f) * tex2D<float>(in, x, y + 1.0f * dy);
  out[pos] = t0;
}

__global__ void k_calc_tensor(cudaTextureObject_t gray, const float* __restrict__ mask, float beta, float gamma,
                              float* A, float* B, float* C, Geom g, int xmax, int cuda_math) {
  int ix, iy;
  if (!pixel(ix, iy, xmax, g.h)) return;
  int pos = ix + iy * g.s;
  if (mask && mask[pos] == 0.0f) return;
  float dx = 1.0f / (float)g.w, dy = 1.0f / (float)g.h;
  float x = ((float)ix + 0.5f) * dx, y = ((float)iy + 0.5f) * dy;
  // calcTensor.cu:27-39: the second assignment of t0 replaces the first.
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
  float wt = tensor_weight(abs_img, beta, gamma, cuda_math);
  if (!(wt > 1e-8f)) wt = 1e-8f;
  A[pos] = wt * nx * nx + ntx * ntx;
  C[pos] = wt * nx * ny + ntx * nty;
  B[pos] = wt * ny * ny + nty * nty;
}

__global__ void k_solve_eta(const float* __restrict__ mask, float alpha0, float alpha1, const float* __restrict__ A,
                            const float* __restrict__ B, const float* __restrict__ C, float* etau, float* etav1,
                            float* etav2, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  if (mask && mask[pos] == 0.0f) return;
  float a = A[pos], b = B[pos], c = C[pos];
  etau[pos] = etau_math(a, b, c, alpha1);
  etav1[pos] = etav1_math(b, c, alpha0, alpha1);
  etav2[pos] = etav2_math(a, c, alpha0, alpha1);
}

__global__ void k_update_dual(DualArgs A, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  long long pos = ix + (long long)iy * g.s;
  long long right = pos + 1, down = pos + g.s, left = pos - 1, up = pos - g.s;
  bool useRight, useDown;
  if (A.mask) {
    if (A.mask[pos] == 0.0f) return;
    float maskRight = (ix + 1 >= g.w) ? 0.0f : A.mask[right];
    float maskDown = (iy + 1 >= g.h) ? 0.0f : A.mask[down];
    useRight = maskRight != 0.0f;
    useDown = maskDown != 0.0f;
  } else {
    if (outside_circle(ix, iy, g.w, g.h)) {
      A.p[pos] = make_float2(0.f, 0.f);
      A.q[pos] = make_float4(0.f, 0.f, 0.f, 0.f);
      return;
    }
    useRight = (ix + 1) < g.w;
    useDown = (iy + 1) < g.h;
  }
  float u_pos = A.u_[pos];
  float2 vp = A.v_[pos];
  float u_xn = useRight ? A.u_[right] : rd1(A.u_, left);
  float u_yn = useDown ? A.u_[down] : rd1(A.u_, up);
  float2 v_xn = useRight ? A.v_[right] : rd2(A.v_, left);
  float2 v_yn = useDown ? A.v_[down] : rd2(A.v_, up);
  float2 pp = A.p[pos];
  float4 qq = A.q[pos];
  dual_math(useRight, useDown, u_pos, u_xn, u_yn, vp, v_xn, v_yn, A.a[pos], A.b[pos], A.c[pos], A.sp, A.sq, pp, qq);
  A.p[pos] = pp;
  A.q[pos] = qq;
}

__global__ void k_solve_tp(const float* __restrict__ mask, const float* __restrict__ A, const float* __restrict__ B,
                           const float* __restrict__ C, const float2* __restrict__ p, float2* Tp, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  if (mask && mask[pos] == 0.0f) return;
  Tp[pos] = tp_math(A[pos], B[pos], C[pos], p[pos]);
}

__global__ void k_thresholding(ThreshArgs A, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  long long pos = ix + (long long)iy * g.s;
  long long left = pos - 1, up = pos - g.s;
  float dxm, dym;
  if (A.mask) {
    if (A.mask[pos] == 0.0f) return;
    float mR = (ix + 1 >= g.w) ? 0.0f : A.mask[pos + 1];
    float mL = (ix - 1 < 0) ? 0.0f : A.mask[left];
    float mD = (iy + 1 >= g.h) ? 0.0f : A.mask[pos + g.s];
    float mU = (iy - 1 < 0) ? 0.0f : A.mask[up];
    if (mL != 0.0f && mR != 0.0f) dxm = A.Tp[pos].x - A.Tp[left].x;
    else if (mR == 0.0f) dxm = -rd2(A.Tp, left).x;
    else dxm = A.Tp[pos].x;
    if (mU != 0.0f && mD != 0.0f) dym = A.Tp[pos].y - A.Tp[up].y;
    else if (mD == 0.0f) dym = -rd2(A.Tp, up).y;
    else dym = A.Tp[pos].y;
  } else {
    if (outside_circle(ix, iy, g.w, g.h)) {
      A.us[pos] = 0.0f;
      return;
    }
    if ((ix - 1) >= 0) dxm = A.Tp[pos].x - A.Tp[left].x;
    else if (ix == g.w - 1) dxm = -rd2(A.Tp, left).x;
    else dxm = A.Tp[pos].x;
    if ((iy - 1) >= 0) dym = A.Tp[pos].y - A.Tp[up].y;
    else if (iy == g.h - 1) dym = -rd2(A.Tp, up).y;
    else dym = A.Tp[pos].y;
  }
  A.us[pos] = threshold_math(dxm, dym, A.etau[pos], A.tau, A.u_[pos], A.u[pos], A.Iu[pos], A.Iz[pos], A.lambda);
}

__global__ void k_update_primal(PrimalArgs A, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  long long pos = ix + (long long)iy * g.s;
  long long left = pos - 1, up = pos - g.s;
  bool zR, zD, hasL, hasU;
  if (A.mask) {
    if (A.mask[pos] == 0.0f) return;
    float mR = (ix + 1 >= g.w) ? 0.0f : A.mask[pos + 1];
    float mL = (ix - 1 < 0) ? 0.0f : A.mask[left];
    float mD = (iy + 1 >= g.h) ? 0.0f : A.mask[pos + g.s];
    float mU = (iy - 1 < 0) ? 0.0f : A.mask[up];
    zR = mR == 0.0f;
    zD = mD == 0.0f;
    hasL = mL != 0.0f;
    hasU = mU != 0.0f;
  } else {
    if (outside_circle(ix, iy, g.w, g.h)) {
      A.u_s[pos] = 0.0f;
      A.v_s[pos] = make_float2(0.f, 0.f);
      return;
    }
    zR = ix == g.w - 1;
    zD = iy == g.h - 1;
    hasL = (ix - 1) >= 0;
    hasU = (iy - 1) >= 0;
  }
  float4 qc = A.q[pos];
  if (zR) qc.x = qc.w = 0.0f;
  if (zD) qc.y = qc.z = 0.0f;
  float4 ql = hasL ? A.q[left] : make_float4(0.f, 0.f, 0.f, 0.f);
  float4 qu = hasU ? A.q[up] : make_float4(0.f, 0.f, 0.f, 0.f);
  float us_;
  float2 vs, vo;
  primal_math(qc, ql, qu, A.p[pos], A.a[pos], A.b[pos], A.c[pos], A.etav1[pos], A.etav2[pos], A.tau, A.alpha0,
              A.alpha1, A.mu, A.v_[pos], A.u[pos], A.u_[pos], us_, vs, vo);
  A.v[pos] = vo;
  A.u_s[pos] = us_;
  A.v_s[pos] = vs;
}

// medianFilter.cu:264-319
__global__ void k_median5(const float* __restrict__ in, float* out, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  out[ix + iy * g.s] = median5_at(in, ix, iy, g.w, g.h, g.s);
}

__global__ void k_warp_epilogue(float* u, const float* __restrict__ u_last, float* du, float* u_,
                                const float2* __restrict__ tv2, float2* dwarpUV, float2* warpUV, float limitRange,
                                Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  float ul = u_last[pos];
  float d = u[pos] - ul;             // scalar.cu:130-141
  d = d > limitRange ? limitRange : d;  // limitRange.cu:4-24
  du[pos] = d;
  float un = ul + d;  // scalar.cu:78-89
  u[pos] = un;
  u_[pos] = un;  // copyClone.cu:3-12
  float2 t = tv2[pos];
  float2 dw = make_float2(d * t.x, d * t.y);  // warpImage.cu:136-150
  dwarpUV[pos] = dw;
  float2 wv = warpUV[pos];
  warpUV[pos] = make_float2(wv.x + dw.x, wv.y + dw.y);  // scalar.cu:103-115
}

__global__ void k_clone(float* dst, const float* __restrict__ src, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  dst[pos] = src[pos];
}
__global__ void k_clone2(float2* dst, const float2* __restrict__ src, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  dst[pos] = src[pos];
}

__global__ void k_upscale1(cudaTextureObject_t coarse, float* out, float scale, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  float x = ((float)ix + 0.5f) / (float)g.w;
  float y = ((float)iy + 0.5f) / (float)g.h;
  out[ix + iy * g.s] = tex2D<float>(coarse, x, y) * scale;
}
__global__ void k_upscale2(cudaTextureObject_t coarse, float2* out, float scale, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  float x = ((float)ix + 0.5f) / (float)g.w;
  float y = ((float)iy + 0.5f) / (float)g.h;
  float2 v = tex2D<float2>(coarse, x, y);
  out[ix + iy * g.s] = make_float2(v.x * scale, v.y * scale);
}

// conversion.cu:3-69: Kannala-Brandt unprojection by 5 Newton steps and
// triangulation along x.  Arguments keep the reference's order, in which the
// pixel offset is divided by `cx` and shifted by `focalx` (conversion.cu:19-28).
__device__ float kb_theta(float ru, float d1, float d2, float d3, float d4) {
  float th = 0.0f;
  for (int it = 0; it < 5; it++) {
    float thd = th + d1 * powf(th, 3.0f) + d2 * powf(th, 5.0f) + d3 * powf(th, 7.0f) + d4 * powf(th, 9.0f);
    float dthd = 1.0f + 3.0f * d1 * powf(th, 2.0f) + 5.0f * d2 * powf(th, 4.0f) + 7.0f * d3 * powf(th, 6.0f) +
                 9.0f * d4 * powf(th, 8.0f);
    float f = ru - thd;
    float fp = -dthd;
    th = th - f / fp;
  }
  return th;
}
__global__ void k_convert_kb(const float2* __restrict__ disp, float focalx, float focaly, float cx, float cy,
                             float d1, float d2, float d3, float d4, float t1, float t2, float t3, float3* X,
                             float* depth, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  float u0 = (float)ix, v0 = (float)iy;
  float xp0 = (u0 - focalx) / cx, yp0 = (v0 - focaly) / cy;
  float2 d = disp[pos];
  float u1 = u0 + d.x, v1 = v0 + d.y;
  float xp1 = (u1 - focalx) / cx, yp1 = (v1 - focaly) / cy;
  float ru0 = sqrtf(xp0 * xp0 + yp0 * yp0);
  float th0 = kb_theta(ru0, d1, d2, d3, d4);
  float x0o = tanf(th0) * xp0 / ru0, y0o = tanf(th0) * yp0 / ru0;
  float ru1 = sqrtf(xp1 * xp1 + yp1 * yp1);
  float th1 = kb_theta(ru1, d1, d2, d3, d4);
  float x1o = tanf(th1) * xp1 / ru1, y1o = tanf(th1) * yp1 / ru1;
  (void)y1o;
  (void)t2;
  float Z = (t1 - x1o * t3) / (x1o - x0o);
  float3 Xv = make_float3(x0o * Z, y0o * Z, Z);
  X[pos] = Xv;
  depth[pos] = sqrtf(Xv.x * Xv.x + Xv.y * Xv.y + Xv.z * Xv.z);
}

// flowToHsv.cu:4-110: Middlebury colour wheel (segments RY 15, YG 6, GC 4, CB 11,
// BM 13, MR 6), indexed from 1 as in the reference.
__device__ float3 wheel_colour(int k) {
  // k in 1..55 (the reference's 1-based index); returns RGB in 0..255
  int i = k - 1;
  if (i < 0) i = 0;
  if (i > 54) i = 54;
  const int RY = 15, YG = 6, GC = 4, CB = 11, BM = 13;
  if (i < RY) return make_float3(255.f, floorf(255.f * i / RY), 0.f);
  i -= RY;
  if (i < YG) return make_float3(255.f - floorf(255.f * i / YG), 255.f, 0.f);
  i -= YG;
  if (i < GC) return make_float3(0.f, 255.f, floorf(255.f * i / GC));
  i -= GC;
  if (i < CB) return make_float3(0.f, 255.f - floorf(255.f * i / CB), 255.f);
  i -= CB;
  if (i < BM) return make_float3(floorf(255.f * i / BM), 0.f, 255.f);
  i -= BM;
  return make_float3(255.f, 0.f, 255.f - floorf(255.f * i / 6));
}
__global__ void k_flow_to_hsv(const float2* __restrict__ uv, float3* rgb, float flowscale, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  int pos = ix + iy * g.s;
  float du = uv[pos].x / flowscale, dv = uv[pos].y / flowscale;
  const int ncols = 55;
  float rad = sqrtf(du * du + dv * dv);
  float a = atan2f(-dv, -du) / 3.14159f;
  float fk = (a + 1) / 2 * ((float)ncols - 1) + 1;
  int k0 = (int)floorf(fk);
  int k1 = k0 + 1;
  if (k1 == ncols + 1) k1 = 1;
  float f = fk - (float)k0;
  // the reference's wheel arrays are 0-based while k0/k1 are 1-based
  float3 c0 = wheel_colour(k0 + 1), c1 = wheel_colour(k1 + 1);
  float colR = (1 - f) * (c0.x / 255.0f) + f * (c1.x / 255.0f);
  float colG = (1 - f) * (c0.y / 255.0f) + f * (c1.y / 255.0f);
  float colB = (1 - f) * (c0.z / 255.0f) + f * (c1.z / 255.0f);
  if (rad <= 1) {
    colR = 1 - rad * (1 - colR);
    colG = 1 - rad * (1 - colG);
    colB = 1 - rad * (1 - colB);
  } else {
    colR = colR * 0.75f;
    colG = colG * 0.75f;
    colB = colB * 0.75f;
  }
  rgb[pos] = make_float3(colB, colG, colR);
}

__global__ void k_pack(const float* __restrict__ src, int comps, float* dst, Geom g) {
  int ix, iy;
  if (!pixel(ix, iy, g.w, g.h)) return;
  for (int k = 0; k < comps; k++) dst[((size_t)iy * g.w + ix) * comps + k] = src[((size_t)iy * g.s + ix) * comps + k];
}

// ---------------------------------------------------------------------------
#define L2D(g) grid2d((g).w, (g).h), block2d(), 0, st
void launch_cv8u_to_gray(const uint8_t* src, float* dst, Geom g, cudaStream_t st) {
  k_cv8u_to_gray<<<L2D(g)>>>(src, dst, g);
  VFS_LAUNCH_CHECK();
}
void launch_cv8u_tight_to_gray2(const uint8_t* s0, const uint8_t* s1, float* d0, float* d1, Geom g, cudaStream_t st) {
  k_cv8u_tight_to_gray2<<<L2D(g)>>>(s0, s1, d0, d1, g);
  VFS_LAUNCH_CHECK();
}
void launch_pack_tight(const float* src, float* dst, int comps, Geom g, cudaStream_t st) {
  k_pack_tight<<<L2D(g)>>>(src, dst, comps, g);
  VFS_LAUNCH_CHECK();
}
void launch_pack_tight_half(const void* src, float* dst, Geom g, cudaStream_t st) {
  k_pack_tight_half<<<L2D(g)>>>((const __half*)src, dst, g);
  VFS_LAUNCH_CHECK();
}
void launch_cv8uc3_to_gray(const uchar3* src, float* dst, Geom g, cudaStream_t st) {
  k_cv8uc3_to_gray<<<L2D(g)>>>(src, dst, g);
  VFS_LAUNCH_CHECK();
}
void launch_downscale(cudaTextureObject_t fine, int comps, float* out, Geom g, cudaStream_t st) {
  if (comps == 2) k_downscale2<<<L2D(g)>>>(fine, (float2*)out, g);
  else k_downscale1<<<L2D(g)>>>(fine, out, g);
  VFS_LAUNCH_CHECK();
}
void launch_downscale_scaled(cudaTextureObject_t fine, float* out, float scale, Geom g, cudaStream_t st) {
  k_downscale_scaled<<<L2D(g)>>>(fine, out, scale, g);
  VFS_LAUNCH_CHECK();
}
void launch_downscale_nearest(cudaTextureObject_t fine, float* out, Geom g, cudaStream_t st) {
  k_downscale_nearest<<<L2D(g)>>>(fine, out, g);
  VFS_LAUNCH_CHECK();
}
void launch_warp_image(cudaTextureObject_t src, const float2* warpUV, float* out, Geom g, cudaStream_t st) {
  k_warp_image<<<L2D(g)>>>(src, warpUV, out, g);
  VFS_LAUNCH_CHECK();
}
void launch_find_warping_vector(cudaTextureObject_t tv, const float2* warpUV, float2* tv2, Geom g, cudaStream_t st) {
  k_find_warping_vector<<<L2D(g)>>>(tv, warpUV, tv2, g);
  VFS_LAUNCH_CHECK();
}
void launch_optical_flow_vector(const float* u, const float2* tv2, float2* warpUV, Geom g, cudaStream_t st) {
  k_optical_flow_vector<<<L2D(g)>>>(u, tv2, warpUV, g);
  VFS_LAUNCH_CHECK();
}
void launch_derivatives_fisheye(cudaTextureObject_t i0, cudaTextureObject_t i1w, const float2* tv, float* Iu,
                                float* Iz, Geom g, cudaStream_t st) {
  k_derivatives_fisheye<<<L2D(g)>>>(i0, i1w, tv, Iu, Iz, g);
  VFS_LAUNCH_CHECK();
}
void launch_gaussian(cudaTextureObject_t in, const float* mask, float* out, Geom g, cudaStream_t st) {
  k_gaussian<<<L2D(g)>>>(in, mask, out, g);
  VFS_LAUNCH_CHECK();
}
void launch_calc_tensor(cudaTextureObject_t gray, const float* mask, float beta, float gamma, float* a, float* b,
                        float* c, Geom g, int xmax, int cuda_math, cudaStream_t st) {
  if (xmax <= 0) return;
  k_calc_tensor<<<grid2d(xmax, g.h), block2d(), 0, st>>>(gray, mask, beta, gamma, a, b, c, g, xmax, cuda_math);
  VFS_LAUNCH_CHECK();
}
void launch_solve_eta(const float* mask, float alpha0, float alpha1, const float* a, const float* b, const float* c,
                      float* etau, float* etav1, float* etav2, Geom g, cudaStream_t st) {
  k_solve_eta<<<L2D(g)>>>(mask, alpha0, alpha1, a, b, c, etau, etav1, etav2, g);
  VFS_LAUNCH_CHECK();
}
void launch_update_dual(const DualArgs& A0, Geom g, cudaStream_t st) {
  DualArgs A = A0;
  A.sp = A.alpha1 * A.sigma / A.eta_p;  // updateDualVariables.cu:174-176, uniform per launch
  A.sq = A.alpha0 * A.sigma / A.eta_q;  // updateDualVariables.cu:217
  k_update_dual<<<L2D(g)>>>(A, g);
  VFS_LAUNCH_CHECK();
}
void launch_solve_tp(const float* mask, const float* a, const float* b, const float* c, const float2* p, float2* Tp,
                     Geom g, cudaStream_t st) {
  k_solve_tp<<<L2D(g)>>>(mask, a, b, c, p, Tp, g);
  VFS_LAUNCH_CHECK();
}
void launch_thresholding(const ThreshArgs& A, Geom g, cudaStream_t st) {
  k_thresholding<<<L2D(g)>>>(A, g);
  VFS_LAUNCH_CHECK();
}
void launch_update_primal(const PrimalArgs& A, Geom g, cudaStream_t st) {
  k_update_primal<<<L2D(g)>>>(A, g);
  VFS_LAUNCH_CHECK();
}
void launch_median5(const float* in, float* out, Geom g, cudaStream_t st) {
  k_median5<<<L2D(g)>>>(in, out, g);
  VFS_LAUNCH_CHECK();
}
void launch_warp_epilogue(float* u, const float* u_last, float* du, float* u_, const float2* tv2, float2* dwarpUV,
                          float2* warpUV, float limitRange, Geom g, cudaStream_t st) {
  k_warp_epilogue<<<L2D(g)>>>(u, u_last, du, u_, tv2, dwarpUV, warpUV, limitRange, g);
  VFS_LAUNCH_CHECK();
}
void launch_clone(float* dst, const float* src, Geom g, cudaStream_t st) {
  k_clone<<<L2D(g)>>>(dst, src, g);
  VFS_LAUNCH_CHECK();
}
void launch_clone2(float2* dst, const float2* src, Geom g, cudaStream_t st) {
  k_clone2<<<L2D(g)>>>(dst, src, g);
  VFS_LAUNCH_CHECK();
}
void launch_upscale(cudaTextureObject_t coarse, int comps, float* out, float scale, Geom g, cudaStream_t st) {
  if (comps == 2) k_upscale2<<<L2D(g)>>>(coarse, (float2*)out, scale, g);
  else k_upscale1<<<L2D(g)>>>(coarse, out, scale, g);
  VFS_LAUNCH_CHECK();
}
void launch_convert_kb(const float2* disparity, float focalx, float focaly, float cx, float cy, float d1, float d2,
                       float d3, float d4, float t1, float t2, float t3, float3* X, float* depth, Geom g,
                       cudaStream_t st) {
  k_convert_kb<<<L2D(g)>>>(disparity, focalx, focaly, cx, cy, d1, d2, d3, d4, t1, t2, t3, X, depth, g);
  VFS_LAUNCH_CHECK();
}
void launch_flow_to_hsv(const float2* uv, float3* rgb, float flowscale, Geom g, cudaStream_t st) {
  k_flow_to_hsv<<<L2D(g)>>>(uv, rgb, flowscale, g);
  VFS_LAUNCH_CHECK();
}
void launch_pack(const float* src, int comps, float* dst, Geom g, cudaStream_t st) {
  k_pack<<<L2D(g)>>>(src, comps, dst, g);
  VFS_LAUNCH_CHECK();
}

}  // namespace vfs
