// Deterministic float exp / log / pow for the diffusion-tensor weight
// w = exp(-beta * |grad I|^gamma) (calcTensor.cu:60-64).
//
// Built only from IEEE-754 operations that are correctly rounded on every
// platform (+, -, *, /, fmaf, frexpf, ldexpf by exact powers of two), so the
// same input gives the same bits on the GPU and in a host restatement.
//   exp: Cody-Waite reduction x = k ln2 + r (ln2 split into an exactly
//        representable high part and the remainder), |r| <= ln2/2, then the
//        Taylor series of e^r to degree 7 in Horner form, scaled by 2^k.
//   log: a = m 2^e with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s),
//        s = (m-1)/(m+1), by the odd power series of atanh to s^11.
// Accuracy is within a few ulp over the range the tensor uses.
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define TGV_HD __host__ __device__ __forceinline__
#else
#define TGV_HD inline
#endif

namespace vfs {

TGV_HD float tgv_fma(float a, float b, float c) {
#ifdef __CUDA_ARCH__
  return __fmaf_rn(a, b, c);
#else
  return fmaf(a, b, c);
#endif
}

constexpr float kLn2Hi = 0.693145751953125f;    // ln 2 rounded to 16 significant bits (exact)
constexpr float kLn2Lo = 1.4286068203e-06f;     // ln 2 - kLn2Hi
constexpr float kInvLn2 = 1.44269504088896f;    // 1 / ln 2

TGV_HD float tgv_exp(float x) {
  if (x != x) return x;
  if (x < -87.0f) return 0.0f;      // below the normal range: the tensor clamps at 1e-8 anyway
  if (x > 88.0f) return INFINITY;
  float k = rintf(x * kInvLn2);
  float r = tgv_fma(-k, kLn2Hi, x);
  r = tgv_fma(-k, kLn2Lo, r);
  float p = 1.0f / 5040.0f;
  p = tgv_fma(p, r, 1.0f / 720.0f);
  p = tgv_fma(p, r, 1.0f / 120.0f);
  p = tgv_fma(p, r, 1.0f / 24.0f);
  p = tgv_fma(p, r, 1.0f / 6.0f);
  p = tgv_fma(p, r, 0.5f);
  p = tgv_fma(p, r, 1.0f);
  p = tgv_fma(p, r, 1.0f);
  return ldexpf(p, (int)k);
}

// natural log of a > 0 (finite)
TGV_HD float tgv_log(float a) {
  int e;
  float m = frexpf(a, &e);  // a = m 2^e, m in [0.5, 1)
  if (m < 0.70710678f) {
    m = m * 2.0f;
    e -= 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float q = 1.0f / 11.0f;
  q = tgv_fma(q, s2, 1.0f / 9.0f);
  q = tgv_fma(q, s2, 1.0f / 7.0f);
  q = tgv_fma(q, s2, 1.0f / 5.0f);
  q = tgv_fma(q, s2, 1.0f / 3.0f);
  q = tgv_fma(q, s2, 1.0f);
  float lnm = 2.0f * s * q;
  float fe = (float)e;
  return tgv_fma(fe, kLn2Hi, tgv_fma(fe, kLn2Lo, lnm));
}

// a^g for a >= 0, g > 0 (the tensor's |grad I|^gamma)
TGV_HD float tgv_pow(float a, float g) {
  if (a == 0.0f) return 0.0f;
  if (!(a > 0.0f) || a == INFINITY) return a != a ? a : (a == INFINITY ? INFINITY : NAN);
  float l = tgv_log(a);
  float y = g * l;
  float err = tgv_fma(g, l, -y);  // rounding error of the product, exactly
  float t = tgv_exp(y);
  return tgv_fma(t, err, t);      // e^(y + err) ~ e^y (1 + err)
}

#ifdef __CUDACC__
// Diffusion-tensor weight exp(-beta |grad I|^gamma) before its 1e-8 floor (calcTensor.cu:60-64).
// cuda_math != 0: CUDA's expf / powf, the calls the reference makes, so the tensor is the
// reference's to the bit (the default).  cuda_math == 0: the portable construction above,
// which a host restatement reproduces bit for bit.
__device__ __forceinline__ float tensor_weight(float abs_img, float beta, float gamma, int cuda_math) {
  if (cuda_math) return expf(-beta * powf(abs_img, gamma));
  return tgv_exp(-beta * tgv_pow(abs_img, gamma));
}
#endif

}  // namespace vfs
