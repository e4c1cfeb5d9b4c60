// CPU oracle for the variational fisheye stereo (TGV-L1) solve path.
//
// TEST INFRASTRUCTURE ONLY. This file restates, on the host, the algorithm of
// the reference `StereoTgv` solver (menandro/vfs, stereotgv/*.cu) so that the
// CUDA implementation in vfs_b200/csrc can be checked against it. Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load it; the product
// path never calls into it.
//
// Parity pins: the texture-unit model below is checked bit-for-bit against
// samples recorded from B200 texture hardware (tests/golden/texunit), and the
// full masked solve is checked against the reference's own known-answer depth
// maps z16.png / depth16.png (tests/golden/wang_half).
//
// Design: the reference keeps ~40 device buffers of the full-resolution pitched
// size (stride0 * height0 elements), reuses them at every pyramid level with the
// level's own stride, swaps pointers between ping-pong pairs, and lets masked
// kernels skip masked-out pixels.  Masked-out pixels therefore keep stale values
// that later leak into the median filter and the divergence edge rules.  This
// oracle reproduces that memory model literally: every reference buffer is a
// flat array of the same size, Swap() swaps the arrays, and every kernel writes
// exactly the pixels the reference kernel writes.
//
// Arithmetic type R: double ("FP64 oracle", the accuracy reference) or float
// (an FP32 restatement whose operation order follows the reference kernels, used
// for tight parity of the FP32 CUDA path).  Compile with -ffp-contract=off.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

namespace vfs_oracle {

// ---------------------------------------------------------------------------
// Texture unit model (normalized coordinates, mirror addressing, pitch-2D,
// element read mode) as used by every tex2D() in the reference.  Measured on
// B200 hardware: the probes are tests/golden/texunit/texprobe.cu and texprobe_weights.cu, the
// recorded samples tests/golden/texunit/texunit.npz (made by make_fixture.py there).
//   1. the normalized coordinate c is truncated to 21 fractional bits;
//   2. linear: t = X*N - 0.5, i = floor(t), A = round_half_up(frac(t)*256)
//      (A == 256 moves to i+1 with A = 0);
//   3. corner weights in 1/256 units: w11 = round_half_up(A*B/256),
//      w10 = A - w11, w01 = B - w11, w00 = 256 - A - B + w11;
//   4. texel indices are mirrored with period 2N;
//   5. the weighted sum is exact and rounded to float with ties away from zero.
//   point: i = floor(X*N), mirrored.
// ---------------------------------------------------------------------------
static inline int64_t mirror_index(int64_t k, int n) {
  int64_t p = k % (2 * (int64_t)n);
  if (p < 0) p += 2 * (int64_t)n;
  return p < n ? p : 2 * (int64_t)n - 1 - p;
}

static inline double quant_coord(double c) { return std::floor(c * 2097152.0) / 2097152.0; }

static inline void lin_index(double c, int n, int64_t& i, int& A) {
  double t = quant_coord(c) * (double)n - 0.5;
  double fl = std::floor(t);
  i = (int64_t)fl;
  A = (int)std::floor((t - fl) * 256.0 + 0.5);
  if (A == 256) { i += 1; A = 0; }
}

// round a double to float, ties away from zero
static inline float round_f32_rna(double x) {
  float f = (float)x;
  double fd = (double)f;
  if (fd == x) return f;
  float other = std::nextafter(f, x > fd ? INFINITY : -INFINITY);
  double od = (double)other;
  if (std::fabs(od - x) == std::fabs(x - fd) && std::fabs(od) > std::fabs(fd)) return other;
  return f;
}

template <class R> struct TexOut { static R cvt(double v) { return (R)v; } };
template <> struct TexOut<float> { static float cvt(double v) { return round_f32_rna(v); } };

// Global switch: 1 = hardware texture model (default); 0 = exact bilinear
// weights (for analysis of the quantisation effect only).
static int g_hw_texture = 1;

// Bilinear sample of component `comp` of a pitched buffer with `comps`
// interleaved components, logical size w x h, row stride s (elements per
// component-row).
template <class R>
static inline R tex_linear(const R* buf, int comps, int comp, int w, int h, int s, R xn, R yn) {
  if (!g_hw_texture) {
    double tx = (double)xn * w - 0.5, ty = (double)yn * h - 0.5;
    double fx = std::floor(tx), fy = std::floor(ty);
    double a = tx - fx, b = ty - fy;
    int64_t ix = (int64_t)fx, iy = (int64_t)fy;
    int64_t x0 = mirror_index(ix, w), x1 = mirror_index(ix + 1, w);
    int64_t y0 = mirror_index(iy, h), y1 = mirror_index(iy + 1, h);
    auto T = [&](int64_t x, int64_t y) { return (double)buf[((size_t)y * s + x) * comps + comp]; };
    double v = (1 - a) * (1 - b) * T(x0, y0) + a * (1 - b) * T(x1, y0) + (1 - a) * b * T(x0, y1) + a * b * T(x1, y1);
    return (R)v;
  }
  int64_t ix, iy;
  int A, B;
  lin_index((double)xn, w, ix, A);
  lin_index((double)yn, h, iy, B);
  int w11 = (int)std::floor((double)(A * B) / 256.0 + 0.5);
  int w10 = A - w11, w01 = B - w11, w00 = 256 - A - B + w11;
  int64_t x0 = mirror_index(ix, w), x1 = mirror_index(ix + 1, w);
  int64_t y0 = mirror_index(iy, h), y1 = mirror_index(iy + 1, h);
  auto T = [&](int64_t x, int64_t y) { return (double)buf[((size_t)y * s + x) * comps + comp]; };
  double v = ((double)w00 * T(x0, y0) + (double)w10 * T(x1, y0) + (double)w01 * T(x0, y1) + (double)w11 * T(x1, y1)) / 256.0;
  return TexOut<R>::cvt(v);
}

template <class R>
static inline R tex_point(const R* buf, int comps, int comp, int w, int h, int s, R xn, R yn) {
  int64_t ix = (int64_t)std::floor(quant_coord((double)xn) * w);
  int64_t iy = (int64_t)std::floor(quant_coord((double)yn) * h);
  if (!g_hw_texture) { ix = (int64_t)std::floor((double)xn * w); iy = (int64_t)std::floor((double)yn * h); }
  ix = mirror_index(ix, w);
  iy = mirror_index(iy, h);
  return buf[((size_t)iy * s + ix) * comps + comp];
}

// ---------------------------------------------------------------------------
// Float exp / log / pow from correctly rounded operations only: Cody-Waite
// reduction x = k ln2 + r and the degree-7 Taylor series of e^r; ln a =
// e ln2 + 2 atanh((m-1)/(m+1)) with m in [sqrt(1/2), sqrt(2)), atanh by its odd
// power series to s^11.
static const float kLn2Hi = 0.693145751953125f;
static const float kLn2Lo = 1.4286068203e-06f;
static const float kInvLn2 = 1.44269504088896f;

static float f32_exp(float x) {
  if (x != x) return x;
  if (x < -87.0f) return 0.0f;
  if (x > 88.0f) return INFINITY;
  float k = std::rint(x * kInvLn2);
  float r = std::fma(-k, kLn2Hi, x);
  r = std::fma(-k, kLn2Lo, r);
  float p = 1.0f / 5040.0f;
  p = std::fma(p, r, 1.0f / 720.0f);
  p = std::fma(p, r, 1.0f / 120.0f);
  p = std::fma(p, r, 1.0f / 24.0f);
  p = std::fma(p, r, 1.0f / 6.0f);
  p = std::fma(p, r, 0.5f);
  p = std::fma(p, r, 1.0f);
  p = std::fma(p, r, 1.0f);
  return std::ldexp(p, (int)k);
}

static float f32_log(float a) {
  int e;
  float m = std::frexp(a, &e);
  if (m < 0.70710678f) { m = m * 2.0f; e -= 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float q = 1.0f / 11.0f;
  q = std::fma(q, s2, 1.0f / 9.0f);
  q = std::fma(q, s2, 1.0f / 7.0f);
  q = std::fma(q, s2, 1.0f / 5.0f);
  q = std::fma(q, s2, 1.0f / 3.0f);
  q = std::fma(q, s2, 1.0f);
  float lnm = 2.0f * s * q;
  float fe = (float)e;
  return std::fma(fe, kLn2Hi, std::fma(fe, kLn2Lo, lnm));
}

static float f32_pow(float a, float g) {
  if (a == 0.0f) return 0.0f;
  if (!(a > 0.0f) || std::isinf(a)) return a != a ? a : (std::isinf(a) ? INFINITY : NAN);
  float l = f32_log(a);
  float y = g * l;
  float err = std::fma(g, l, -y);
  float t = f32_exp(y);
  return std::fma(t, err, t);
}

// ---------------------------------------------------------------------------
struct Params {
  int width, height;
  float beta, gamma, alpha0, alpha1, timestep_lambda, lambda;
  int nLevels;
  float fScale;
  int nWarpIters, nSolverIters;
  float limitRange;
  int blockWidth, strideAlignment;
};

typedef std::vector<double> Buf64;

template <class R>
struct Solver {
  typedef std::vector<R> Buf;
  Params P;
  int width = 0, height = 0, stride = 0;
  size_t full = 0;  // elements per component of a full-resolution buffer
  std::vector<int> pW, pH, pS;
  std::vector<Buf> pI0, pI1, pTvF, pMask;
  // full-resolution buffers (stereotgv.cu:106-153); float2 buffers are
  // interleaved (2 components), float4 buffers 4 components.
  Buf i1calibrated, i1warp, i0smooth, Iu, Iz, u, du, us, warpUV, dwarpUV, warpUVs, tv2, cv;
  Buf a, b, c, etau, etav1, etav2, p, q, u_, u_last, u_s, v, v_, v_s, Tp;
  Buf X, depth;  // ConvertKB outputs (float3 and float)

  int iAlignUp(int n) const {  // stereotgv.cu:571-580
    int m = P.strideAlignment;
    int mod = n % m;
    return mod ? n + m - mod : n;
  }

  // stereotgv.cu:44-168
  void initialize(const Params& prm) {
    P = prm;
    width = P.width;
    height = P.height;
    stride = iAlignUp(width);
    full = (size_t)stride * height;
    int L = P.nLevels;
    pW.assign(L, 0); pH.assign(L, 0); pS.assign(L, 0);
    pI0.assign(L, Buf()); pI1.assign(L, Buf()); pTvF.assign(L, Buf()); pMask.assign(L, Buf());
    int newHeight = height, newWidth = width, newStride = iAlignUp(width);
    for (int level = 0; level < L; level++) {
      size_t n = (size_t)newStride * newHeight;
      pI0[level].assign(n, R(0));
      pI1[level].assign(n, R(0));
      pTvF[level].assign(2 * n, R(0));
      pMask[level].assign(n, R(0));
      pW[level] = newWidth; pH[level] = newHeight; pS[level] = newStride;
      newHeight = (int)((float)newHeight / P.fScale);
      newWidth = (int)((float)newWidth / P.fScale);
      newStride = iAlignUp(newWidth);
    }
    for (Buf* bf : {&i1calibrated, &i1warp, &i0smooth, &Iu, &Iz, &u, &du, &us, &a, &b, &c, &etau, &etav1,
                    &etav2, &u_, &u_last, &u_s, &depth})
      bf->assign(full, R(0));
    for (Buf* bf : {&warpUV, &dwarpUV, &warpUVs, &tv2, &cv, &p, &v, &v_, &v_s, &Tp}) bf->assign(2 * full, R(0));
    q.assign(4 * full, R(0));
    X.assign(3 * full, R(0));
  }

  // ---- kernels -----------------------------------------------------------
  // downscale.cu:10-30 (float) / :98-122 (float2)
  void Downscale(const Buf& src, int comps, int w, int h, int s, int nw, int nh, int ns, Buf& out) {
#pragma omp parallel for
    for (int iy = 0; iy < nh; iy++)
      for (int ix = 0; ix < nw; ix++) {
        R dx = R(1) / (R)nw, dy = R(1) / (R)nh;
        R x = ((R)ix + R(0.5)) * dx, y = ((R)iy + R(0.5)) * dy;
        size_t pos = (size_t)ix + (size_t)iy * ns;
        for (int k = 0; k < comps; k++) {
          R t1 = tex_linear(src.data(), comps, k, w, h, s, x - dx * R(0.25), y);
          R t2 = tex_linear(src.data(), comps, k, w, h, s, x + dx * R(0.25), y);
          R t3 = tex_linear(src.data(), comps, k, w, h, s, x, y - dy * R(0.25));
          R t4 = tex_linear(src.data(), comps, k, w, h, s, x, y + dy * R(0.25));
          out[pos * comps + k] = R(0.25) * (t1 + t2 + t3 + t4);
        }
      }
  }

  // downscale.cu:52-73 (point sampling)
  void DownscaleNearest(const Buf& src, int w, int h, int s, int nw, int nh, int ns, Buf& out) {
#pragma omp parallel for
    for (int iy = 0; iy < nh; iy++)
      for (int ix = 0; ix < nw; ix++) {
        R dx = R(1) / (R)nw, dy = R(1) / (R)nh;
        R x = ((R)ix + R(0.5)) * dx, y = ((R)iy + R(0.5)) * dy;
        out[(size_t)ix + (size_t)iy * ns] = tex_point(src.data(), 1, 0, w, h, s, x, y);
      }
  }

  // warpImage.cu:9-23 (texture of src bound with w, h, s)
  void WarpImage(const Buf& src, int w, int h, int s, const Buf& wuv, Buf& out) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) {
        size_t pos = (size_t)ix + (size_t)iy * s;
        R x = ((R)ix + wuv[2 * pos] + R(0.5)) / (R)w;
        R y = ((R)iy + wuv[2 * pos + 1] + R(0.5)) / (R)h;
        out[pos] = tex_linear(src.data(), 1, 0, w, h, s, x, y);
      }
  }

  // warpImage.cu:96-111
  void FindWarpingVector(const Buf& wuv, const Buf& tv, int w, int h, int s, Buf& out) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) {
        size_t pos = (size_t)ix + (size_t)iy * s;
        R x = ((R)ix + wuv[2 * pos] + R(0.5)) / (R)w;
        R y = ((R)iy + wuv[2 * pos + 1] + R(0.5)) / (R)h;
        out[2 * pos] = tex_linear(tv.data(), 2, 0, w, h, s, x, y);
        out[2 * pos + 1] = tex_linear(tv.data(), 2, 1, w, h, s, x, y);
      }
  }

  // warpImage.cu:136-150
  void ComputeOpticalFlowVector(const Buf& uu, const Buf& t2, int w, int h, int s, Buf& out) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) {
        size_t pos = (size_t)ix + (size_t)iy * s;
        R usv = uu[pos];
        out[2 * pos] = usv * t2[2 * pos];
        out[2 * pos + 1] = usv * t2[2 * pos + 1];
      }
  }

  // computeDerivatives.cu:89-129 (texI0 = I0, texI1 = I1 warped)
  void ComputeDerivativesFisheye(const Buf& I0, const Buf& I1, const Buf& vec, int w, int h, int s, Buf& Iw,
                                 Buf& Izo) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) {
        size_t pos = (size_t)ix + (size_t)iy * s;
        R vx = vec[2 * pos], vy = vec[2 * pos + 1];
        R r = std::sqrt(vx * vx + vy * vy);
        R dx = (vx / r) / (R)w;
        R dy = (vy / r) / (R)h;
        R x = ((R)ix + R(0.5)) / (R)w;
        R y = ((R)iy + R(0.5)) / (R)h;
        auto T0 = [&](R xx, R yy) { return tex_linear(I0.data(), 1, 0, w, h, s, xx, yy); };
        auto T1 = [&](R xx, R yy) { return tex_linear(I1.data(), 1, 0, w, h, s, xx, yy); };
        R t0 = T0(x - R(2) * dx, y - R(2) * dy);
        t0 -= T0(x - R(1) * dx, y - R(1) * dy) * R(8);
        t0 += T0(x + R(1) * dx, y + R(1) * dy) * R(8);
        t0 -= T0(x + R(2) * dx, y + R(2) * dy);
        t0 /= R(12);
        R t1 = T1(x - R(2) * dx, y - R(2) * dy);
        t1 -= T1(x - R(1) * dx, y - R(1) * dy) * R(8);
        t1 += T1(x + R(1) * dx, y + R(1) * dy) * R(8);
        t1 -= T1(x + R(2) * dx, y + R(2) * dy);
        t1 /= R(12);
        Iw[pos] = (t0 + t1) * R(0.5);
        Izo[pos] = T1(x, y) - T0(x, y);
      }
  }

  // calcTensor.cu:99-128 (plain) and :245-273 (masked)
  void Gaussian(const Buf& in, const R* mask, int w, int h, int s, Buf& out) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) {
        size_t pos = (size_t)ix + (size_t)iy * s;
        if (mask && mask[pos] == R(0)) continue;
        R dx = R(1) / (R)w, dy = R(1) / (R)h;
        R x = ((R)ix + R(0.5)) * dx, y = ((R)iy + R(0.5)) * dy;
        auto T = [&](R xx, R yy) { return tex_linear(in.data(), 1, 0, w, h, s, xx, yy); };
        R t0 = (R(1) / R(4)) * T(x, y);
        t0 += (R(1) / R(16)) * T(x - R(1) * dx, y - R(1) * dy);
        t0 += (R(1) / R(16)) * T(x - R(1) * dx, y + R(1) * dy);
        t0 += (R(1) / R(16)) * T(x + R(1) * dx, y - R(1) * dy);
        t0 += (R(1) / R(16)) * T(x + R(1) * dx, y + R(1) * dy);
        t0 += (R(1) / R(8)) * T(x - R(1) * dx, y);
        t0 += (R(1) / R(8)) * T(x + R(1) * dx, y);
        t0 += (R(1) / R(8)) * T(x, y - R(1) * dy);
        t0 += (R(1) / R(8)) * T(x, y + R(1) * dy);
        out[pos] = t0;
      }
  }

  // expf(-beta * powf(abs_img, gamma)) (calcTensor.cu:61-64).  The float
  // restatement evaluates exp and pow with f32_exp / f32_pow (below), the
  // same correctly-rounded-operation construction the CUDA kernel uses, so both
  // produce identical bits; in double it is the libm double exp / pow.
  static R tensor_exp_weight(R beta, R gamma, R abs_img) {
    if (sizeof(R) == sizeof(float)) return (R)f32_exp(-(float)beta * f32_pow((float)abs_img, (float)gamma));
    return (R)std::exp((double)(-beta) * std::pow((double)abs_img, (double)gamma));
  }

  // calcTensor.cu:8-73 (plain) and :155-219 (masked). The launch grid of the
  // reference covers columns ix < blockWidth * ceil(h / blockWidth)
  // (calcTensor.cu:81,227), so columns beyond that keep a = b = c = 0.
  void CalcTensor(const Buf& gray, const R* mask, R beta, R gamma, int w, int h, int s, Buf& A, Buf& B, Buf& C) {
    int bw = P.blockWidth;
    int xcov = ((h + bw - 1) / bw) * bw;
    int xmax = std::min(w, xcov);
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < xmax; ix++) {
        size_t pos = (size_t)ix + (size_t)iy * s;
        if (mask && mask[pos] == R(0)) continue;
        R dx = R(1) / (R)w, dy = R(1) / (R)h;
        R x = ((R)ix + R(0.5)) * dx, y = ((R)iy + R(0.5)) * dy;
        auto T = [&](R xx, R yy) { return tex_linear(gray.data(), 1, 0, w, h, s, xx, yy); };
        R gx = T(x + R(1) * dx, y + R(1) * dy) - T(x, y + R(1) * dy);
        R gy = T(x + R(1) * dx, y + R(1) * dy) - T(x + R(1) * dx, y);
        R abs_img = std::sqrt(gx * gx + gy * gy);
        R norm_n = abs_img;
        R nx = gx / norm_n, ny = gy / norm_n;
        if (norm_n < R(1e-8f)) { nx = R(1); ny = R(0); }
        R ntx = ny, nty = -nx;
        R wt = tensor_exp_weight(beta, gamma, abs_img);
        if (!(wt > R(1e-8f))) wt = R(1e-8f);
        A[pos] = wt * nx * nx + ntx * ntx;
        C[pos] = wt * nx * ny + ntx * nty;
        B[pos] = wt * ny * ny + nty * nty;
      }
  }

  // preconditioning.cu:3-22 (plain) and :41-60 (masked)
  void SolveEta(const R* mask, R alpha0, R alpha1, int w, int h, int s) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) {
        size_t pos = (size_t)ix + (size_t)iy * s;
        if (mask && mask[pos] == R(0)) continue;
        R aa = a[pos], bb = b[pos], cc = c[pos];
        etau[pos] = (aa * aa + bb * bb + R(2) * cc * cc + (aa + cc) * (aa + cc) + (bb + cc) * (bb + cc)) * (alpha1 * alpha1);
        etav1[pos] = (alpha1 * alpha1) * (bb * bb + cc * cc) + R(4) * alpha0 * alpha0;
        etav2[pos] = (alpha1 * alpha1) * (aa * aa + cc * cc) + R(4) * alpha0 * alpha0;
      }
  }

  static inline bool outside_circle(int ix, int iy, int w, int h) {
    // updateDualVariables.cu:13-16 (float arithmetic in every mode: a discrete decision)
    float desiredRadius = (float)w / 2.20f;
    float halfWidth = (float)w / 2.0f;
    float halfHeight = (float)h / 2.0f;
    float radius = std::sqrt((iy - halfHeight) * (iy - halfHeight) + (ix - halfWidth) * (ix - halfWidth));
    return radius >= desiredRadius;
  }

  // flat read used by the masked edge rules: a flat index before the buffer
  // start (only reachable for masks that are on in row 0 / column 0) reads 0.
  static inline R rd(const Buf& B, int64_t k, int comps, int comp) {
    return k < 0 ? R(0) : B[(size_t)k * comps + comp];
  }

  // updateDualVariables.cu:4-101 (plain, circle) and :122-237 (masked)
  void UpdateDual(const R* mask, R alpha0, R alpha1, R sigma, R eta_p, R eta_q, int w, int h, int s) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) {
        int64_t pos = (int64_t)ix + (int64_t)iy * s;
        int64_t right = pos + 1, down = pos + s, left = pos - 1, up = pos - s;
        bool useRight, useDown;
        if (mask) {
          if (mask[pos] == R(0)) continue;
          R maskRight = (ix + 1 >= w) ? R(0) : mask[right];
          R maskDown = (iy + 1 >= h) ? R(0) : mask[down];
          useRight = maskRight != R(0);
          useDown = maskDown != R(0);
        } else {
          if (outside_circle(ix, iy, w, h)) {
            p[2 * pos] = p[2 * pos + 1] = R(0);
            for (int k = 0; k < 4; k++) q[4 * pos + k] = R(0);
            continue;
          }
          useRight = (ix + 1) < w;
          useDown = (iy + 1) < h;
        }
        R u_pos = u_[pos];
        R vpx = v_[2 * pos], vpy = v_[2 * pos + 1];
        R u_x = useRight ? u_[right] - u_pos - vpx : u_pos - rd(u_, left, 1, 0) - vpx;
        R u_y = useDown ? u_[down] - u_pos - vpy : u_pos - rd(u_, up, 1, 0) - vpy;
        R dtx = a[pos] * u_x + c[pos] * u_y;
        R dty = c[pos] * u_x + b[pos] * u_y;
        R ppx = p[2 * pos] + (alpha1 * sigma / eta_p) * dtx;
        R ppy = p[2 * pos + 1] + (alpha1 * sigma / eta_p) * dty;
        R rep = std::sqrt(ppx * ppx + ppy * ppy);
        if (rep < R(1)) rep = R(1);
        p[2 * pos] = ppx / rep;
        p[2 * pos + 1] = ppy / rep;
        R gvx = useRight ? v_[2 * right] - vpx : vpx - rd(v_, left, 2, 0);
        R gvy = useDown ? v_[2 * down + 1] - vpy : vpy - rd(v_, up, 2, 1);
        R gvz = useDown ? v_[2 * down] - vpx : vpx - rd(v_, up, 2, 0);
        R gvw = useRight ? v_[2 * right + 1] - vpy : vpy - rd(v_, left, 2, 1);
        R ase = alpha0 * sigma / eta_q;
        R qx = q[4 * pos] + ase * gvx;
        R qy = q[4 * pos + 1] + ase * gvy;
        R qz = q[4 * pos + 2] + ase * gvz;
        R qw = q[4 * pos + 3] + ase * gvw;
        R reproj = std::sqrt(qx * qx + qy * qy + qz * qz + qw * qw);
        if (reproj < R(1)) reproj = R(1);
        q[4 * pos] = qx / reproj;
        q[4 * pos + 1] = qy / reproj;
        q[4 * pos + 2] = qz / reproj;
        q[4 * pos + 3] = qw / reproj;
      }
  }

  // thresholdingL1.cu:104-115 (plain, all pixels) and :234-244 (masked)
  void SolveTp(const R* mask, int w, int h, int s) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) {
        size_t pos = (size_t)ix + (size_t)iy * s;
        if (mask && mask[pos] == R(0)) continue;
        R px = p[2 * pos], py = p[2 * pos + 1];
        Tp[2 * pos] = a[pos] * px + c[pos] * py;
        Tp[2 * pos + 1] = c[pos] * px + b[pos] * py;
      }
  }

  // thresholdingL1.cu:3-86 (plain) and :128-216 (masked); reads u, writes us.
  void ThresholdingL1(const R* mask, R lambda, R tau, int w, int h, int s) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) {
        int64_t pos = (int64_t)ix + (int64_t)iy * s;
        int64_t left = pos - 1, up = pos - s;
        R dxm, dym;
        if (mask) {
          if (mask[pos] == R(0)) continue;
          R mR = (ix + 1 >= w) ? R(0) : mask[pos + 1];
          R mL = (ix - 1 < 0) ? R(0) : mask[left];
          R mD = (iy + 1 >= h) ? R(0) : mask[pos + s];
          R mU = (iy - 1 < 0) ? R(0) : mask[up];
          if (mL != R(0) && mR != R(0)) dxm = Tp[2 * pos] - Tp[2 * left];
          else if (mR == R(0)) dxm = -rd(Tp, left, 2, 0);
          else dxm = Tp[2 * pos];
          if (mU != R(0) && mD != R(0)) dym = Tp[2 * pos + 1] - Tp[2 * up + 1];
          else if (mD == R(0)) dym = -rd(Tp, up, 2, 1);
          else dym = Tp[2 * pos + 1];
        } else {
          if (outside_circle(ix, iy, w, h)) { us[pos] = R(0); continue; }
          if ((ix - 1) >= 0) dxm = Tp[2 * pos] - Tp[2 * left];
          else if (ix == w - 1) dxm = -rd(Tp, left, 2, 0);
          else dxm = Tp[2 * pos];
          if ((iy - 1) >= 0) dym = Tp[2 * pos + 1] - Tp[2 * up + 1];
          else if (iy == h - 1) dym = -rd(Tp, up, 2, 1);
          else dym = Tp[2 * pos + 1];
        }
        R div_p = dxm + dym;
        R tau_eta_u = (etau[pos] == R(0)) ? tau : tau / etau[pos];
        R uhat = u_[pos] + tau_eta_u * div_p;
        R dun = uhat - u[pos];
        R Ius = Iu[pos];
        R rho = Ius * dun + Iz[pos];
        R upper = lambda * tau_eta_u * (Ius * Ius);
        R lower = -lambda * tau_eta_u * (Ius * Ius);
        R d = R(0);
        if ((rho <= upper) && (rho >= lower)) {
          if (Ius == R(0)) d = dun;
          else d = dun - rho / Ius;
        } else if (rho < lower) {
          d = dun + lambda * tau_eta_u * Ius;
        } else if (rho > upper) {
          d = dun - lambda * tau_eta_u * Ius;
        }
        us[pos] = u[pos] + d;
      }
  }

  // updatePrimalVariables.cu:3-113 (plain) and :139-245 (masked); reads u
  // (the thresholded iterate), writes v, u_s, v_s.
  void UpdatePrimal(const R* mask, R tau, R alpha0, R alpha1, R mu, int w, int h, int s) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) {
        int64_t pos = (int64_t)ix + (int64_t)iy * s;
        int64_t left = pos - 1, up = pos - s;
        bool zR, zD, hasL, hasU;
        if (mask) {
          if (mask[pos] == R(0)) continue;
          R mR = (ix + 1 >= w) ? R(0) : mask[pos + 1];
          R mL = (ix - 1 < 0) ? R(0) : mask[left];
          R mD = (iy + 1 >= h) ? R(0) : mask[pos + s];
          R mU = (iy - 1 < 0) ? R(0) : mask[up];
          zR = mR == R(0); zD = mD == R(0); hasL = mL != R(0); hasU = mU != R(0);
        } else {
          if (outside_circle(ix, iy, w, h)) {
            u_s[pos] = R(0);
            v_s[2 * pos] = v_s[2 * pos + 1] = R(0);
            continue;
          }
          zR = ix == w - 1; zD = iy == h - 1; hasL = (ix - 1) >= 0; hasU = (iy - 1) >= 0;
        }
        R qcx = zR ? R(0) : q[4 * pos], qcw = zR ? R(0) : q[4 * pos + 3];
        R qcy = zD ? R(0) : q[4 * pos + 1], qcz = zD ? R(0) : q[4 * pos + 2];
        R qwx = hasL ? q[4 * left] : R(0), qww = hasL ? q[4 * left + 3] : R(0);
        R qny = hasU ? q[4 * up + 1] : R(0), qnz = hasU ? q[4 * up + 2] : R(0);
        R dqx = (qcx - qwx) + (qcz - qnz);
        R dqy = (qcw - qww) + (qcy - qny);
        R ppx = p[2 * pos], ppy = p[2 * pos + 1];
        R dtx = a[pos] * ppx + c[pos] * ppy;
        R dty = c[pos] * ppx + b[pos] * ppy;
        R ev1 = etav1[pos], ev2 = etav2[pos];
        R vbx = v_[2 * pos], vby = v_[2 * pos + 1];
        R vx, vy;
        if (ev1 != R(0)) vx = vbx + (tau / ev1) * (alpha1 * dtx + alpha0 * dqx);
        else vx = vbx + (tau) * (alpha1 * dtx + alpha0 * dqx);
        if (ev2 != R(0)) vy = vby + (tau / ev2) * (alpha1 * dty + alpha0 * dqy);
        else {  // reference writes .x again and leaves .y unset (updatePrimalVariables.cu:103-105)
          vx = vbx + (tau) * (alpha1 * dtx + alpha0 * dqx);
          vy = vby;
        }
        v[2 * pos] = vx;
        v[2 * pos + 1] = vy;
        u_s[pos] = u[pos] + mu * (u[pos] - u_[pos]);
        v_s[2 * pos] = vx + mu * (vx - vbx);
        v_s[2 * pos + 1] = vy + mu * (vy - vby);
      }
  }

  // medianFilter.cu:264-319 (5x5; out-of-range corner taps stay 0)
  void MedianFilter5(const Buf& in, int w, int h, int s, Buf& out) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) {
        R mu[25];
        for (int j = 0; j < 5; j++)
          for (int i = 0; i < 5; i++) {
            int col = ix + i - 2, row = iy + j - 2;
            R val = R(0);
            bool cin = col >= 0 && col < w, rin = row >= 0 && row < h;
            if (cin && rin) val = in[(size_t)col + (size_t)s * row];
            else if (col < 0 && rin) val = in[(size_t)s * row];
            else if (col >= w && rin) val = in[(size_t)(w - 1) + (size_t)s * row];
            else if (cin && row < 0) val = in[(size_t)col];
            else if (cin && row >= h) val = in[(size_t)col + (size_t)s * (h - 1)];
            mu[j * 5 + i] = val;
          }
        for (int j = 0; j < 13; j++)
          for (int i = j + 1; i < 25; i++)
            if (mu[j] > mu[i]) std::swap(mu[j], mu[i]);
        out[(size_t)ix + (size_t)iy * s] = mu[12];
      }
  }

  // upscale.cu:8-21 / :46-61
  void Upscale(const Buf& src, int comps, int w, int h, int s, int nw, int nh, int ns, R scale, Buf& out) {
#pragma omp parallel for
    for (int iy = 0; iy < nh; iy++)
      for (int ix = 0; ix < nw; ix++) {
        R x = ((R)ix + R(0.5)) / (R)nw;
        R y = ((R)iy + R(0.5)) / (R)nh;
        size_t pos = (size_t)ix + (size_t)iy * ns;
        for (int k = 0; k < comps; k++) out[pos * comps + k] = tex_linear(src.data(), comps, k, w, h, s, x, y) * scale;
      }
  }

  // scalar.cu / limitRange.cu / copyClone.cu point-wise helpers (all px < w, h)
  template <class F>
  void pointwise(int w, int h, int s, F f) {
#pragma omp parallel for
    for (int iy = 0; iy < h; iy++)
      for (int ix = 0; ix < w; ix++) f((size_t)ix + (size_t)iy * s);
  }

  // ---- host API ----------------------------------------------------------
  // stereotgv.cu:171-199 (translation field pyramid; the backward field is
  // never used by the solver and is not kept)
  void loadVectorFields(const float* tv, const float* cvf) {
    std::fill(pTvF[0].begin(), pTvF[0].end(), R(0));
    std::fill(cv.begin(), cv.end(), R(0));
    for (int y = 0; y < height; y++)
      for (int x = 0; x < width; x++)
        for (int k = 0; k < 2; k++) {
          pTvF[0][((size_t)y * stride + x) * 2 + k] = (R)tv[((size_t)y * width + x) * 2 + k];
          cv[((size_t)y * stride + x) * 2 + k] = (R)cvf[((size_t)y * width + x) * 2 + k];
        }
    for (int l = 1; l < P.nLevels; l++)
      Downscale(pTvF[l - 1], 2, pW[l - 1], pH[l - 1], pS[l - 1], pW[l], pH[l], pS[l], pTvF[l]);
  }

  // stereotgv.cu:241-252
  void copyMaskToDevice(const float* mask) {
    std::fill(pMask[0].begin(), pMask[0].end(), R(0));
    for (int y = 0; y < height; y++)
      for (int x = 0; x < width; x++) pMask[0][(size_t)y * stride + x] = (R)mask[(size_t)y * width + x];
    for (int l = 1; l < P.nLevels; l++)
      DownscaleNearest(pMask[l - 1], pW[l - 1], pH[l - 1], pS[l - 1], pW[l], pH[l], pS[l], pMask[l]);
  }

  // stereotgv.cu:201-213 + imageConverter.cu:4-15
  void copyImagesToDevice(const uint8_t* i0, const uint8_t* i1) {
    for (int y = 0; y < height; y++)
      for (int x = 0; x < width; x++) {
        pI0[0][(size_t)y * stride + x] = (R)((float)i0[(size_t)y * width + x] / 256.0f);
        pI1[0][(size_t)y * stride + x] = (R)((float)i1[(size_t)y * width + x] / 256.0f);
      }
  }
  // stereotgv.cu:227-230 (CV_32F input: copied as is)
  void copyImagesToDeviceF32(const float* i0, const float* i1) {
    for (int y = 0; y < height; y++)
      for (int x = 0; x < width; x++) {
        pI0[0][(size_t)y * stride + x] = (R)i0[(size_t)y * width + x];
        pI1[0][(size_t)y * stride + x] = (R)i1[(size_t)y * width + x];
      }
  }

  // stereotgv.cu:389-515 (masked) and :256-387 (plain)
  void solve(bool masked) {
    WarpImage(pI1[0], width, height, stride, cv, i1calibrated);
    std::swap(pI1[0], i1calibrated);
    std::fill(u.begin(), u.end(), R(0));
    std::fill(u_.begin(), u_.end(), R(0));
    std::fill(warpUV.begin(), warpUV.end(), R(0));
    for (int l = 1; l < P.nLevels; l++) {
      Downscale(pI0[l - 1], 1, pW[l - 1], pH[l - 1], pS[l - 1], pW[l], pH[l], pS[l], pI0[l]);
      Downscale(pI1[l - 1], 1, pW[l - 1], pH[l - 1], pS[l - 1], pW[l], pH[l], pS[l], pI1[l]);
    }
    const R alpha0 = (R)P.alpha0, alpha1 = (R)P.alpha1, lambda = (R)P.lambda;
    for (int level = P.nLevels - 1; level >= 0; level--) {
      int w = pW[level], h = pH[level], s = pS[level];
      const R* mk = masked ? pMask[level].data() : nullptr;
      for (Buf* bf : {&a, &b, &c, &etau, &etav1, &etav2, &i0smooth}) std::fill(bf->begin(), bf->end(), R(0));
      const R eta_p = R(3), eta_q = R(2);
      if (level == P.nLevels - 1) ComputeOpticalFlowVector(u, pTvF[level], w, h, s, warpUV);
      Gaussian(pI0[level], mk, w, h, s, i0smooth);
      CalcTensor(i0smooth, mk, (R)P.beta, (R)P.gamma, w, h, s, a, b, c);
      SolveEta(mk, alpha0, alpha1, w, h, s);
      for (int warpIter = 0; warpIter < P.nWarpIters; warpIter++) {
        std::fill(p.begin(), p.end(), R(0));
        std::fill(q.begin(), q.end(), R(0));
        std::fill(v.begin(), v.end(), R(0));
        pointwise(w, h, s, [&](size_t pos) { v_[2 * pos] = v[2 * pos]; v_[2 * pos + 1] = v[2 * pos + 1]; });
        std::fill(du.begin(), du.end(), R(0));
        FindWarpingVector(warpUV, pTvF[level], w, h, s, tv2);
        WarpImage(pI1[level], w, h, s, warpUV, i1warp);
        ComputeDerivativesFisheye(pI0[level], i1warp, pTvF[level], w, h, s, Iu, Iz);
        pointwise(w, h, s, [&](size_t pos) { u_last[pos] = u[pos]; });
        // host-side step schedule (stereotgv.cu:449-456,476-477), float on the
        // host in the reference; R here.
        R tau = R(1);
        R sigma = R(1) / tau;
        for (int iter = 0; iter < P.nSolverIters; iter++) {
          R mu;
          if (sizeof(R) == sizeof(float)) {
            float tf = (float)tau, sg = (float)sigma;
            mu = sg < 1000.0f ? (R)(1.0f / std::sqrt(1 + 0.7f * tf * P.timestep_lambda)) : R(1);
          } else {
            mu = sigma < R(1000) ? R(1) / std::sqrt(R(1) + R(0.7f) * tau * (R)P.timestep_lambda) : R(1);
          }
          UpdateDual(mk, alpha0, alpha1, sigma, eta_p, eta_q, w, h, s);
          SolveTp(mk, w, h, s);
          ThresholdingL1(mk, lambda, tau, w, h, s);
          std::swap(u, us);
          UpdatePrimal(mk, tau, alpha0, alpha1, mu, w, h, s);
          std::swap(u_, u_s);
          std::swap(v_, v_s);
          sigma = sigma / mu;
          tau = tau * mu;
        }
        if (masked) {
          MedianFilter5(u, w, h, s, us);
          std::swap(u, us);
        }
        const R lr = (R)P.limitRange;
        pointwise(w, h, s, [&](size_t pos) { du[pos] = u[pos] - u_last[pos]; });
        pointwise(w, h, s, [&](size_t pos) { du[pos] = du[pos] > lr ? lr : du[pos]; });
        pointwise(w, h, s, [&](size_t pos) { u[pos] = u_last[pos] + du[pos]; });
        pointwise(w, h, s, [&](size_t pos) { u_[pos] = u[pos]; });
        ComputeOpticalFlowVector(du, tv2, w, h, s, dwarpUV);
        pointwise(w, h, s, [&](size_t pos) {
          warpUV[2 * pos] = warpUV[2 * pos] + dwarpUV[2 * pos];
          warpUV[2 * pos + 1] = warpUV[2 * pos + 1] + dwarpUV[2 * pos + 1];
        });
      }
      if (level > 0) {
        R scale = (R)P.fScale;
        int nw = pW[level - 1], nh = pH[level - 1], ns = pS[level - 1];
        Upscale(u, 1, w, h, s, nw, nh, ns, scale, us);
        Upscale(u_, 1, w, h, s, nw, nh, ns, scale, u_s);
        Upscale(warpUV, 2, w, h, s, nw, nh, ns, scale, warpUVs);
        std::swap(u, us);
        std::swap(u_, u_s);
        std::swap(warpUV, warpUVs);
      }
    }
  }

  // conversion.cu:3-69, called by copyStereoToHost (stereotgv.cu:517-531) with
  // the parameters in the reference's order (focalx, focaly, cx, cy, ...).
  void ConvertKB(R focalx, R focaly, R cx, R cy, R d1, R d2, R d3, R d4, R t1, R t2, R t3) {
    pointwise(width, height, stride, [&](size_t pos) {
      int ix = (int)(pos % stride), iy = (int)(pos / stride);
      R u0 = (R)ix, v0 = (R)iy;
      R xp0 = (u0 - focalx) / cx, yp0 = (v0 - focaly) / cy;
      R uu = warpUV[2 * pos], vv = warpUV[2 * pos + 1];
      R u1 = u0 + uu, v1 = v0 + vv;
      R xp1 = (u1 - focalx) / cx, yp1 = (v1 - focaly) / cy;
      auto newton = [&](R ru) {
        R th = R(0);
        for (int it = 0; it < 5; it++) {
          R thd = th + d1 * std::pow(th, R(3)) + d2 * std::pow(th, R(5)) + d3 * std::pow(th, R(7)) + d4 * std::pow(th, R(9));
          R dthd = R(1) + R(3) * d1 * std::pow(th, R(2)) + R(5) * d2 * std::pow(th, R(4)) + R(7) * d3 * std::pow(th, R(6)) +
                   R(9) * d4 * std::pow(th, R(8));
          R f = ru - thd;
          R fp = -dthd;
          th = th - f / fp;
        }
        return th;
      };
      R ru0 = std::sqrt(xp0 * xp0 + yp0 * yp0);
      R th0 = newton(ru0);
      R x0o = std::tan(th0) * xp0 / ru0, y0o = std::tan(th0) * yp0 / ru0;
      R ru1 = std::sqrt(xp1 * xp1 + yp1 * yp1);
      R th1 = newton(ru1);
      R x1o = std::tan(th1) * xp1 / ru1, y1o = std::tan(th1) * yp1 / ru1;
      R Zx = (t1 - x1o * t3) / (x1o - x0o);
      R Z = Zx;
      X[3 * pos] = x0o * Z;
      X[3 * pos + 1] = y0o * Z;
      X[3 * pos + 2] = Z;
      depth[pos] = std::sqrt(X[3 * pos] * X[3 * pos] + X[3 * pos + 1] * X[3 * pos + 1] + X[3 * pos + 2] * X[3 * pos + 2]);
    });
  }

  // buffer lookup for the C API getters
  const Buf* named(const char* n) const {
    struct E { const char* n; const Buf* b; };
    E tab[] = {{"u", &u}, {"u_", &u_}, {"warpUV", &warpUV}, {"a", &a}, {"b", &b}, {"c", &c}, {"etau", &etau},
               {"etav1", &etav1}, {"etav2", &etav2}, {"Iu", &Iu}, {"Iz", &Iz}, {"i1warp", &i1warp}, {"tv2", &tv2},
               {"i0smooth", &i0smooth}, {"p", &p}, {"q", &q}, {"v_", &v_}, {"Tp", &Tp}, {"us", &us},
               {"u_s", &u_s}, {"v_s", &v_s}, {"du", &du}, {"u_last", &u_last}, {"X", &X}, {"depth", &depth},
               {"warpUVs", &warpUVs}, {"i1calibrated", &i1calibrated}};
    for (auto& e : tab)
      if (!std::strcmp(e.n, n)) return e.b;
    return nullptr;
  }
};

struct Handle {
  int precision;  // 32 or 64
  Solver<float> s32;
  Solver<double> s64;
};

}  // namespace vfs_oracle

using namespace vfs_oracle;

extern "C" {

void* oracle_create(int precision) {
  Handle* h = new Handle();
  h->precision = precision == 32 ? 32 : 64;
  return h;
}
void oracle_destroy(void* hp) { delete (Handle*)hp; }
void oracle_set_hw_texture(int on) { g_hw_texture = on; }
// OpenMP threads of the calling thread's later solves (n > 0); returns the previous count, so
// that a single-threaded timing can put it back
int oracle_set_threads(int n) {
  const int prev = omp_get_max_threads();
  if (n > 0) omp_set_num_threads(n);
  return prev;
}

int oracle_initialize(void* hp, int width, int height, float beta, float gamma, float alpha0, float alpha1,
                      float timestep_lambda, float lambda, int nLevels, float fScale, int nWarpIters,
                      int nSolverIters, float limitRange, int blockWidth, int strideAlignment) {
  Handle* h = (Handle*)hp;
  if (width <= 0 || height <= 0 || nLevels <= 0 || strideAlignment <= 0 || blockWidth <= 0) return -1;
  Params P{width, height, beta, gamma, alpha0, alpha1, timestep_lambda, lambda, nLevels, fScale, nWarpIters,
           nSolverIters, limitRange, blockWidth, strideAlignment};
  if (h->precision == 32) h->s32.initialize(P);
  else h->s64.initialize(P);
  return 0;
}

#define DISPATCH(expr) \
  do { Handle* h = (Handle*)hp; if (h->precision == 32) { auto& S = h->s32; expr; } else { auto& S = h->s64; expr; } } while (0)

int oracle_set_limit_range(void* hp, float lr) { DISPATCH(S.P.limitRange = lr); return 0; }
int oracle_load_vector_fields(void* hp, const float* tv, const float* cvf) { DISPATCH(S.loadVectorFields(tv, cvf)); return 0; }
int oracle_copy_mask(void* hp, const float* mask) { DISPATCH(S.copyMaskToDevice(mask)); return 0; }
int oracle_copy_images_u8(void* hp, const uint8_t* i0, const uint8_t* i1) { DISPATCH(S.copyImagesToDevice(i0, i1)); return 0; }
int oracle_copy_images_f32(void* hp, const float* i0, const float* i1) { DISPATCH(S.copyImagesToDeviceF32(i0, i1)); return 0; }
int oracle_solve(void* hp, int masked) { DISPATCH(S.solve(masked != 0)); return 0; }
int oracle_convert_kb(void* hp, float fx, float fy, float cx, float cy, float d1, float d2, float d3, float d4,
                      float t1, float t2, float t3) {
  DISPATCH(S.ConvertKB(fx, fy, cx, cy, d1, d2, d3, d4, t1, t2, t3));
  return 0;
}
int oracle_stride(void* hp) { int r = 0; DISPATCH(r = S.stride); return r; }

// Copy buffer `name` (level-0 layout: width x height, `comps` components,
// pitched by the full-resolution stride) into a tight float64 array.
int oracle_get(void* hp, const char* name, int comps, double* out) {
  int rc = 0;
  DISPATCH({
    auto* B = S.named(name);
    if (!B) { rc = -1; break; }
    for (int y = 0; y < S.height; y++)
      for (int x = 0; x < S.width; x++)
        for (int k = 0; k < comps; k++)
          out[((size_t)y * S.width + x) * comps + k] = (double)(*B)[((size_t)y * S.stride + x) * comps + k];
  });
  return rc;
}

// Raw flat copy of a buffer (all stride*height*comps elements).
int oracle_get_raw(void* hp, const char* name, double* out, size_t n) {
  int rc = 0;
  DISPATCH({
    auto* B = S.named(name);
    if (!B || B->size() < n) { rc = -1; break; }
    for (size_t i = 0; i < n; i++) out[i] = (double)(*B)[i];
  });
  return rc;
}

// Texture model entry for tests: sample `n` coordinates of a tight w x h
// texture with `comps` components (float data), linear (1) or point (0).
void oracle_tex_sample(const float* tex, int w, int h, int comps, int linear, const float* xy, int n, float* out) {
  for (int i = 0; i < n; i++)
    for (int k = 0; k < comps; k++) {
      float xn = xy[2 * i], yn = xy[2 * i + 1];
      out[(size_t)i * comps + k] = linear ? tex_linear<float>(tex, comps, k, w, h, w, xn, yn)
                                          : tex_point<float>(tex, comps, k, w, h, w, xn, yn);
    }
}

}  // extern "C"
