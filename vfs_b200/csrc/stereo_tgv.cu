// StereoTgvImpl: device state and the coarse-to-fine schedule of the reference
// solver (stereotgv/stereotgv.cu:44-598), on one CUDA stream.
#include <cmath>
#include <cstring>

#include "stereo_tgv.cuh"

#include <atomic>

namespace vfs {

StereoTgvImpl::StereoTgvImpl(int bw, int bh, int sa) : blockWidth(bw), blockHeight(bh), strideAlignment(sa) {}

StereoTgvImpl::~StereoTgvImpl() {
  release();
  for (auto e : evpool_) cudaEventDestroy(e);
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

cudaStream_t StereoTgvImpl::own_stream() {
  if (!own_stream_) VFS_CUDA(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
  return own_stream_;
}

std::atomic<long long>& launch_counter() {
  static std::atomic<long long> n{0};
  return n;
}

const char* level_range_name(int level) {
  static const char* names[16] = {"level 0",  "level 1",  "level 2",  "level 3", "level 4",  "level 5",
                                  "level 6",  "level 7",  "level 8",  "level 9", "level 10", "level 11",
                                  "level 12", "level 13", "level 14", "level 15"};
  return names[level < 0 ? 0 : level > 15 ? 15 : level];
}

uint64_t next_generation() {
  static std::atomic<uint64_t> gen{0};
  return ++gen;
}

std::atomic<bool>& pdl_enabled() {
  static std::atomic<bool> on{true};
  return on;
}

int& launch_priority() {
  static thread_local int p = 0;
  return p;
}

cudaEvent_t StereoTgvImpl::profEvent() {
  if (capture_events) {
    cudaEvent_t e;
    VFS_CUDA(cudaEventCreate(&e));
    capture_events->push_back(e);
    return e;
  }
  if (evused_ == evpool_.size()) {
    cudaEvent_t e;
    VFS_CUDA(cudaEventCreate(&e));
    evpool_.push_back(e);
  }
  return evpool_[evused_++];
}

static void record(cudaEvent_t e, cudaStream_t st, bool external) {
  if (external) VFS_CUDA(cudaEventRecordWithFlags(e, st, cudaEventRecordExternal));
  else VFS_CUDA(cudaEventRecord(e, st));
}

void StereoTgvImpl::profBegin(int tag, int level, int iters) {
  profBeginPx(tag, (long long)pW[level] * pH[level], iters);
}

void StereoTgvImpl::profBeginPx(int tag, long long px, int iters, cudaStream_t st, int launches) {
  if (!profiling) return;
  ProfRec r{tag, 0, px, iters, profEvent(), profEvent(), launches > 0 ? launches : iters};
  record(r.a, st ? st : stream_, capture_events != nullptr);
  prof_.push_back(r);
}

void StereoTgvImpl::profEnd(cudaStream_t st) {
  if (!profiling || prof_.empty()) return;
  record(prof_.back().b, st ? st : stream_, capture_events != nullptr);
}

void StereoTgvImpl::profReset() {
  prof_.clear();
  evused_ = 0;
}

void StereoTgvImpl::profRead(int tag, long long* count, double* total_ms, double* pixel_iters) {
  VFS_CUDA(cudaStreamSynchronize(stream_));
  for (auto& r : prof_) VFS_CUDA(cudaEventSynchronize(r.b));  // records may sit on other streams
  long long n = 0;
  double t = 0, pi = 0;
  for (auto& r : prof_) {
    if (r.tag != tag) continue;
    float ms = 0;
    VFS_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
    n++;
    t += ms;
    pi += (double)r.px * r.iters;
  }
  if (count) *count = n;
  if (total_ms) *total_ms = t;
  if (pixel_iters) *pixel_iters = pi;
}

// Test hook (vfs_debug_fail_allocation): when n > 0, the n-th following device-pool allocation
// of any handle fails as if the device were out of memory.
std::atomic<int>& alloc_failure_countdown() {
  static std::atomic<int> n{0};
  return n;
}

static cudaError_t pool_malloc(void** p, size_t bytes) {
  int n = alloc_failure_countdown().load();
  while (n > 0 && !alloc_failure_countdown().compare_exchange_weak(n, n - 1)) {
  }
  if (n == 1) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

void StereoTgvImpl::release() {
  engine.clear();
  tex.clear();
  if (pool_) cudaFree(pool_);
  pool_ = nullptr;
  if (fpool_) cudaFree(fpool_);
  fpool_ = nullptr;
  f_p = f_q = f_vh = f_vhs = nullptr;
  f_abce = nullptr;
  f_rv = nullptr;
  code_masked.clear();
  code_plain.clear();
  codes_valid = false;
  pool_bytes_ = pool_used_ = 0;
  guards_.clear();
  initialized_ = false;
}

float* StereoTgvImpl::alloc(size_t bytes) {
  size_t off = (pool_used_ + 511) & ~(size_t)511;  // texture base alignment
  if (off + bytes + kGuardBytes > pool_bytes_) throw ArgError{"internal: device pool overflow"};
  pool_used_ = off + bytes + kGuardBytes;
  guards_.push_back(pool_ + off + bytes);
  return (float*)(pool_ + off);
}

void StereoTgvImpl::fillGuards(size_t from, cudaStream_t st) {
  for (size_t k = from; k < guards_.size(); k++) VFS_CUDA(cudaMemsetAsync(guards_[k], kGuardByte, kGuardBytes, st));
}

int StereoTgvImpl::checkGuards() {
  if (guards_.empty()) return 0;
  VFS_CUDA(cudaStreamSynchronize(stream_));
  std::vector<unsigned char> h(kGuardBytes);
  int bad = 0;
  for (char* g : guards_) {
    VFS_CUDA(cudaMemcpy(h.data(), g, kGuardBytes, cudaMemcpyDeviceToHost));
    for (unsigned char c : h)
      if (c != kGuardByte) {
        bad++;
        break;
      }
  }
  return bad;
}

static int align_up(int n, int m) {
  int mod = n % m;
  return mod ? n + m - mod : n;
}

// pool: pyramid (5 planes/level: I0, I1, mask, tv x2); full-resolution planes:
// 18 float, 10 float2, 1 float4, 2 float3, 1 four-plane staging; u8 and uchar3
// image staging; 512 B alignment slack per buffer.
static size_t pool_bytes_for(const std::vector<int>& pS, const std::vector<int>& pH, size_t full) {
  size_t bytes = 0;
  for (size_t l = 0; l < pS.size(); l++)
    bytes += (size_t)pS[l] * pH[l] * sizeof(float) * 5 + 4 * 512 + 4 * StereoTgvImpl::kGuardBytes;
  const size_t planes = 18 + 10 * 2 + 4 + 2 * 3 + 4;
  return bytes + full * sizeof(float) * planes + full * (2 + 2 * 3) + 64 * 512 + 40 * StereoTgvImpl::kGuardBytes;
}

// p, q two planes each (float: 8 + 16 bytes per pixel and plane), half v-bar pair, and
// two edge-code bytes per pixel and level.
static size_t fused_bytes_for(const std::vector<int>& pS, const std::vector<int>& pH, size_t full) {
  size_t bytes = full * 2 * 8 + full * 2 * 16 + full * 4 * 2 + full * 16 + full * 8 + 8 * 512 +
                 8 * StereoTgvImpl::kGuardBytes;
  for (size_t l = 0; l < pS.size(); l++) bytes += 2 * ((size_t)pS[l] * pH[l] + 512 + StereoTgvImpl::kGuardBytes);
  return bytes;
}

size_t estimate_device_bytes(int width, int height, int nLevels, float fScale, int sa, bool fused) {
  if (width <= 0 || height <= 0 || nLevels <= 0 || sa <= 0 || !(fScale > 0.0f)) return 0;
  std::vector<int> pS, pH;
  int nh = height, nw = width;
  for (int l = 0; l < nLevels; l++) {
    if (nw <= 0 || nh <= 0) return 0;
    pS.push_back(align_up(nw, sa));
    pH.push_back(nh);
    nh = (int)((float)nh / fScale);
    nw = (int)((float)nw / fScale);
  }
  size_t full = (size_t)pS[0] * pH[0];
  if (full * 8 >= ((size_t)1 << 31)) return 0;  // initialize refuses this geometry
  return pool_bytes_for(pS, pH, full) + (fused ? fused_bytes_for(pS, pH, full) : 0);
}

// stereotgv.cu:44-168
void StereoTgvImpl::initialize(const SolverParams& p) {
  if (p.width <= 0 || p.height <= 0 || p.nLevels <= 0 || p.nWarpIters < 0 || p.nSolverIters < 0 ||
      !(p.fScale > 0.0f))
    throw ArgError{"initialize: invalid size or iteration count"};
  if (strideAlignment <= 0 || blockWidth <= 0 || blockHeight <= 0)
    throw ArgError{"initialize: invalid block or stride alignment"};
  have_prev = false;
  release();
  if (!stream_) stream_ = own_stream();
  generation = next_generation();
  P = p;
  width = p.width;
  height = p.height;
  stride = align_up(width, strideAlignment);
  int pitchAlign = 0;
  int dev = 0;
  VFS_CUDA(cudaGetDevice(&dev));
  VFS_CUDA(cudaDeviceGetAttribute(&pitchAlign, cudaDevAttrTexturePitchAlignment, dev));
  pW.assign(p.nLevels, 0);
  pH.assign(p.nLevels, 0);
  pS.assign(p.nLevels, 0);
  int nh = height, nw = width, ns = stride;
  for (int l = 0; l < p.nLevels; l++) {
    if (nw <= 0 || nh <= 0) throw ArgError{"initialize: pyramid level " + std::to_string(l) + " has zero size"};
    if (((size_t)ns * sizeof(float)) % (size_t)pitchAlign != 0)
      throw ArgError{"initialize: row pitch is not a multiple of the texture pitch alignment"};
    pW[l] = nw;
    pH[l] = nh;
    pS[l] = ns;
    nh = (int)((float)nh / p.fScale);
    nw = (int)((float)nw / p.fScale);
    ns = align_up(nw, strideAlignment);
  }
  full_ = (size_t)stride * height;
  if (full_ * 8 >= ((size_t)1 << 31))
    throw ArgError{"initialize: image too large (row pitch x height x 8 must stay below 2^31)"};
  size_t f = full_ * sizeof(float);
  pool_bytes_ = pool_bytes_for(pS, pH, full_);
  cudaError_t e = pool_malloc((void**)&pool_, pool_bytes_);
  if (e != cudaSuccess) {
    pool_ = nullptr;
    (void)cudaGetLastError();
    throw CudaError{e, "cudaMalloc(solver pool)", __FILE__, __LINE__};
  }
  pool_used_ = 0;
  pI0.assign(p.nLevels, nullptr);
  pI1.assign(p.nLevels, nullptr);
  pMask.assign(p.nLevels, nullptr);
  pTvF.assign(p.nLevels, nullptr);
  for (int l = 0; l < p.nLevels; l++) {
    size_t n = (size_t)pS[l] * pH[l] * sizeof(float);
    pI0[l] = alloc(n);
    pI1[l] = alloc(n);
    pMask[l] = alloc(n);
    pTvF[l] = (float2*)alloc(2 * n);
  }
  d_i1calibrated = alloc(f);
  d_i1warp = alloc(f);
  d_i0smooth = alloc(f);
  d_Iu = alloc(f);
  d_Iz = alloc(f);
  d_u = alloc(f);
  d_du = alloc(f);
  d_us = alloc(f);
  d_a = alloc(f);
  d_b = alloc(f);
  d_c = alloc(f);
  d_etau = alloc(f);
  d_etav1 = alloc(f);
  d_etav2 = alloc(f);
  d_u_ = alloc(f);
  d_u_last = alloc(f);
  d_u_s = alloc(f);
  d_depth = alloc(f);
  d_warpUV = (float2*)alloc(2 * f);
  d_dwarpUV = (float2*)alloc(2 * f);
  d_warpUVs = (float2*)alloc(2 * f);
  d_tv2 = (float2*)alloc(2 * f);
  d_cv = (float2*)alloc(2 * f);
  d_p = (float2*)alloc(2 * f);
  d_v = (float2*)alloc(2 * f);
  d_v_ = (float2*)alloc(2 * f);
  d_v_s = (float2*)alloc(2 * f);
  d_Tp = (float2*)alloc(2 * f);
  d_q = (float4*)alloc(4 * f);
  d_X = (float3*)alloc(3 * f);
  d_uvrgb = (float3*)alloc(3 * f);
  d_i08u = (uint8_t*)alloc(full_);
  d_i18u = (uint8_t*)alloc(full_);
  d_i08uc3 = (uchar3*)alloc(3 * full_);
  d_i18uc3 = (uchar3*)alloc(3 * full_);
  d_pack = alloc(4 * f);
  // The reference leaves its buffers uninitialised after cudaMalloc; this
  // implementation starts from all-zero state so that results are deterministic.
  VFS_CUDA(cudaMemsetAsync(pool_, 0, pool_bytes_, stream_));
  fillGuards(0, stream_);
  VFS_CUDA(cudaStreamSynchronize(stream_));
  initialized_ = true;
}

// stereotgv.cu:171-199.  The reference also builds a negated copy of the field
// (pTvBackward) that the solver never reads; it is not kept here.
void StereoTgvImpl::loadVectorFields(const float* tv, const float* cvf) {
  have_prev = false;  // a warm start follows the fields it was solved with
  if (!initialized_) throw ArgError{"loadVectorFields before initialize"};
  if (!tv || !cvf) throw ArgError{"loadVectorFields: null field"};
  size_t row = (size_t)width * sizeof(float2);
  VFS_CUDA(cudaMemsetAsync(pTvF[0], 0, full_ * sizeof(float2), stream_));
  VFS_CUDA(cudaMemsetAsync(d_cv, 0, full_ * sizeof(float2), stream_));
  VFS_CUDA(cudaMemcpy2DAsync(pTvF[0], (size_t)stride * sizeof(float2), tv, row, row, height, cudaMemcpyHostToDevice,
                             stream_));
  VFS_CUDA(cudaMemcpy2DAsync(d_cv, (size_t)stride * sizeof(float2), cvf, row, row, height, cudaMemcpyHostToDevice,
                             stream_));
  for (int l = 1; l < P.nLevels; l++) launch_downscale(t2(pTvF[l - 1], l - 1), 2, (float*)pTvF[l], geom(l), stream_);
  VFS_CUDA(cudaStreamSynchronize(stream_));
}

// stereotgv.cu:241-252
void StereoTgvImpl::copyMaskToDevice(const float* mask) {
  if (!initialized_) throw ArgError{"copyMaskToDevice before initialize"};
  if (!mask) throw ArgError{"copyMaskToDevice: null mask"};
  size_t row = (size_t)width * sizeof(float);
  VFS_CUDA(cudaMemsetAsync(pMask[0], 0, full_ * sizeof(float), stream_));
  VFS_CUDA(cudaMemcpy2DAsync(pMask[0], (size_t)stride * sizeof(float), mask, row, row, height, cudaMemcpyHostToDevice,
                             stream_));
  for (int l = 1; l < P.nLevels; l++) launch_downscale_nearest(t1(pMask[l - 1], l - 1, false), pMask[l], geom(l), stream_);
  codes_valid = false;
  VFS_CUDA(cudaStreamSynchronize(stream_));
}

// stereotgv.cu:201-213 (u8) and 215-239 (f32, u8c3)
void StereoTgvImpl::copyImagesU8(const uint8_t* i0, const uint8_t* i1, bool device_src) {
  copyImagesU8On(i0, i1, device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream_);
  if (!device_src) VFS_CUDA(cudaStreamSynchronize(stream_));
}

void StereoTgvImpl::copyImagesU8On(const uint8_t* i0, const uint8_t* i1, cudaMemcpyKind kind, cudaStream_t st) {
  if (!initialized_) throw ArgError{"copyImagesToDevice before initialize"};
  if (!i0 || !i1) throw ArgError{"copyImagesToDevice: null image"};
  // one contiguous copy per image into the staging buffers (tight rows), then one kernel
  // converts both into the pitched planes
  const size_t n = (size_t)width * height;
  VFS_CUDA(cudaMemcpyAsync(d_i08u, i0, n, kind, st));
  VFS_CUDA(cudaMemcpyAsync(d_i18u, i1, n, kind, st));
  launch_cv8u_tight_to_gray2(d_i08u, d_i18u, pI0[0], pI1[0], geom(0), st);
}

void StereoTgvImpl::copyImagesF32(const float* i0, const float* i1) {
  if (!initialized_) throw ArgError{"copyImagesToDevice before initialize"};
  if (!i0 || !i1) throw ArgError{"copyImagesToDevice: null image"};
  size_t row = (size_t)width * sizeof(float);
  VFS_CUDA(cudaMemcpy2DAsync(pI0[0], (size_t)stride * sizeof(float), i0, row, row, height, cudaMemcpyHostToDevice,
                             stream_));
  VFS_CUDA(cudaMemcpy2DAsync(pI1[0], (size_t)stride * sizeof(float), i1, row, row, height, cudaMemcpyHostToDevice,
                             stream_));
  VFS_CUDA(cudaStreamSynchronize(stream_));
}

void StereoTgvImpl::copyImagesU8C3(const uint8_t* i0, const uint8_t* i1) {
  if (!initialized_) throw ArgError{"copyImagesToDevice before initialize"};
  if (!i0 || !i1) throw ArgError{"copyImagesToDevice: null image"};
  size_t row = (size_t)width * 3;
  VFS_CUDA(cudaMemcpy2DAsync(d_i08uc3, (size_t)stride * 3, i0, row, row, height, cudaMemcpyHostToDevice, stream_));
  VFS_CUDA(cudaMemcpy2DAsync(d_i18uc3, (size_t)stride * 3, i1, row, row, height, cudaMemcpyHostToDevice, stream_));
  launch_cv8uc3_to_gray(d_i08uc3, pI0[0], geom(0), stream_);
  launch_cv8uc3_to_gray(d_i18uc3, pI1[0], geom(0), stream_);
  VFS_CUDA(cudaStreamSynchronize(stream_));
}

void StereoTgvImpl::solve(bool masked) {
  if (!initialized_) throw ArgError{"solve before initialize"};
  if (path == SolvePath::kFused) {
    std::vector<StereoTgvImpl*> one{this};
    engine.solve(one, masked, half_storage, stream_);
  } else {
    solveReference(masked);
    have_prev = true;
  }
}

void StereoTgvImpl::startState(int top, cudaStream_t st) {
  const size_t f = full_ * sizeof(float);
  if (!(warm_level >= 0 && have_prev)) {  // stereotgv.cu:395-397
    VFS_CUDA(cudaMemsetAsync(d_u, 0, f, st));
    VFS_CUDA(cudaMemsetAsync(d_u_, 0, f, st));
    VFS_CUDA(cudaMemsetAsync(d_warpUV, 0, 2 * f, st));
    return;
  }
  for (int l = 1; l <= top; l++) {
    launch_downscale_scaled(t1(d_u, l - 1), d_us, 1.0f / P.fScale, geom(l), st);
    std::swap(d_u, d_us);
  }
  launch_clone(d_u_, d_u, geom(top), st);
  VFS_CUDA(cudaMemsetAsync(d_warpUV, 0, 2 * f, st));
}

// Fused-path buffers: p and q in two planes each (float: 8 + 16 bytes per pixel per
// plane; half: 4 + 8), half v-bar ping-pong pair (4 + 4), and per-level edge codes.
void StereoTgvImpl::ensureFused() {
  if (fpool_) return;
  size_t n = full_;
  size_t bytes = fused_bytes_for(pS, pH, full_);
  cudaError_t e = pool_malloc((void**)&fpool_, bytes);
  if (e != cudaSuccess) {
    fpool_ = nullptr;
    (void)cudaGetLastError();
    throw CudaError{e, "cudaMalloc(fused buffers)", __FILE__, __LINE__};
  }
  size_t off = 0;
  const size_t guards_before = guards_.size();
  auto take = [&](size_t b) {
    off = (off + 511) & ~(size_t)511;
    if (off + b + kGuardBytes > bytes) throw ArgError{"internal: fused pool overflow"};
    char* p = fpool_ + off;
    off += b;
    guards_.push_back(fpool_ + off);
    off += kGuardBytes;
    return p;
  };
  f_p = take(n * 2 * 8);
  f_q = take(n * 2 * 16);
  f_vh = take(n * 4);
  f_vhs = take(n * 4);
  f_abce = (float4*)take(n * 16);
  f_rv = (float2*)take(n * 8);
  code_masked.assign(levels(), nullptr);
  code_plain.assign(levels(), nullptr);
  for (int l = 0; l < levels(); l++) {
    code_masked[l] = (uint8_t*)take((size_t)pS[l] * pH[l]);
    code_plain[l] = (uint8_t*)take((size_t)pS[l] * pH[l]);
  }
  VFS_CUDA(cudaMemsetAsync(fpool_, 0, bytes, stream_));
  fillGuards(guards_before, stream_);
  for (int l = 0; l < levels(); l++) launch_edge_codes(nullptr, code_plain[l], pW[l], pH[l], pS[l], stream_);
  codes_valid = false;
}

// stereotgv.cu:389-515 (masked) and 256-387 (plain).  Pointer swaps are the
// reference's Swap() calls; the plain form skips the median filter like the
// reference (stereotgv.cu:350-351 is commented out).
void StereoTgvImpl::solveReference(bool masked) {
  cudaStream_t st = stream_;
  i1warp_half = false;
  const size_t f = full_ * sizeof(float);
  launch_warp_image(t1(pI1[0], 0), d_cv, d_i1calibrated, geom(0), st);
  std::swap(pI1[0], d_i1calibrated);
  const int top = topLevel();
  startState(top, st);
  for (int l = 1; l < P.nLevels; l++) {
    launch_downscale(t1(pI0[l - 1], l - 1), 1, pI0[l], geom(l), st);
    launch_downscale(t1(pI1[l - 1], l - 1), 1, pI1[l], geom(l), st);
  }
  for (int level = top; level >= 0; level--) {
    TraceRange trace(level_range_name(level));
    Geom g = geom(level);
    const float* mk = masked ? pMask[level] : nullptr;
    for (float* b : {d_a, d_b, d_c, d_etau, d_etav1, d_etav2, d_i0smooth}) VFS_CUDA(cudaMemsetAsync(b, 0, f, st));
    const float eta_p = 3.0f, eta_q = 2.0f;
    if (level == top) launch_optical_flow_vector(d_u, pTvF[level], d_warpUV, g, st);
    launch_gaussian(t1(pI0[level], level), mk, d_i0smooth, g, st);
    int xcov = ((g.h + blockWidth - 1) / blockWidth) * blockWidth;  // calcTensor.cu:81,227
    launch_calc_tensor(t1(d_i0smooth, level), mk, P.beta, P.gamma, d_a, d_b, d_c, g, std::min(g.w, xcov),
                       tensor_cuda_math, st);
    launch_solve_eta(mk, P.alpha0, P.alpha1, d_a, d_b, d_c, d_etau, d_etav1, d_etav2, g, st);
    for (int warpIter = 0; warpIter < P.nWarpIters; warpIter++) {
      VFS_CUDA(cudaMemsetAsync(d_p, 0, 2 * f, st));
      VFS_CUDA(cudaMemsetAsync(d_q, 0, 4 * f, st));
      VFS_CUDA(cudaMemsetAsync(d_v, 0, 2 * f, st));
      launch_clone2(d_v_, d_v, g, st);
      VFS_CUDA(cudaMemsetAsync(d_du, 0, f, st));
      launch_find_warping_vector(t2(pTvF[level], level), d_warpUV, d_tv2, g, st);
      launch_warp_image(t1(pI1[level], level), d_warpUV, d_i1warp, g, st);
      launch_derivatives_fisheye(t1(pI0[level], level), t1(d_i1warp, level), pTvF[level], d_Iu, d_Iz, g, st);
      launch_clone(d_u_last, d_u, g, st);
      // host step schedule in float (stereotgv.cu:449-456, 476-477)
      float tau = 1.0f;
      float sigma = 1.0f / tau;
      for (int iter = 0; iter < P.nSolverIters; iter++) {
        float mu;
        if (sigma < 1000.0f) mu = 1.0f / std::sqrt(1 + 0.7f * tau * P.timestep_lambda);
        else mu = 1;
        profBegin(kProfInner, level, 1);
        DualArgs da{mk, d_u_, d_v_, d_a, d_b, d_c, d_p, d_q, P.alpha0, P.alpha1, sigma, eta_p, eta_q};
        launch_update_dual(da, g, st);
        launch_solve_tp(mk, d_a, d_b, d_c, d_p, d_Tp, g, st);
        ThreshArgs ta{mk, d_Tp, d_u_, d_Iu, d_Iz, d_etau, d_u, d_us, P.lambda, tau};
        launch_thresholding(ta, g, st);
        std::swap(d_u, d_us);
        PrimalArgs pa{mk, d_u_, d_v_, d_p, d_q, d_a, d_b, d_c, d_etav1, d_etav2, d_u, d_v, d_u_s, d_v_s,
                      tau, P.alpha0, P.alpha1, mu};
        launch_update_primal(pa, g, st);
        profEnd();
        std::swap(d_u_, d_u_s);
        std::swap(d_v_, d_v_s);
        sigma = sigma / mu;
        tau = tau * mu;
      }
      if (masked) {
        launch_median5(d_u, d_us, g, st);
        std::swap(d_u, d_us);
      }
      launch_warp_epilogue(d_u, d_u_last, d_du, d_u_, d_tv2, d_dwarpUV, d_warpUV, P.limitRange, g, st);
    }
    if (level > 0) {
      Geom gf = geom(level - 1);
      float scale = P.fScale;
      launch_upscale(t1(d_u, level), 1, d_us, scale, gf, st);
      launch_upscale(t1(d_u_, level), 1, d_u_s, scale, gf, st);
      launch_upscale(t2(d_warpUV, level), 2, (float*)d_warpUVs, scale, gf, st);
      std::swap(d_u, d_us);
      std::swap(d_u_, d_u_s);
      std::swap(d_warpUV, d_warpUVs);
    }
  }
}

// ---- state export / import ----------------------------------------------------------
namespace {
constexpr uint32_t kStateMagic = 0x53534656u;  // "VFSS"
constexpr uint32_t kStateVersion = 1;
constexpr int kStateRoles = 12;
struct StateHeader {
  uint32_t magic, version;
  int32_t width, height, stride, levels, stride_alignment, has_fused;
  float fScale;
  int32_t f_parity, have_prev, i1warp_half;
  uint64_t pool_bytes, fpool_bytes;
  int64_t role[kStateRoles];  // byte offsets in their pool (the last two: the fused pool); -1 = null
};
}  // namespace

size_t StereoTgvImpl::stateBytes() const {
  if (!initialized_) return 0;
  return sizeof(StateHeader) + pool_bytes_ + (fpool_ ? fused_bytes_for(pS, pH, full_) : 0);
}

void StereoTgvImpl::exportState(void* host, size_t bytes) {
  if (!initialized_) throw ArgError{"export_state before initialize"};
  if (!host) throw ArgError{"export_state: null buffer"};
  const size_t need = stateBytes();
  if (bytes < need) throw ArgError{"export_state: buffer smaller than vfs_state_bytes"};
  const size_t fbytes = fpool_ ? fused_bytes_for(pS, pH, full_) : 0;
  StateHeader h{};
  h.magic = kStateMagic;
  h.version = kStateVersion;
  h.width = width;
  h.height = height;
  h.stride = stride;
  h.levels = levels();
  h.stride_alignment = strideAlignment;
  h.has_fused = fpool_ ? 1 : 0;
  h.fScale = P.fScale;
  h.f_parity = f_parity;
  h.have_prev = have_prev ? 1 : 0;
  h.i1warp_half = i1warp_half ? 1 : 0;
  h.pool_bytes = pool_bytes_;
  h.fpool_bytes = fbytes;
  const void* roles[kStateRoles] = {pI1[0], d_i1calibrated, d_u, d_us, d_u_, d_u_s,
                                    d_v_, d_v_s, d_warpUV, d_warpUVs, f_vh, f_vhs};
  for (int k = 0; k < kStateRoles; k++) {
    const char* base = k < 10 ? pool_ : fpool_;
    h.role[k] = roles[k] ? (int64_t)((const char*)roles[k] - base) : -1;
  }
  VFS_CUDA(cudaStreamSynchronize(stream_));
  char* out = (char*)host;
  std::memcpy(out, &h, sizeof(h));
  VFS_CUDA(cudaMemcpy(out + sizeof(h), pool_, pool_bytes_, cudaMemcpyDeviceToHost));
  if (fbytes) VFS_CUDA(cudaMemcpy(out + sizeof(h) + pool_bytes_, fpool_, fbytes, cudaMemcpyDeviceToHost));
}

void StereoTgvImpl::importState(const void* host, size_t bytes) {
  if (!initialized_) throw ArgError{"import_state before initialize"};
  if (!host || bytes < sizeof(StateHeader)) throw ArgError{"import_state: no state"};
  StateHeader h;
  std::memcpy(&h, host, sizeof(h));
  if (h.magic != kStateMagic || h.version != kStateVersion) throw ArgError{"import_state: not a vfs_b200 state"};
  if (h.width != width || h.height != height || h.stride != stride || h.levels != levels() ||
      h.stride_alignment != strideAlignment || h.fScale != P.fScale || h.pool_bytes != pool_bytes_)
    throw ArgError{"import_state: the handle's geometry differs from the exported one"};
  const size_t fbytes = fused_bytes_for(pS, pH, full_);
  if (bytes != sizeof(h) + h.pool_bytes + h.fpool_bytes || (h.has_fused && h.fpool_bytes != fbytes))
    throw ArgError{"import_state: size mismatch"};
  for (int k = 0; k < kStateRoles; k++) {
    const uint64_t lim = k < 10 ? h.pool_bytes : h.fpool_bytes;
    if (h.role[k] < -1 || (h.role[k] >= 0 && (uint64_t)h.role[k] >= lim))
      throw ArgError{"import_state: corrupt buffer roles"};
  }
  if (h.has_fused) ensureFused();
  VFS_CUDA(cudaStreamSynchronize(stream_));
  const char* in = (const char*)host + sizeof(h);
  VFS_CUDA(cudaMemcpy(pool_, in, pool_bytes_, cudaMemcpyHostToDevice));
  if (h.has_fused) VFS_CUDA(cudaMemcpy(fpool_, in + pool_bytes_, fbytes, cudaMemcpyHostToDevice));
  auto at = [&](int k) -> void* {
    if (h.role[k] < 0) return nullptr;
    return (k < 10 ? pool_ : fpool_) + h.role[k];
  };
  pI1[0] = (float*)at(0);
  d_i1calibrated = (float*)at(1);
  d_u = (float*)at(2);
  d_us = (float*)at(3);
  d_u_ = (float*)at(4);
  d_u_s = (float*)at(5);
  d_v_ = (float2*)at(6);
  d_v_s = (float2*)at(7);
  d_warpUV = (float2*)at(8);
  d_warpUVs = (float2*)at(9);
  if (h.has_fused) {
    f_vh = at(10);
    f_vhs = at(11);
  }
  f_parity = h.f_parity;
  have_prev = h.have_prev != 0;
  i1warp_half = h.i1warp_half != 0;
  codes_valid = false;  // the masked edge codes and tile spans are derived again from the mask
  generation = next_generation();
}

// stereotgv.cu:517-568 outputs: level-0 views of u, warpUV, the warped image.
void StereoTgvImpl::copyOut(const char* what, float* dst, bool to_host) {
  copyOutOn(what, dst, to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, stream_);
  if (to_host) VFS_CUDA(cudaStreamSynchronize(stream_));
}

void StereoTgvImpl::copyOutOn(const char* what, float* dst, cudaMemcpyKind kind, cudaStream_t st) {
  if (!initialized_) throw ArgError{"copy before initialize"};
  if (!dst) throw ArgError{"copy: null destination"};
  const void* src = nullptr;
  int comps = 1;
  if (!std::strcmp(what, "u")) src = d_u;
  else if (!std::strcmp(what, "warpUV")) { src = d_warpUV; comps = 2; }
  else if (!std::strcmp(what, "i1warp")) src = d_i1warp;
  else if (!std::strcmp(what, "depth")) src = d_depth;
  else if (!std::strcmp(what, "X")) { src = d_X; comps = 3; }
  else if (!std::strcmp(what, "rgb")) { src = d_uvrgb; comps = 3; }
  else throw ArgError{std::string("copy: unknown buffer ") + what};
  if (src == d_i1warp && i1warp_half) {
    // the FP16 form's warped image: widened to float on the device, tight rows either way
    float* out = kind == cudaMemcpyDeviceToHost ? d_pack : dst;
    launch_pack_tight_half(src, out, geom(0), st);
    if (kind == cudaMemcpyDeviceToHost)
      VFS_CUDA(cudaMemcpyAsync(dst, d_pack, (size_t)width * height * sizeof(float), kind, st));
    return;
  }
  if (kind == cudaMemcpyDeviceToHost) {
    // pack on the device, then one contiguous download
    launch_pack_tight((const float*)src, d_pack, comps, geom(0), st);
    VFS_CUDA(cudaMemcpyAsync(dst, d_pack, (size_t)width * height * comps * sizeof(float), kind, st));
    return;
  }
  size_t row = (size_t)width * comps * sizeof(float);
  VFS_CUDA(cudaMemcpy2DAsync(dst, row, src, (size_t)stride * comps * sizeof(float), row, height, kind, st));
}

void StereoTgvImpl::convertKB(float fx, float fy, float cx, float cy, float d1, float d2, float d3, float d4, float t1_,
                              float t2_, float t3_) {
  if (!initialized_) throw ArgError{"copyStereoToHost before initialize"};
  launch_convert_kb(d_warpUV, fx, fy, cx, cy, d1, d2, d3, d4, t1_, t2_, t3_, d_X, d_depth, geom(0), stream_);
}

void StereoTgvImpl::flowToHSV(float flowscale) {
  if (!initialized_) throw ArgError{"copyDisparityVisToHost before initialize"};
  launch_flow_to_hsv(d_warpUV, d_uvrgb, flowscale, geom(0), stream_);
}

void StereoTgvImpl::debugGet(const char* name, int comps, float* out) {
  if (!initialized_) throw ArgError{"debug get before initialize"};
  struct E {
    const char* n;
    const void* p;
    int c;
  } tab[] = {{"u", d_u, 1},          {"u_", d_u_, 1},         {"warpUV", d_warpUV, 2}, {"a", d_a, 1},
             {"b", d_b, 1},          {"c", d_c, 1},           {"etau", d_etau, 1},     {"etav1", d_etav1, 1},
             {"etav2", d_etav2, 1},  {"Iu", d_Iu, 1},         {"Iz", d_Iz, 1},         {"i1warp", d_i1warp, 1},
             {"tv2", d_tv2, 2},      {"i0smooth", d_i0smooth, 1}, {"p", d_p, 2},       {"q", d_q, 4},
             {"v_", d_v_, 2},        {"Tp", d_Tp, 2},         {"us", d_us, 1},         {"u_s", d_u_s, 1},
             {"v_s", d_v_s, 2},      {"du", d_du, 1},         {"u_last", d_u_last, 1}, {"X", d_X, 3},
             {"depth", d_depth, 1},  {"warpUVs", d_warpUVs, 2}, {"i1calibrated", d_i1calibrated, 1}};
  if (!std::strcmp(name, "i1warp") && i1warp_half) {  // half values: widened by copyOut
    if (comps != 1) throw ArgError{"debug get: component count mismatch"};
    copyOut("i1warp", out, true);
    return;
  }
  for (auto& e : tab) {
    if (std::strcmp(e.n, name)) continue;
    if (comps != e.c) throw ArgError{"debug get: component count mismatch"};
    size_t row = (size_t)width * comps * sizeof(float);
    VFS_CUDA(cudaMemcpy2DAsync(out, row, e.p, (size_t)stride * comps * sizeof(float), row, height,
                               cudaMemcpyDeviceToHost, stream_));
    VFS_CUDA(cudaStreamSynchronize(stream_));
    return;
  }
  throw ArgError{std::string("debug get: unknown buffer ") + name};
}

}  // namespace vfs
