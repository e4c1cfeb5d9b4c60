// Host-side solver object behind the C ABI (include/vfs_b200.h) and the C++ class
// (include/stereotgv.h).  It owns the device state of one camera pair and runs the
// reference's coarse-to-fine schedule on its CUDA stream.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace vfs {

struct SolverParams {
  int width = 0, height = 0;
  float beta = 0, gamma = 0, alpha0 = 0, alpha1 = 0, timestep_lambda = 0, lambda = 0;
  int nLevels = 0;
  float fScale = 2.0f;
  int nWarpIters = 0, nSolverIters = 0;
  float limitRange = 1.0f;  // stereotgv.h:45
};

// Which implementation runs the solve.
enum class SolvePath {
  kReference = 0,  // one kernel per reference kernel (drop-in form)
  kFused = 1,      // fused kernels with temporal blocking
};

class StereoTgvImpl {
 public:
  StereoTgvImpl(int blockWidth, int blockHeight, int strideAlignment);
  ~StereoTgvImpl();

  void initialize(const SolverParams& p);
  void setStream(cudaStream_t st) { stream_ = st; }
  cudaStream_t stream() const { return stream_; }
  bool initialized() const { return initialized_; }

  void loadVectorFields(const float* tv_host, const float* cv_host);
  void copyMaskToDevice(const float* mask_host);
  void copyImagesU8(const uint8_t* i0, const uint8_t* i1, bool device_src);
  void copyImagesF32(const float* i0, const float* i1);
  void copyImagesU8C3(const uint8_t* i0, const uint8_t* i1);
  void solve(bool masked);
  void copyOut(const char* what, float* dst, bool to_host);
  void convertKB(float fx, float fy, float cx, float cy, float d1, float d2, float d3, float d4, float t1, float t2,
                 float t3);
  void flowToHSV(float flowscale);
  void debugGet(const char* name, int comps, float* out_host);

  SolverParams P;
  float baseline = 0.0f, focal = 0.0f;
  bool visualizeResults = false;
  int blockWidth, blockHeight, strideAlignment;
  int width = 0, height = 0, stride = 0;
  std::vector<int> pW, pH, pS;
  SolvePath path = SolvePath::kReference;
  std::string last_error;

  // ---- device state (names follow stereotgv.h:48-96) ------------------------
  std::vector<float*> pI0, pI1, pMask;
  std::vector<float2*> pTvF;
  float *d_i1calibrated = nullptr, *d_i1warp = nullptr, *d_i0smooth = nullptr, *d_Iu = nullptr, *d_Iz = nullptr;
  float *d_u = nullptr, *d_du = nullptr, *d_us = nullptr;
  float2 *d_warpUV = nullptr, *d_dwarpUV = nullptr, *d_warpUVs = nullptr, *d_tv2 = nullptr, *d_cv = nullptr;
  float *d_a = nullptr, *d_b = nullptr, *d_c = nullptr, *d_etau = nullptr, *d_etav1 = nullptr, *d_etav2 = nullptr;
  float2* d_p = nullptr;
  float4* d_q = nullptr;
  float *d_u_ = nullptr, *d_u_last = nullptr, *d_u_s = nullptr;
  float2 *d_v = nullptr, *d_v_ = nullptr, *d_v_s = nullptr, *d_Tp = nullptr;
  uint8_t *d_i08u = nullptr, *d_i18u = nullptr;
  uchar3 *d_i08uc3 = nullptr, *d_i18uc3 = nullptr;
  float3* d_X = nullptr;
  float* d_depth = nullptr;
  float3* d_uvrgb = nullptr;
  float* d_pack = nullptr;  // tight staging for device-to-host copies

  size_t pool_bytes() const { return pool_bytes_; }
  TexCache tex;

 private:
  void release();
  float* alloc(size_t bytes);
  Geom geom(int level) const { return Geom{pW[level], pH[level], pS[level]}; }
  cudaTextureObject_t t1(const float* p, int level, bool linear = true) {
    return tex.get(p, pW[level], pH[level], (size_t)pS[level] * sizeof(float), 1, linear);
  }
  cudaTextureObject_t t2(const float2* p, int level) {
    return tex.get(p, pW[level], pH[level], (size_t)pS[level] * sizeof(float2), 2, true);
  }
  void solveReference(bool masked);

  bool initialized_ = false;
  cudaStream_t stream_ = 0;
  char* pool_ = nullptr;
  size_t pool_bytes_ = 0, pool_used_ = 0;
  size_t full_ = 0;  // elements of a full-resolution pitched plane
};

}  // namespace vfs
