// stereotgv.h — drop-in C++ replacement of the reference's StereoTgv class
// (stereotgv/stereotgv.h:14-124) over the vfs_b200 C ABI (vfs_b200.h).
//
// Callers of the reference keep their code: the class name, the constructors, the public
// configuration fields (limitRange, baseline, focal, visualizeResults) and the method names
// and argument orders are the reference's.  Differences:
//   * raw-pointer overloads take tightly packed row-major images / fields (the cv::Mat
//     overloads are compiled only when OpenCV's core header is available);
//   * methods return the library's status (0 = ok, negative = VFS_ERR_*) instead of always 0,
//     and never exit the process (the reference aborts through checkCudaErrors);
//   * cv::Mat& outputs are filled in place by the Mat overloads (the reference hands back
//     ROIs of its internal buffers), and the raw-pointer outputs write to caller memory.
// Link with -lvfs_b200 (vfs_b200/_lib/libvfs_b200.so).
#ifndef VFS_B200_STEREOTGV_H
#define VFS_B200_STEREOTGV_H

#include "vfs_b200.h"

#if defined(__has_include)
#if __has_include(<opencv2/core.hpp>)
#include <opencv2/core.hpp>
#define VFS_B200_HAVE_OPENCV 1
#endif
#endif

class StereoTgv {
 public:
  // stereotgv.cu:32-36
  StereoTgv() { vfs_create(&h_); }
  // stereotgv.cu:38-42
  StereoTgv(int blockWidth, int blockHeight, int strideAlignment) {
    vfs_create_ex(&h_, blockWidth, blockHeight, strideAlignment);
  }
  ~StereoTgv() {
    if (h_) vfs_destroy(h_);
  }
  StereoTgv(const StereoTgv&) = delete;
  StereoTgv& operator=(const StereoTgv&) = delete;

  // public fields of the reference (stereotgv.h:31-45)
  float baseline = 0.0f;
  float focal = 0.0f;
  bool visualizeResults = false;
  float limitRange = 1.0f;
  int width = 0, height = 0;

  // stereotgv.h:107-109
  int initialize(int width_, int height_, float beta, float gamma, float alpha0, float alpha1,
                 float timestep_lambda, float lambda, int nLevels, float fScale, int nWarpIters,
                 int nSolverIters) {
    width = width_;
    height = height_;
    int st = vfs_set_limit_range(h_, limitRange);
    if (st) return st;
    return vfs_initialize(h_, width_, height_, beta, gamma, alpha0, alpha1, timestep_lambda, lambda, nLevels,
                          fScale, nWarpIters, nSolverIters);
  }
  // stereotgv.h:110 (CV_32FC2 fields as H x W x 2 floats)
  int loadVectorFields(const float* translationVector, const float* calibrationVector) {
    return vfs_load_vector_fields(h_, translationVector, calibrationVector);
  }
  // stereotgv.h:112
  int copyImagesToDevice(unsigned char* i0, unsigned char* i1) { return vfs_copy_images_to_device_u8(h_, i0, i1); }
  int copyImagesToDevice(const float* i0, const float* i1) { return vfs_copy_images_to_device_f32(h_, i0, i1); }
  // stereotgv.h:115 (CV_32F mask as H x W floats)
  int copyMaskToDevice(const float* mask) { return vfs_copy_mask_to_device(h_, mask); }
  // stereotgv.h:116-117
  int solveStereoForward() {
    int st = sync_fields();
    return st ? st : vfs_solve_stereo_forward(h_);
  }
  int solveStereoForwardMasked() {
    int st = sync_fields();
    return st ? st : vfs_solve_stereo_forward_masked(h_);
  }
  // stereotgv.h:118-124 (raw-pointer outputs, W x H [x comps] floats)
  int copyStereoToHost(float* depth, float* X, float focalx, float focaly, float cx, float cy, float d1, float d2,
                       float d3, float d4, float t1, float t2, float t3) {
    return vfs_copy_stereo_to_host(h_, depth, X, focalx, focaly, cx, cy, d1, d2, d3, d4, t1, t2, t3);
  }
  int copy1DDisparityToHost(float* u) { return vfs_copy_1d_disparity_to_host(h_, u); }
  int copyDisparityToHost(float* warpUV) { return vfs_copy_disparity_to_host(h_, warpUV); }
  int copyDisparityVisToHost(float* rgb, float flowScale) { return vfs_copy_disparity_vis_to_host(h_, rgb, flowScale); }
  int copyWarpedImageToHost(float* image) { return vfs_copy_warped_image_to_host(h_, image); }

#ifdef VFS_B200_HAVE_OPENCV
  int loadVectorFields(cv::Mat translationVector, cv::Mat calibrationVector) {
    cv::Mat t = translationVector.isContinuous() ? translationVector : translationVector.clone();
    cv::Mat c = calibrationVector.isContinuous() ? calibrationVector : calibrationVector.clone();
    if (t.type() != CV_32FC2 || c.type() != CV_32FC2) return VFS_ERR_ARG;
    return loadVectorFields((const float*)t.ptr(), (const float*)c.ptr());
  }
  int copyImagesToDevice(cv::Mat i0, cv::Mat i1) {
    cv::Mat a = i0.isContinuous() ? i0 : i0.clone(), b = i1.isContinuous() ? i1 : i1.clone();
    if (a.type() == CV_8U) return vfs_copy_images_to_device_u8(h_, a.ptr(), b.ptr());
    if (a.type() == CV_32F) return vfs_copy_images_to_device_f32(h_, (const float*)a.ptr(), (const float*)b.ptr());
    if (a.type() == CV_8UC3) return vfs_copy_images_to_device_u8c3(h_, a.ptr(), b.ptr());
    return VFS_ERR_ARG;
  }
  int copyMaskToDevice(cv::Mat mask) {
    cv::Mat m = mask.isContinuous() ? mask : mask.clone();
    if (m.type() != CV_32F) return VFS_ERR_ARG;
    return copyMaskToDevice((const float*)m.ptr());
  }
  int copyStereoToHost(cv::Mat& depth, cv::Mat& X, float fx, float fy, float cx, float cy, float d1, float d2,
                       float d3, float d4, float t1, float t2, float t3) {
    depth.create(height, width, CV_32F);
    X.create(height, width, CV_32FC3);
    return copyStereoToHost((float*)depth.ptr(), (float*)X.ptr(), fx, fy, cx, cy, d1, d2, d3, d4, t1, t2, t3);
  }
  int copy1DDisparityToHost(cv::Mat& u) {
    u.create(height, width, CV_32F);
    return copy1DDisparityToHost((float*)u.ptr());
  }
  int copyDisparityToHost(cv::Mat& uv) {
    uv.create(height, width, CV_32FC2);
    return copyDisparityToHost((float*)uv.ptr());
  }
  int copyDisparityVisToHost(cv::Mat& rgb, float flowScale) {
    rgb.create(height, width, CV_32FC3);
    return copyDisparityVisToHost((float*)rgb.ptr(), flowScale);
  }
  int copyWarpedImageToHost(cv::Mat& im) {
    im.create(height, width, CV_32F);
    return copyWarpedImageToHost((float*)im.ptr());
  }
#endif

  // additions (no counterpart in the reference)
  vfs_stereo* handle() const { return h_; }
  int setStream(void* cudaStream) { return vfs_set_stream(h_, cudaStream); }
  int setSolvePath(int path, int halfStorage) { return vfs_set_solve_path(h_, path, halfStorage); }
  const char* lastError() const { return vfs_last_error(h_); }

 private:
  int sync_fields() {
    int st = vfs_set_limit_range(h_, limitRange);
    return st ? st : vfs_set_camera(h_, baseline, focal);
  }
  vfs_stereo* h_ = nullptr;
};

#endif  // VFS_B200_STEREOTGV_H
