// Histogram equalisation of 8-bit images on the device, as cv::equalizeHist
// (OpenCV 4.5, imgproc/src/histogram.cpp), which the reference's SolveStereo
// applies to both input images on the host (dllhook/vfs.cpp:36-37):
//   hist = 256-bin histogram; i = first non-empty bin;
//   if hist[i] == total: every pixel becomes i;
//   else scale = 255 / (total - hist[i]); lut[i] = 0;
//        lut[j] = round_half_even(scale * sum_{i<k<=j} hist[k]) for j > i,
//        saturated to 0..255.
#include "common.cuh"
#include "hist.cuh"

namespace vfs {

// Per-block shared-memory histogram, merged into the global 256-bin histogram.
__global__ void k_hist256(const uint8_t* __restrict__ img, size_t n, unsigned int* __restrict__ hist) {
  __shared__ unsigned int sh[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  size_t stride = (size_t)gridDim.x * blockDim.x;
  // 16 pixels per thread per step through uint4 loads where aligned
  size_t n16 = ((uintptr_t)img % 16 == 0) ? n / 16 : 0;
  const uint4* v = reinterpret_cast<const uint4*>(img);
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n16; k += stride) {
    uint4 q = v[k];
    unsigned int w4[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int t = 0; t < 4; t++) {
      atomicAdd(&sh[w4[t] & 255u], 1u);
      atomicAdd(&sh[(w4[t] >> 8) & 255u], 1u);
      atomicAdd(&sh[(w4[t] >> 16) & 255u], 1u);
      atomicAdd(&sh[w4[t] >> 24], 1u);
    }
  }
  for (size_t k = n16 * 16 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
    atomicAdd(&sh[img[k]], 1u);
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// One warp builds the LUT (exclusive of the prefix below the first non-empty bin).
__global__ void k_equalize_lut(const unsigned int* __restrict__ hist, size_t total, uint8_t* __restrict__ lut) {
  if (threadIdx.x != 0) return;
  int i = 0;
  while (i < 255 && hist[i] == 0) i++;
  if ((size_t)hist[i] == total) {
    for (int j = 0; j < 256; j++) lut[j] = (uint8_t)i;
    return;
  }
  float scale = (256 - 1.f) / (float)(total - hist[i]);
  unsigned int sum = 0;
  for (int j = 0; j <= i; j++) lut[j] = 0;
  for (int j = i + 1; j < 256; j++) {
    sum += hist[j];
    float v = (float)sum * scale;
    int r = __float2int_rn(v);
    lut[j] = (uint8_t)(r < 0 ? 0 : r > 255 ? 255 : r);
  }
}

__global__ void k_apply_lut(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, size_t n,
                            const uint8_t* __restrict__ lut) {
  __shared__ uint8_t sl[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) sl[i] = lut[i];
  __syncthreads();
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    dst[k] = sl[src[k]];
}

void launch_equalize_hist(const uint8_t* src, uint8_t* dst, size_t n, unsigned int* hist_scratch,
                          uint8_t* lut_scratch, cudaStream_t st) {
  if (n == 0) return;
  VFS_CUDA(cudaMemsetAsync(hist_scratch, 0, 256 * sizeof(unsigned int), st));
  int blocks = (int)std::min<size_t>((n + 16 * 256 - 1) / (16 * 256), 296);
  if (blocks < 1) blocks = 1;
  k_hist256<<<blocks, 256, 0, st>>>(src, n, hist_scratch);
  VFS_LAUNCH_CHECK();
  k_equalize_lut<<<1, 32, 0, st>>>(hist_scratch, n, lut_scratch);
  VFS_LAUNCH_CHECK();
  int ab = (int)std::min<size_t>((n + 255) / 256, 1184);
  k_apply_lut<<<ab, 256, 0, st>>>(src, dst, n, lut_scratch);
  VFS_LAUNCH_CHECK();
}

}  // namespace vfs
