// Histogram equalisation of 8-bit images on the device, as cv::equalizeHist
// (OpenCV 4.5, imgproc/src/histogram.cpp), which the reference's SolveStereo
// applies to both input images on the host (dllhook/vfs.cpp:36-37):
//   hist = 256-bin histogram; i = first non-empty bin;
//   if hist[i] == total: every pixel becomes i;
//   else scale = 255 / (total - hist[i]); lut[i] = 0;
//        lut[j] = round_half_even(scale * sum_{i<k<=j} hist[k]) for j > i,
//        saturated to 0..255.
#include <mutex>

#include "../../include/vfs_b200.h"
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

// src and dst may be the same buffer (in-place equalisation): each thread reads its element
// before writing it, and the pointers are deliberately not __restrict__.
__global__ void k_apply_lut(const uint8_t* src, uint8_t* dst, size_t n, const uint8_t* __restrict__ lut) {
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

// ---------------------------------------------------------------------------
// Equalisation without any allocation (vfs_equalize_hist_u8_noalloc).
//
// Its scratch -- one 256-bin histogram and one 256-byte LUT per image -- lives in this
// file-scope device array, which every GPU that loads the library holds until the process
// exits.  Host code cannot use the array's name as a device address (on the host it is
// only a stand-in), so the address is resolved with cudaGetSymbolAddress while the device is
// current and cached.  The cache is keyed by the device AND the id of its current CUDA
// context: after cudaDeviceReset (or under another context) the module is loaded again at a
// new address, so a changed context id makes the next call resolve the address afresh.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kSlotBytes = 256 * sizeof(unsigned int) + 256;  // histogram + LUT of one image
static __device__ __align__(256) unsigned char g_noalloc_scratch[VFS_NOALLOC_MAX_IMAGES * kSlotBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
struct NoallocAddr {
  unsigned long long ctx_id = 0;  // context the address belongs to (0 = none yet)
  void* addr = nullptr;
};
NoallocAddr g_noalloc_addr[kMaxDevices];

// cuCtxGetCurrent / cuCtxGetId, reached through the runtime's driver entry points (the library
// does not link libcuda directly).
typedef int (*PfnCtxGetCurrent)(void** ctx);
typedef int (*PfnCtxGetId)(void* ctx, unsigned long long* id);
PfnCtxGetCurrent g_ctx_get_current = nullptr;
PfnCtxGetId g_ctx_get_id = nullptr;
std::once_flag g_ctx_fns_once;

// Id of the calling thread's current context (unique for the life of the process), or 0.
unsigned long long current_context_id() {
  std::call_once(g_ctx_fns_once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = (PfnCtxGetCurrent)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_id = (PfnCtxGetId)f;
    (void)cudaGetLastError();
  });
  if (!g_ctx_get_current || !g_ctx_get_id) return 0;
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (g_ctx_get_current(&ctx) != 0 || !ctx) return 0;
  if (g_ctx_get_id(ctx, &id) != 0) return 0;
  return id;
}
}  // namespace

namespace vfs {
void set_global_error(const char* msg);
}

extern "C" int vfs_equalize_hist_u8_noalloc(const uint8_t* d_src, uint8_t* d_dst, size_t n, int count,
                                            void* cuda_stream) {
  if (count < 0 || count > VFS_NOALLOC_MAX_IMAGES) {
    vfs::set_global_error("vfs_equalize_hist_u8_noalloc: count exceeds VFS_NOALLOC_MAX_IMAGES (16)");
    return VFS_ERR_ARG;
  }
  if (n > 0xFFFFFFFFull) {
    vfs::set_global_error("vfs_equalize_hist_u8_noalloc: more than 2^32 - 1 pixels per image");
    return VFS_ERR_ARG;
  }
  if (count == 0 || n == 0) return VFS_OK;
  if (!d_src || !d_dst) {
    vfs::set_global_error("vfs_equalize_hist_u8_noalloc: null image pointer");
    return VFS_ERR_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    (void)cudaGetLastError();
    vfs::set_global_error("vfs_equalize_hist_u8_noalloc: no usable current device");
    return VFS_ERR_CUDA;
  }
  unsigned long long ctx = current_context_id();
  if (ctx == 0) {
    // No context is current on this thread yet: cudaSetDevice makes the device's primary
    // context current (the one the kernels below will run in).
    if (cudaSetDevice(dev) != cudaSuccess) {
      (void)cudaGetLastError();
      vfs::set_global_error("vfs_equalize_hist_u8_noalloc: no usable current device");
      return VFS_ERR_CUDA;
    }
    ctx = current_context_id();
  }
  unsigned char* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoallocAddr& slot = g_noalloc_addr[dev];
    // Without a context id (driver entry points unavailable) the address is resolved on every call.
    if (!slot.addr || ctx == 0 || slot.ctx_id != ctx) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        (void)cudaGetLastError();
        slot = NoallocAddr{};
        vfs::set_global_error("vfs_equalize_hist_u8_noalloc: cudaGetSymbolAddress failed");
        return VFS_ERR_CUDA;
      }
      slot.addr = p;
      slot.ctx_id = ctx;
    }
    scratch = (unsigned char*)slot.addr;
  }
  cudaStream_t st = (cudaStream_t)cuda_stream;
  try {
    for (int k = 0; k < count; k++) {
      unsigned int* hist = (unsigned int*)(scratch + k * kSlotBytes);
      uint8_t* lut = scratch + k * kSlotBytes + 256 * sizeof(unsigned int);
      // launch_equalize_hist clears the histogram slot first (the array keeps the
      // previous call's contents)
      vfs::launch_equalize_hist(d_src + (size_t)k * n, d_dst + (size_t)k * n, n, hist, lut, st);
    }
  } catch (const vfs::CudaError&) {
    (void)cudaGetLastError();
    vfs::set_global_error("vfs_equalize_hist_u8_noalloc: launch failed");
    return VFS_ERR_CUDA;
  }
  return VFS_OK;
}
