// Temporally blocked form of the fused primal-dual iteration: K iterations per launch.
//
// A block owns an output tile T of TX x TY pixels and keeps the whole state of the region
// R = T extended by 2K pixels to the west / north and K to the east / south in shared
// memory.  One iteration's output at a pixel depends on u-bar and v-bar two pixels west /
// north and one pixel east / south of it, on p and q of the pixel and its west / north
// neighbour, and on u of the pixel, so iteration j (0-based) runs
//   * the dual step on D_j = T extended by 2(K-1-j)+1 west / north and K-1-j east / south,
//   * the threshold and primal steps on O_j = T extended by 2(K-1-j) and K-1-j,
// and after K iterations the values on T are exact.  The per-pixel operations, their order
// and the storage rounding between iterations (half storage of p, q, v-bar) are those of
// k_fused_iter, so results are bit-identical to K launches of it.
//
// Pixels that an iteration leaves unwritten (masked out, padding) alternate between the
// values held by the two ping-pong buffers in the per-iteration form; the block keeps both
// and swaps them after every iteration.  K is odd, so after a launch the results belong in
// the other ping-pong buffers, where they are written, and the pixels left unwritten keep
// the value that buffer holds, as they would after K single iterations.
//
// The reference's west neighbour of column 0 is the flat position before it (the previous
// row's last padding element).  That element is constant during a level when the row has
// padding (stride > width).  When stride == width it is the previous row's last pixel,
// which changes every iteration; the caller then uses this kernel only if no pixel of
// column 0 is on (StereoTgvImpl::tb_ok).
#include "common.cuh"
#include "fused.cuh"
#include "region_step.cuh"

#include <atomic>

namespace vfs {

namespace {

constexpr int kTBX = 32;  // threads of a block in x (its y extent BY is a template parameter)
constexpr int kMaxDevices = 64;

template <class ST, int K, int TX, int TY>
struct TBLayout {
  static constexpr int RX = TX + 3 * K, RY = TY + 3 * K;
  static constexpr int N = ((RX * RY + 3) / 4) * 4;  // elements per array (16-byte aligned arrays)
  static constexpr size_t kBytes = (size_t)N * RegionState<ST>::kBytesPerPixel;
};

}  // namespace

// BY: threads of the block in y.  A thread handles the region pixels (tx + 32 a, ty + BY b);
// with TX + 3K = 32 and TY + 3K = BY that is exactly one pixel.
template <bool MASKED, class ST, int K, int TX, int TY, int BY>
__global__ void __launch_bounds__(kTBX* BY, 1) k_fused_iter_tb(const __grid_constant__ IterTBArgs A) {
  constexpr int kTBY = BY;
  typedef TBLayout<ST, K, TX, TY> L;
  typedef Store2<ST> S;
  typedef typename S::T2 T2;
  typedef typename S::T4 T4;
  constexpr int RX = L::RX, RY = L::RY;
  extern __shared__ __align__(16) unsigned char smem[];
  RegionState<ST> R;
  R.carve(smem, L::N);

  const IterPair& P = A.P;
  const int w = P.w, h = P.h, s = P.s;
  const int gx0 = (int)blockIdx.x * TX - 2 * K, gy0 = (int)blockIdx.y * TY - 2 * K;  // region origin
  const int plane = s * h;
  const T2* pin = (const T2*)P.p + (A.parity ? plane : 0);
  const T4* qin = (const T4*)P.q + (A.parity ? plane : 0);
  T2* pout = (T2*)P.p + (A.parity ? 0 : plane);
  T4* qout = (T4*)P.q + (A.parity ? 0 : plane);
  const int tx = threadIdx.x, ty = threadIdx.y;
  griddep_wait();  // the previous launch's outputs are this one's inputs
  griddep_launch_dependents();

  // ---- load the region --------------------------------------------------------------
  for (int ry = ty; ry < RY; ry += kTBY)
    for (int rx = tx; rx < RX; rx += kTBX) R.template load<MASKED>(P, pin, qin, ry * RX + rx, gx0 + rx, gy0 + ry);
  __syncthreads();

#pragma unroll 1
  for (int j = 0; j < K; j++) {
    // ---- dual step on D_j ----------------------------------------------------------------
    const int dlo = 2 * j + 1, dhx = RX - (j + 1), dhy = RY - (j + 1);
    for (int ry = dlo + ty; ry < dhy; ry += kTBY) {
      const int gy = gy0 + ry;
      for (int rx = dlo + tx; rx < dhx; rx += kTBX) {
        const int gx = gx0 + rx;
        if (!(gx >= 0 && gx < w && gy >= 0 && gy < h)) continue;
        R.template dual<MASKED>(ry * RX + rx, RX, gx, gy, w, h, A.sp[j], A.sq[j]);
      }
    }
    __syncthreads();
    // ---- threshold and primal steps on O_j; alternation of the unwritten pixels --------
    const int olo = 2 * j + 2, ohx = RX - (j + 1), ohy = RY - (j + 1);
    for (int ry = ty; ry < RY; ry += kTBY) {
      const int gy = gy0 + ry;
      for (int rx = tx; rx < RX; rx += kTBX) {
        const int gx = gx0 + rx;
        const int i = ry * RX + rx;
        const bool in = gx >= 0 && gx < w && gy >= 0 && gy < h;
        const bool act = MASKED ? (in && (R.code[i] & kOn)) : in;
        if (!act) {
          if (MASKED) R.keep(i);
          continue;
        }
        if (rx < olo || rx >= ohx || ry < olo || ry >= ohy) continue;
        R.template primal<MASKED>(P, i, RX, gx, gy, A.tau[j], A.mu[j]);
      }
    }
    __syncthreads();
  }

  // ---- write the tile into the other ping-pong buffers ------------------------------------
  for (int ry = 2 * K + ty; ry < 2 * K + TY; ry += kTBY) {
    const int gy = gy0 + ry;
    if (gy >= h) break;
    for (int rx = 2 * K + tx; rx < 2 * K + TX; rx += kTBX) {
      const int gx = gx0 + rx;
      if (gx >= w) break;
      const int i = ry * RX + rx;
      if (MASKED && !(R.code[i] & kOn)) continue;
      const int pos = gx + gy * s;
      P.us[pos] = R.u[i];
      P.u_s[pos] = R.ub[i];
      ((T2*)P.v_s)[pos] = R.v[i];
      pout[pos] = R.p[i];
      qout[pos] = S::rnd4(R.q[i]);
      if (A.write_tp) P.Tp[pos] = R.tp[i];
    }
  }
}

namespace {

template <bool MASKED, class ST, int K, int TX, int TY, int BY>
void launch_tb_k(const IterTBArgs& A, cudaStream_t st) {
  typedef TBLayout<ST, K, TX, TY> L;
  auto k = k_fused_iter_tb<MASKED, ST, K, TX, TY, BY>;
  // the shared-memory limit is raised once per instantiation and device
  static std::atomic<bool> configured[kMaxDevices];
  int dev = 0;
  VFS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices || !configured[dev].load(std::memory_order_acquire)) {
    VFS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::kBytes));
    if (dev >= 0 && dev < kMaxDevices) configured[dev].store(true, std::memory_order_release);
  }
  const dim3 grid((A.P.w + TX - 1) / TX, (A.P.h + TY - 1) / TY), blk(kTBX, BY);
  launch_overlapped_smem(k, grid, blk, L::kBytes, st, A);
}

template <bool MASKED, class ST, int K, int TX, int TY, int BY>
int tb_blocks_per_sm_k() {
  typedef TBLayout<ST, K, TX, TY> L;
  auto k = k_fused_iter_tb<MASKED, ST, K, TX, TY, BY>;
  VFS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::kBytes));
  int n = 0;
  VFS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kTBX * BY, L::kBytes));
  return n;
}

template <int K, int TX, int TY, int BY>
double tb_share(bool masked, bool half, int w, int h) {
  int per_sm;
  if (masked) per_sm = half ? tb_blocks_per_sm_k<true, __half, K, TX, TY, BY>() : tb_blocks_per_sm_k<true, float, K, TX, TY, BY>();
  else per_sm = half ? tb_blocks_per_sm_k<false, __half, K, TX, TY, BY>() : tb_blocks_per_sm_k<false, float, K, TX, TY, BY>();
  const long long blocks = (long long)((w + TX - 1) / TX) * ((h + TY - 1) / TY);
  int dev = 0, sms = 1;
  VFS_CUDA(cudaGetDevice(&dev));
  VFS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const double cap = (double)sms * (per_sm > 0 ? per_sm : 1);
  return blocks >= cap ? 1.0 : (double)blocks / cap;
}

template <int K, int TX, int TY, int BY>
void launch_tb_3(const IterTBArgs& A, bool masked, bool half_storage, cudaStream_t st) {
  if (masked) {
    if (half_storage) launch_tb_k<true, __half, K, TX, TY, BY>(A, st);
    else launch_tb_k<true, float, K, TX, TY, BY>(A, st);
  } else {
    if (half_storage) launch_tb_k<false, __half, K, TX, TY, BY>(A, st);
    else launch_tb_k<false, float, K, TX, TY, BY>(A, st);
  }
}

}  // namespace

int tb_iterations(int variant) {
  switch (variant) {
    case kIterFirstTBVariant: return 3;
    case kIterFirstTBVariant + 1: return 5;
    case kIterFirstTBVariant + 2: return 3;
    case kIterFirstTBVariant + 3: return 5;
    case kIterFirstDeepTBVariant: return 7;
    case kIterFirstDeepTBVariant + 1: return 9;
    default: return 1;
  }
}

double tb_gpu_share(int variant, bool masked, bool half, int w, int h) {
  switch (variant) {
    case kIterFirstTBVariant: return tb_share<3, 64, 24, 16>(masked, half, w, h);
    case kIterFirstTBVariant + 1: return tb_share<5, 32, 24, 16>(masked, half, w, h);
    case kIterFirstTBVariant + 2: return tb_share<3, 23, 23, 32>(masked, half, w, h);
    case kIterFirstTBVariant + 3: return tb_share<5, 17, 17, 32>(masked, half, w, h);
    case kIterFirstDeepTBVariant: return tb_share<7, 11, 11, 32>(masked, half, w, h);
    case kIterFirstDeepTBVariant + 1: return tb_share<9, 5, 5, 32>(masked, half, w, h);
    default: throw ArgError{"not a temporally blocked iteration variant"};
  }
}

void launch_fused_iteration_tb(const IterTBArgs& A, bool masked, bool half_storage, cudaStream_t st, int variant) {
  if (A.P.w <= 0 || A.P.h <= 0) return;
  switch (variant) {
    case kIterFirstTBVariant: launch_tb_3<3, 64, 24, 16>(A, masked, half_storage, st); break;
    case kIterFirstTBVariant + 1: launch_tb_3<5, 32, 24, 16>(A, masked, half_storage, st); break;
    // one region pixel per thread: 32 x 32 regions
    case kIterFirstTBVariant + 2: launch_tb_3<3, 23, 23, 32>(A, masked, half_storage, st); break;
    case kIterFirstTBVariant + 3: launch_tb_3<5, 17, 17, 32>(A, masked, half_storage, st); break;
    case kIterFirstDeepTBVariant: launch_tb_3<7, 11, 11, 32>(A, masked, half_storage, st); break;
    case kIterFirstDeepTBVariant + 1: launch_tb_3<9, 5, 5, 32>(A, masked, half_storage, st); break;
    default: throw ArgError{"not a temporally blocked iteration variant"};
  }
  VFS_LAUNCH_CHECK();
}

}  // namespace vfs
