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
#include "tgv_pixel.cuh"
#include "tgv_pixel_fast.cuh"

#include <atomic>
#include <type_traits>

namespace vfs {

namespace {

constexpr int kTBX = 32;  // threads of a block in x (its y extent BY is a template parameter)
constexpr int kMaxDevices = 64;

template <class ST, int K, int TX, int TY>
struct TBLayout {
  typedef typename Store2<ST>::T2 T2;
  typedef typename Store2<ST>::T4 T4;
  static constexpr int RX = TX + 3 * K, RY = TY + 3 * K;
  static constexpr int N = ((RX * RY + 3) / 4) * 4;  // elements per array (16-byte aligned arrays)
  // float arrays: ubar, ubar_alt, u, a, b, c, Iu, Iz; T2: v, v_alt, p; float4: q; float2: Tp;
  // u8: code.  q is kept unrounded: within an iteration the threshold and primal steps read
  // this iteration's q at full precision (as the one-iteration kernel does from registers and
  // shared memory); the next iteration's dual step reads it in the stored precision.
  static constexpr size_t kBytes =
      (size_t)N * (8 * sizeof(float) + 3 * sizeof(T2) + sizeof(float4) + sizeof(float2) + 1);
};

}  // namespace

// BY: threads of the block in y.  A thread handles the region pixels (tx + 32 a, ty + BY b);
// with TX + 3K = 32 and TY + 3K = BY that is exactly one pixel.
template <bool MASKED, class ST, int K, int TX, int TY, int BY>
__global__ void __launch_bounds__(kTBX* BY, 1) k_fused_iter_tb(const __grid_constant__ IterTBArgs A) {
  constexpr int kTBY = BY;
  typedef TBLayout<ST, K, TX, TY> L;
  typedef typename L::T2 T2;
  typedef typename L::T4 T4;
  typedef Store2<ST> S;
  constexpr int RX = L::RX, RY = L::RY, N = L::N;
  constexpr bool kFast = !std::is_same<ST, float>::value;
  extern __shared__ __align__(16) unsigned char smem[];
  float* s_ub = reinterpret_cast<float*>(smem);
  float* s_uba = s_ub + N;
  float* s_u = s_uba + N;
  float* s_a = s_u + N;
  float* s_b = s_a + N;
  float* s_c = s_b + N;
  float* s_Iu = s_c + N;
  float* s_Iz = s_Iu + N;
  T2* s_v = reinterpret_cast<T2*>(s_Iz + N);
  T2* s_va = s_v + N;
  T2* s_p = s_va + N;
  float4* s_q = reinterpret_cast<float4*>(s_p + N);
  float2* s_tp = reinterpret_cast<float2*>(s_q + N);
  uint8_t* s_code = reinterpret_cast<uint8_t*>(s_tp + N);

  const IterPair& P = A.P;
  const int w = P.w, h = P.h, s = P.s;
  const int gx0 = (int)blockIdx.x * TX - 2 * K, gy0 = (int)blockIdx.y * TY - 2 * K;  // region origin
  const int plane = s * h;
  const T2* pin = (const T2*)P.p + (A.parity ? plane : 0);
  const T4* qin = (const T4*)P.q + (A.parity ? plane : 0);
  T2* pout = (T2*)P.p + (A.parity ? 0 : plane);
  T4* qout = (T4*)P.q + (A.parity ? 0 : plane);
  const T2* vin = (const T2*)P.v_;
  const T2* valt = (const T2*)P.v_s;  // the other ping-pong buffer of v-bar (also the output)
  const int tx = threadIdx.x, ty = threadIdx.y;
  griddep_wait();  // the previous launch's outputs are this one's inputs
  griddep_launch_dependents();

  // ---- load the region --------------------------------------------------------------
  for (int ry = ty; ry < RY; ry += kTBY) {
    const int gy = gy0 + ry;
    for (int rx = tx; rx < RX; rx += kTBX) {
      const int gx = gx0 + rx;
      const int i = ry * RX + rx;
      const int pos = gx + gy * s;
      const bool in = gx >= 0 && gx < w && gy >= 0 && gy < h;
      // flat positions the reference may read: columns [-1, w) of rows < h, at or after the
      // buffer start (column -1 is the previous row's last padding element)
      const bool flat = gx >= -1 && gx < w && gy < h && pos >= 0;
      const uint8_t code = in ? P.code[pos] : (uint8_t)0;
      const bool act = MASKED ? (in && (code & kOn)) : in;  // written by every iteration
      s_code[i] = code;
      s_ub[i] = flat ? P.u_[pos] : 0.0f;
      s_v[i] = flat ? vin[pos] : S::ld2z();
      if (MASKED) {
        s_uba[i] = (flat && !act) ? P.u_s[pos] : 0.0f;
        s_va[i] = (flat && !act) ? valt[pos] : S::ld2z();
      }
      s_u[i] = act ? P.u[pos] : 0.0f;
      s_p[i] = act ? pin[pos] : S::ld2z();
      s_q[i] = act ? S::cvt4(qin[pos]) : make_float4(0.f, 0.f, 0.f, 0.f);
      s_a[i] = in ? P.a[pos] : 0.0f;
      s_b[i] = in ? P.b[pos] : 0.0f;
      s_c[i] = in ? P.c[pos] : 0.0f;
      s_Iu[i] = act ? P.Iu[pos] : 0.0f;
      s_Iz[i] = act ? P.Iz[pos] : 0.0f;
      // stored T p: read where a pixel keeps its values (masked form) and west of column 0
      const bool tps = (MASKED && in && !act) || (gx == -1 && gy >= 1 && gy < h);
      s_tp[i] = tps ? P.Tp[pos] : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();

#pragma unroll 1
  for (int j = 0; j < K; j++) {
    const float sp = A.sp[j], sq = A.sq[j], tau = A.tau[j], mu = A.mu[j];
    // ---- dual step on D_j ----------------------------------------------------------------
    const int dlo = 2 * j + 1, dhx = RX - (j + 1), dhy = RY - (j + 1);
    for (int ry = dlo + ty; ry < dhy; ry += kTBY) {
      const int gy = gy0 + ry;
      for (int rx = dlo + tx; rx < dhx; rx += kTBX) {
        const int gx = gx0 + rx;
        const int i = ry * RX + rx;
        const uint8_t code = s_code[i];
        const bool in = gx >= 0 && gx < w && gy >= 0 && gy < h;
        if (!in) continue;
        bool useRight, useDown;
        const float a = s_a[i], b = s_b[i], c = s_c[i];
        if (MASKED) {
          if (!(code & kOn)) continue;  // keeps its values; its stored T p is in s_tp
          useRight = code & kR;
          useDown = code & kD;
        } else {
          if (!(code & kOn)) {  // outside the circle: p = q = 0, T p = T 0
            const float2 z = make_float2(0.f, 0.f);
            s_p[i] = S::ld2z();
            s_q[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            s_tp[i] = kFast ? fast::tp(a, b, c, z) : tp_math(a, b, c, z);
            continue;
          }
          useRight = (gx + 1) < w;
          useDown = (gy + 1) < h;
        }
        const float ubar = s_ub[i];
        const float2 vb = S::cvt2(s_v[i]);
        const float u_xn = useRight ? s_ub[i + 1] : s_ub[i - 1];
        const float u_yn = useDown ? s_ub[i + RX] : s_ub[i - RX];
        const float2 v_xn = S::cvt2(useRight ? s_v[i + 1] : s_v[i - 1]);
        const float2 v_yn = S::cvt2(useDown ? s_v[i + RX] : s_v[i - RX]);
        float2 pp = S::cvt2(s_p[i]);
        float4 qq = S::cvt4(S::rnd4(s_q[i]));  // the stored (rounded) q of the last iteration
        float2 tp;
        if (kFast) {
          fast::dual(useRight, useDown, ubar, u_xn, u_yn, vb, v_xn, v_yn, a, b, c, sp, sq, pp, qq);
          tp = fast::tp(a, b, c, pp);
        } else {
          dual_math(useRight, useDown, ubar, u_xn, u_yn, vb, v_xn, v_yn, a, b, c, sp, sq, pp, qq);
          tp = tp_math(a, b, c, pp);
        }
        s_p[i] = S::rnd2(pp);
        s_q[i] = qq;
        s_tp[i] = tp;
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
        const uint8_t code = s_code[i];
        const bool in = gx >= 0 && gx < w && gy >= 0 && gy < h;
        const bool act = MASKED ? (in && (code & kOn)) : in;
        if (!act) {
          if (MASKED) {
            const float t = s_ub[i];
            s_ub[i] = s_uba[i];
            s_uba[i] = t;
            const T2 tv = s_v[i];
            s_v[i] = s_va[i];
            s_va[i] = tv;
          }
          continue;
        }
        if (rx < olo || rx >= ohx || ry < olo || ry >= ohy) continue;
        float dxm, dym;
        bool zR, zD, hasL, hasU;
        const float2 tp = s_tp[i], tpW = s_tp[i - 1], tpN = s_tp[i - RX];
        if (MASKED) {
          const bool mR = code & kR, mL = code & kL, mD = code & kD, mU = code & kU;
          if (mL && mR) dxm = tp.x - tpW.x;
          else if (!mR) dxm = -tpW.x;
          else dxm = tp.x;
          if (mU && mD) dym = tp.y - tpN.y;
          else if (!mD) dym = -tpN.y;
          else dym = tp.y;
          zR = !mR;
          zD = !mD;
          hasL = mL;
          hasU = mU;
        } else {
          if (!(code & kOn)) {
            s_u[i] = 0.0f;
            s_ub[i] = 0.0f;
            s_v[i] = S::rnd2(make_float2(0.f, 0.f));
            continue;
          }
          if ((gx - 1) >= 0) dxm = tp.x - tpW.x;
          else if (gx == w - 1) dxm = -tpW.x;
          else dxm = tp.x;
          if ((gy - 1) >= 0) dym = tp.y - tpN.y;
          else if (gy == h - 1) dym = -tpN.y;
          else dym = tp.y;
          zR = gx == w - 1;
          zD = gy == h - 1;
          hasL = (gx - 1) >= 0;
          hasU = (gy - 1) >= 0;
        }
        const float a = s_a[i], b = s_b[i], c = s_c[i];
        const float ubar = s_ub[i];
        const float2 vb = S::cvt2(s_v[i]);
        float unew;
        if (kFast) {
          float eu = fast::etau(a, b, c, P.alpha1 * P.alpha1);
          unew = fast::threshold(dxm, dym, eu, tau, ubar, s_u[i], s_Iu[i], s_Iz[i], P.lambda);
        } else {
          float eu = etau_math(a, b, c, P.alpha1);
          unew = threshold_math(dxm, dym, eu, tau, ubar, s_u[i], s_Iu[i], s_Iz[i], P.lambda);
        }
        float4 qc = s_q[i];
        if (zR) qc.x = qc.w = 0.0f;
        if (zD) qc.y = qc.z = 0.0f;
        const float4 ql = hasL ? s_q[i - 1] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 qu = hasU ? s_q[i - RX] : make_float4(0.f, 0.f, 0.f, 0.f);
        float us_;
        float2 vs;
        if (kFast) {
          const float a1s = P.alpha1 * P.alpha1, a0s4 = 4.0f * P.alpha0 * P.alpha0;
          float ev1 = fast::etav(b, c, a1s, a0s4), ev2 = fast::etav(a, c, a1s, a0s4);
          fast::primal(qc, ql, qu, tp, ev1, ev2, tau, P.alpha0, P.alpha1, mu, vb, unew, ubar, us_, vs);
        } else {
          float ev1 = etav1_math(b, c, P.alpha0, P.alpha1), ev2 = etav2_math(a, c, P.alpha0, P.alpha1);
          float2 vo;
          const float2 pp = S::cvt2(s_p[i]);
          primal_math(qc, ql, qu, pp, a, b, c, ev1, ev2, tau, P.alpha0, P.alpha1, mu, vb, unew, ubar, us_, vs, vo);
        }
        s_u[i] = unew;
        s_ub[i] = us_;
        s_v[i] = S::rnd2(vs);
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
      const uint8_t code = s_code[i];
      if (MASKED && !(code & kOn)) continue;
      const int pos = gx + gy * s;
      P.us[pos] = s_u[i];
      P.u_s[pos] = s_ub[i];
      ((T2*)P.v_s)[pos] = s_v[i];
      pout[pos] = s_p[i];
      qout[pos] = S::rnd4(s_q[i]);
      if (A.write_tp) P.Tp[pos] = s_tp[i];
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
