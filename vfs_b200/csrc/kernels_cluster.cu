// Cluster-resident form of the fused primal-dual iteration: all iterations of one warp of a
// small pyramid level in one launch.
//
// One thread-block cluster of C CTAs (16, or the portable 8) holds the whole level in shared
// memory.  CTA k owns the image rows [k R, k R + R) (R = ceil(h / C)) and keeps them with a
// one-row halo north and south and the columns -1 .. w (column -1 is the flat position before
// column 0, the reference's west neighbour of column 0).  One iteration is
//   * the dual step and T p at the owned pixels; a pixel of the last owned row also stores its
//     T p and (unrounded) q into the south CTA's north halo row (distributed shared memory);
//   * a cluster barrier;
//   * the threshold and primal steps at the owned pixels; a pixel of the first / last owned
//     row also stores its u-bar and v-bar into the north / south CTA's halo row;
//   * a cluster barrier.
// The dual step reads u-bar and v-bar of the pixel and of its east / south (or west / north)
// neighbours; the threshold and primal steps read T p and q of the pixel and of its west /
// north neighbours.  The barriers order every halo store between the phase that produces it
// and the phase that reads it.  A cluster barrier after the initial load keeps the first
// halo stores from landing before a neighbour has started or has loaded its halo rows from
// global memory, and after the last iteration no CTA touches another's memory.
// The per-pixel operations are those of k_fused_iter (region_step.cuh), so the results are
// bit-identical to one launch per iteration: no halo pixel is recomputed, no launch is made
// per iteration, and the level's state never leaves the chip between iterations.
//
// Pixels that an iteration leaves unwritten (masked out, and column -1) alternate between the
// values the two ping-pong buffers hold; the CTA keeps both and swaps them after each
// iteration.  At the end the owned active pixels are written into the buffers that hold the
// current state after n iterations: the other ping-pong buffers for odd n, the launch's
// input buffers for even n.  The values the other buffers would hold are those of the
// iteration before the last, which no later step reads: every iteration writes them before
// anything reads them.
//
// When the level has no row padding (stride == width), column -1 of a row is the previous
// row's last pixel, which changes every iteration; the caller then uses this kernel only if
// no pixel of column 0 is on (StereoTgvImpl::tb_ok), as for the temporally blocked form.
#include "common.cuh"
#include "fused.cuh"
#include "region_step.cuh"

#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

namespace vfs {

namespace {

constexpr int kMaxDevices = 64;
constexpr int kCLMaxThreads = 1024;
constexpr int kCLMaxPixelsPerThread = 3;

struct CLGeometry {
  int rows = 0;         // image rows per CTA
  int rx = 0, ry = 0;   // region columns (w + 2) and rows (rows + 2)
  int n = 0;            // elements per array (a multiple of 4)
  size_t bytes = 0;     // dynamic shared memory per CTA
  int ppt = 0;          // owned pixels per thread (1 .. kCLMaxPixelsPerThread)
  int threads = 0;      // threads per CTA
};

template <class ST>
CLGeometry cl_geometry(int ctas, int w, int h) {
  CLGeometry g;
  g.rows = (h + ctas - 1) / ctas;
  g.rx = w + 2;
  g.ry = g.rows + 2;
  g.n = ((g.rx * g.ry + 3) / 4) * 4;
  g.bytes = (size_t)g.n * RegionState<ST>::kBytesPerPixel;
  const int px = g.rows * w;
  for (int k = 1; k <= kCLMaxPixelsPerThread; k++) {
    const int t = ((px + k - 1) / k + 31) / 32 * 32;
    if (t <= kCLMaxThreads) {
      g.ppt = k;
      g.threads = t;
      break;
    }
  }
  return g;
}

// ---- cluster primitives, in PTX with memory clobbers so that the compiler keeps every
// shared-memory access on its side of a barrier ----

// All threads of all CTAs of the cluster: stores before it (local and remote) are visible
// to every thread of the cluster after it.
__device__ __forceinline__ void cluster_barrier() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cluster_size() {
  unsigned n;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
  return n;
}
// the shared::cluster address of the same shared-memory element in CTA `rank`
__device__ __forceinline__ unsigned cluster_addr(const void* local, unsigned rank) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(local);
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_cluster(unsigned addr, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}
__device__ __forceinline__ void st_cluster(unsigned addr, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void st_cluster(unsigned addr, float4 v) {
  asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(v.x), "f"(v.y), "f"(v.z),
               "f"(v.w)
               : "memory");
}
__device__ __forceinline__ void st_cluster(unsigned addr, __half2 v) {
  const unsigned b = *reinterpret_cast<const unsigned*>(&v);
  asm volatile("st.shared::cluster.b32 [%0], %1;" ::"r"(addr), "r"(b) : "memory");
}

}  // namespace

// PPT: owned pixels per thread (thread t owns the owned-pixel indices t + k blockDim.x).
template <bool MASKED, class ST, int PPT>
__global__ void __launch_bounds__(kCLMaxThreads, 1) k_fused_iter_cluster(const __grid_constant__ IterCLArgs A) {
  typedef Store2<ST> S;
  typedef typename S::T2 T2;
  typedef typename S::T4 T4;
  extern __shared__ __align__(16) unsigned char smem[];
  const int rank = (int)cluster_rank();
  // The grid must be exactly one cluster of A.ctas CTAs; any other shape would address CTAs
  // that do not exist.  The test is the same for every CTA, so all of them leave together,
  // before any barrier or distributed-shared-memory access.
  if ((int)cluster_size() != A.ctas || (int)(gridDim.x * gridDim.y * gridDim.z) != A.ctas) return;

  const IterPair& P = A.P;
  const int w = P.w, h = P.h, s = P.s;
  const int rows = A.rows, RX = w + 2, RY = rows + 2, N = ((RX * RY + 3) / 4) * 4;
  const int r0 = rank * rows;                                // first owned row
  const int nown = max(0, min(rows, h - r0));                // owned rows (0 for trailing CTAs)
  // The halo partners, and the first and last owned rows, are kept in shared memory and read
  // back (volatile) inside every phase: no flag computed before the cluster barriers is
  // carried across them in a register.  (Flags held that way were evaluated wrongly on
  // B200 in some builds of this kernel; the volatile reads keep every evaluation after the
  // barrier that precedes it.)
  __shared__ int s_geo[4];  // north rank or -1, south rank or -1, first owned row, last owned row
  if (threadIdx.x == 0) {
    s_geo[0] = (rank > 0 && nown > 0) ? rank - 1 : -1;               // a CTA owns the rows above
    s_geo[1] = (rank + 1 < A.ctas && (rank + 1) * rows < h) ? rank + 1 : -1;  // ... and below
    s_geo[2] = nown > 0 ? r0 : -1;
    s_geo[3] = nown > 0 ? r0 + nown - 1 : -1;
  }
  const volatile int* geo = s_geo;
  RegionState<ST> R;
  R.carve(smem, N);
  // a halo value goes to the same array element of a neighbour (every CTA has the same layout)
  auto to = [](const void* local, int rank_to) { return cluster_addr(local, (unsigned)rank_to); };

  const int plane = s * h;
  const T2* pin = (const T2*)P.p + (A.parity ? plane : 0);
  const T4* qin = (const T4*)P.q + (A.parity ? plane : 0);
  const int tid = (int)threadIdx.x, nthr = (int)blockDim.x;
  griddep_wait();

  // ---- load the owned rows and the halo rows -------------------------------------------
  if (nown > 0)
    for (int l = tid; l < RX * (nown + 2); l += nthr) {
      const int ry = l / RX, rx = l - ry * RX;
      R.template load<MASKED>(P, pin, qin, ry * RX + rx, rx - 1, r0 - 1 + ry);
    }
  // this thread's owned pixels: region index (< 0: none) and image column | row << 16
  int pi[PPT], pxy[PPT];
#pragma unroll
  for (int k = 0; k < PPT; k++) {
    const int l = tid + k * nthr;
    const int ry = l / max(w, 1), rx = l - ry * w;
    const bool own = l < nown * w;
    pi[k] = own ? (ry + 1) * RX + rx + 1 : -1;
    pxy[k] = own ? rx | ((r0 + ry) << 16) : 0;
  }
  // A cluster barrier, not a CTA barrier: every CTA of the cluster must have started and
  // finished loading its halo rows before a neighbour stores the first iteration's values
  // into them.
  cluster_barrier();

#pragma unroll 1
  for (int j = 0; j < A.n; j++) {
    // ---- dual step; the last owned row's T p and q go to the south CTA's halo ----------
    // (one copy of the per-pixel code: under the 64-register limit of 1024-thread CTAs
    // unrolled copies spill)
#pragma unroll 1
    for (int k = 0; k < PPT; k++) {
      const int i = pi[k];
      if (i < 0) continue;
      const int gx = pxy[k] & 0xffff, gy = pxy[k] >> 16;
      const bool wrote = R.template dual<MASKED>(i, RX, gx, gy, w, h, A.sp[j], A.sq[j]);
      const int south = geo[1];
      if (wrote && south >= 0 && gy == geo[3]) {
        const int hi = i - nown * RX;  // row 0 of the south CTA's region
        st_cluster(to(R.tp + hi, south), R.tp[i]);
        st_cluster(to(R.q + hi, south), R.q[i]);
      }
    }
    cluster_barrier();
    // ---- threshold and primal steps; u-bar and v-bar of the edge rows to the halos -------
#pragma unroll 1
    for (int k = 0; k < PPT; k++) {
      const int i = pi[k];
      if (i < 0) continue;
      const int gx = pxy[k] & 0xffff, gy = pxy[k] >> 16;
      if (MASKED && !(R.code[i] & kOn)) R.keep(i);
      else R.template primal<MASKED>(P, i, RX, gx, gy, A.tau[j], A.mu[j]);
      const int north = geo[0], south = geo[1];
      if (north >= 0 && gy == geo[2]) {
        const int hi = i + rows * RX;  // row rows + 1 of the north CTA's region
        st_cluster(to(R.ub + hi, north), R.ub[i]);
        st_cluster(to(R.v + hi, north), R.v[i]);
      }
      if (south >= 0 && gy == geo[3]) {
        const int hi = i - nown * RX;
        st_cluster(to(R.ub + hi, south), R.ub[i]);
        st_cluster(to(R.v + hi, south), R.v[i]);
      }
    }
    // column -1 of the owned rows is never written: it alternates like a masked-out pixel
    if (MASKED)
      for (int r = tid; r < nown; r += nthr) R.keep((r + 1) * RX);
    cluster_barrier();
  }

  // ---- write the owned active pixels into the buffers current after n iterations --------
  const bool odd = A.n & 1;
  float* uo = odd ? P.us : const_cast<float*>(P.u);
  float* ubo = odd ? P.u_s : const_cast<float*>(P.u_);
  T2* vo = (T2*)(odd ? P.v_s : const_cast<void*>(P.v_));
  const int pl = (A.parity + A.n) & 1;  // p / q plane written by the last iteration
  T2* po = (T2*)P.p + (pl ? plane : 0);
  T4* qo = (T4*)P.q + (pl ? plane : 0);
#pragma unroll
  for (int k = 0; k < PPT; k++) {
    const int i = pi[k];
    if (i < 0) continue;
    if (MASKED && !(R.code[i] & kOn)) continue;
    const int pos = (pxy[k] & 0xffff) + (pxy[k] >> 16) * s;
    uo[pos] = R.u[i];
    ubo[pos] = R.ub[i];
    vo[pos] = R.v[i];
    po[pos] = R.p[i];
    qo[pos] = S::rnd4(R.q[i]);
    if (A.write_tp) P.Tp[pos] = R.tp[i];
  }
}

namespace {

typedef void (*CLKernel)(IterCLArgs);

template <bool MASKED, class ST, int PPT>
CLKernel cl_kernel() {
  return k_fused_iter_cluster<MASKED, ST, PPT>;
}

// Dynamic shared memory a CTA of the kernel may use: the device's opt-in maximum less the
// kernel's static shared memory.
int max_dynamic_smem() {
  int dev = 0, optin = 0;
  VFS_CUDA(cudaGetDevice(&dev));
  VFS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes f0{};
  VFS_CUDA(cudaFuncGetAttributes(&f0, k_fused_iter_cluster<true, float, 1>));
  return optin - (int)f0.sharedSizeBytes;
}

template <bool MASKED, class ST, int PPT>
void set_cl_attributes() {
  const CLKernel k = cl_kernel<MASKED, ST, PPT>();
  static std::atomic<bool> configured[kMaxDevices];
  int dev = 0;
  VFS_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < kMaxDevices && configured[dev].load(std::memory_order_acquire)) return;
  VFS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dynamic_smem()));
  VFS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  if (dev >= 0 && dev < kMaxDevices) configured[dev].store(true, std::memory_order_release);
}

cudaLaunchConfig_t cl_config(const CLGeometry& g, int ctas, cudaStream_t st, cudaLaunchAttribute* at, unsigned& nat) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(g.threads);
  cfg.dynamicSmemBytes = g.bytes;
  cfg.stream = st;
  nat = 0;
  at[nat].id = cudaLaunchAttributeClusterDimension;
  at[nat].val.clusterDim.x = ctas;
  at[nat].val.clusterDim.y = 1;
  at[nat].val.clusterDim.z = 1;
  nat++;
  cfg.attrs = at;
  cfg.numAttrs = nat;
  return cfg;
}

// can a cluster of this shape be resident on the device (0 or the number of such clusters)
template <bool MASKED, class ST, int PPT>
int cl_max_clusters(const CLGeometry& g, int ctas) {
  set_cl_attributes<MASKED, ST, PPT>();
  cudaLaunchAttribute at[2];
  unsigned nat = 0;
  cudaLaunchConfig_t cfg = cl_config(g, ctas, 0, at, nat);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, cl_kernel<MASKED, ST, PPT>(), &cfg) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return n;
}

template <bool MASKED, class ST, int PPT>
void launch_cl(const IterCLArgs& A, const CLGeometry& g, int ctas, cudaStream_t st) {
  set_cl_attributes<MASKED, ST, PPT>();
  cudaLaunchAttribute at[2];
  unsigned nat = 0;
  cudaLaunchConfig_t cfg = cl_config(g, ctas, st, at, nat);
  const int prio = launch_priority();
  if (prio != 0) {
    at[nat].id = cudaLaunchAttributePriority;
    at[nat].val.priority = prio;
    nat++;
    cfg.numAttrs = nat;
  }
  VFS_CUDA(cudaLaunchKernelEx(&cfg, cl_kernel<MASKED, ST, PPT>(), A));
}

// run F<MASKED, ST, PPT> for the runtime form, storage and pixels per thread
template <template <bool, class, int> class F, typename... Args>
auto cl_dispatch(bool masked, bool half, int ppt, Args&&... args) {
#define VFS_CL_PPT(M, T)                                      \
  switch (ppt) {                                              \
    case 1: return F<M, T, 1>::run(args...);                  \
    case 2: return F<M, T, 2>::run(args...);                  \
    case 3: return F<M, T, 3>::run(args...);                  \
    default: throw ArgError{"cluster-resident iteration: level too large"}; \
  }
#define VFS_CL_ST(M) \
  if (half) { VFS_CL_PPT(M, __half) } else { VFS_CL_PPT(M, float) }
  if (masked) { VFS_CL_ST(true) } else { VFS_CL_ST(false) }
#undef VFS_CL_ST
#undef VFS_CL_PPT
}

template <bool MASKED, class ST, int PPT>
struct MaxClusters {
  static int run(const CLGeometry& g, int ctas) { return cl_max_clusters<MASKED, ST, PPT>(g, ctas); }
};
template <bool MASKED, class ST, int PPT>
struct Launch {
  static int run(const IterCLArgs& A, const CLGeometry& g, int ctas, cudaStream_t st) {
    launch_cl<MASKED, ST, PPT>(A, g, ctas, st);
    return 0;
  }
};

CLGeometry geometry_of(int variant, bool half, int w, int h) {
  const int ctas = cluster_ctas(variant);
  return half ? cl_geometry<__half>(ctas, w, h) : cl_geometry<float>(ctas, w, h);
}

}  // namespace

int cluster_ctas(int variant) {
  switch (variant) {
    case kIterFirstClusterVariant: return 16;
    case kIterFirstClusterVariant + 1: return 8;
    default: return 0;
  }
}

bool cluster_fits(int variant, bool masked, bool half, int w, int h) {
  const int ctas = cluster_ctas(variant);
  if (ctas <= 0 || w <= 0 || h <= 0) return false;
  int dev = 0;
  VFS_CUDA(cudaGetDevice(&dev));
  // the answer depends only on the device and the shape; ask the runtime once per shape
  static std::mutex mu;
  static std::map<std::tuple<int, int, bool, bool, int, int>, bool> known;
  const auto key = std::make_tuple(dev, variant, masked, half, w, h);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = known.find(key);
    if (it != known.end()) return it->second;
  }
  const CLGeometry g = geometry_of(variant, half, w, h);
  // (a thread packs a pixel's column and row into one int: 16 bits each)
  bool ok = g.ppt > 0 && g.bytes <= (size_t)max_dynamic_smem() && w + 2 <= 4096 && h < 32768;
  if (ok) ok = cl_dispatch<MaxClusters>(masked, half, g.ppt, g, ctas) >= 1;
  std::lock_guard<std::mutex> lk(mu);
  known[key] = ok;
  return ok;
}

int cluster_pixels_per_thread(int variant, bool half, int w, int h) {
  if (cluster_ctas(variant) <= 0 || w <= 0 || h <= 0) return 0;
  return geometry_of(variant, half, w, h).ppt;
}

int cluster_rows(int variant, int h) {
  const int ctas = cluster_ctas(variant);
  return ctas > 0 ? (h + ctas - 1) / ctas : 0;
}

double cluster_gpu_share(int variant, int w, int h) {
  (void)w;
  (void)h;
  int dev = 0, sms = 1;
  VFS_CUDA(cudaGetDevice(&dev));
  VFS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // one CTA per SM (the level's state takes most of an SM's shared memory or threads)
  return std::min(1.0, (double)cluster_ctas(variant) / (double)sms);
}

void launch_fused_iteration_cluster(const IterCLArgs& A, bool masked, bool half_storage, cudaStream_t st,
                                    int variant) {
  const int ctas = cluster_ctas(variant);
  if (ctas <= 0) throw ArgError{"not a cluster-resident iteration variant"};
  if (A.n < 1 || A.n > kCLMaxIters) throw ArgError{"cluster-resident iteration: bad iteration count"};
  if (A.P.w <= 0 || A.P.h <= 0) return;
  const CLGeometry g = geometry_of(variant, half_storage, A.P.w, A.P.h);
  if (A.rows != g.rows || A.ctas != ctas || g.ppt == 0) throw ArgError{"cluster-resident iteration: bad geometry"};
  cl_dispatch<Launch>(masked, half_storage, g.ppt, A, g, ctas, st);
  VFS_LAUNCH_CHECK();
}

}  // namespace vfs
