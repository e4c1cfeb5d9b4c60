// Shared host/device helpers of the vfs_b200 library.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <map>
#include <string>
#include <tuple>

namespace vfs {

// Error carried from a failing CUDA call to the C ABI as a status code.
struct CudaError {
  cudaError_t err;
  const char* what;
  const char* file;
  int line;
};

#define VFS_CUDA(call)                                            \
  do {                                                            \
    cudaError_t e_ = (call);                                      \
    if (e_ != cudaSuccess) throw ::vfs::CudaError{e_, #call, __FILE__, __LINE__}; \
  } while (0)

// Every kernel launch of the library goes through VFS_LAUNCH_CHECK, which also
// counts it (vfs_launch_count in the C ABI).
std::atomic<long long>& launch_counter();
#define VFS_LAUNCH_CHECK()                                                  \
  do {                                                                      \
    VFS_CUDA(cudaGetLastError());                                           \
    ::vfs::launch_counter().fetch_add(1, std::memory_order_relaxed);        \
  } while (0)

// Host-side trace ranges (NVTX) around the library's entry points and solve phases, for
// profilers that record them (ncu --nvtx, Nsight Systems); without one attached they cost a
// null check.  In graph replays a range covers the enqueue, not the GPU work.
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};
// "level 0" .. "level 15"
const char* level_range_name(int level);

// Opt-in timing of launch groups with CUDA events on the solver's stream.
struct ProfRec {
  int tag;        // ProfTag
  int level;
  long long px;   // pixels of the level
  int iters;      // inner iterations covered by the record
  cudaEvent_t a, b;
  int launches;   // kernel launches of the record's group
};
enum ProfTag { kProfInner = 0, kProfFused = 1, kProfPrologue = 2, kProfEpilogue = 3, kProfTags = 4 };

struct ArgError {
  std::string msg;
};

// Programmatic dependent launch of the fused iteration kernels.  With it on, the next launch
// on a stream may be scheduled while the previous one drains; every kernel launched this way
// executes griddep_wait() before its first global-memory access, which returns once the
// previous launch has completed and its writes are visible, so results do not depend on the
// overlap.  Process-wide switch (vfs_set_launch_overlap), on by default.
std::atomic<bool>& pdl_enabled();
// Scheduling priority given to the fused iteration kernels launched by this host thread (0:
// none; otherwise a stream-priority value, numerically lower = higher priority).  Set around
// the launches of the work that should win the block scheduler (kept in captured graphs).
int& launch_priority();
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <typename... KArgs, typename... Args>
inline void launch_overlapped_smem(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                                   Args... args) {
  const bool pdl = pdl_enabled().load(std::memory_order_relaxed);
  const int prio = launch_priority();
  if (!pdl && prio == 0) {
    k<<<grid, block, smem, st>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[2];
  unsigned n = 0;
  if (pdl) {
    at[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[n].val.programmaticStreamSerializationAllowed = 1;
    n++;
  }
  if (prio != 0) {
    at[n].id = cudaLaunchAttributePriority;
    at[n].val.priority = prio;
    n++;
  }
  cfg.attrs = at;
  cfg.numAttrs = n;
  VFS_CUDA(cudaLaunchKernelEx(&cfg, k, args...));
}
template <typename... KArgs, typename... Args>
inline void launch_overlapped(void (*k)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
  launch_overlapped_smem(k, grid, block, 0, st, args...);
}

inline int iDivUp(int n, int m) { return (n + m - 1) / m; }

// Launch shape of the plain per-pixel kernels: 32 columns x 8 rows, so a warp reads
// one row segment (coalesced for float, float2 and float4 rows).
constexpr int kBX = 32;
constexpr int kBY = 8;
inline dim3 grid2d(int w, int h) { return dim3(iDivUp(w, kBX), iDivUp(h, kBY)); }
inline dim3 block2d() { return dim3(kBX, kBY); }

// Texture objects with the sampling setup of every gather of the reference
// (normalized coordinates, mirror addressing, pitch-2D float / float2 memory, or one
// half per texel for the FP16 form's warped image, read back as float).
// Objects are created once per (pointer, geometry, filter, element) and kept for the
// life of the cache, so a launch never creates or destroys one.
class TexCache {
 public:
  ~TexCache() { clear(); }
  // comps: 1 float, 2 float2, kHalf1 one half per texel
  static constexpr int kHalf1 = -1;
  cudaTextureObject_t get(const void* ptr, int w, int h, size_t pitchBytes, int comps, bool linear) {
    Key k{(uintptr_t)ptr, w, h, pitchBytes, comps, linear};
    auto it = map_.find(k);
    if (it != map_.end()) return it->second;
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = const_cast<void*>(ptr);
    rd.res.pitch2D.desc = comps == 2        ? cudaCreateChannelDesc<float2>()
                          : comps == kHalf1 ? cudaCreateChannelDescHalf()
                                            : cudaCreateChannelDesc<float>();
    rd.res.pitch2D.width = w;
    rd.res.pitch2D.height = h;
    rd.res.pitch2D.pitchInBytes = pitchBytes;
    cudaTextureDesc td = {};
    td.addressMode[0] = cudaAddressModeMirror;
    td.addressMode[1] = cudaAddressModeMirror;
    td.filterMode = linear ? cudaFilterModeLinear : cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    cudaTextureObject_t t = 0;
    VFS_CUDA(cudaCreateTextureObject(&t, &rd, &td, nullptr));
    map_[k] = t;
    return t;
  }
  void clear() {
    for (auto& kv : map_) cudaDestroyTextureObject(kv.second);
    map_.clear();
  }

 private:
  typedef std::tuple<uintptr_t, int, int, size_t, int, bool> Key;
  std::map<Key, cudaTextureObject_t> map_;
};

}  // namespace vfs
