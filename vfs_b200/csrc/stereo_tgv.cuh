// Host-side solver object behind the C ABI (include/vfs_b200.h) and the C++ class
// (include/stereotgv.h).  It owns the device state of one camera pair and runs the
// reference's coarse-to-fine schedule on its CUDA stream.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "common.cuh"
#include "fused.cuh"
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
  kFused = 1,      // fused kernels (one or several iterations per launch), CUDA graphs
};

class StereoTgvImpl;

// physical buffers that the solve's pointer swaps move between roles
struct PairPtrs {
  float *pI1_0, *i1cal, *u, *us, *u_, *u_s;
  float2 *v_, *v_s, *warpUV, *warpUVs;
  void *vh, *vhs;
};

// Runs the fused path for a set of pairs, optionally through a cache of captured
// CUDA graphs (one per batch composition and pointer state).
class FusedEngine {
 public:
  bool use_graph = true;
  bool autotune = true;  // pick the iteration kernel's tile variant per level on first use
  int forced_variant = -1;  // >= 0: this iteration-kernel variant at every level (no tuning)
  std::vector<int> forced_levels;  // non-empty: variant per level, finest first (no tuning)
  int concurrency = 1;      // one-pair solves run at the same time (set by a concurrent batch)
  // tuned tile variant per level, keyed by batch composition (form, storage, sizes)
  const std::map<std::vector<int>, std::vector<int>>& tuned() const { return tuned_; }
  ~FusedEngine();
  void clear();
  // part: 0 whole solve; 1 everything before the full-resolution level; 2 that level alone
  void solve(std::vector<StereoTgvImpl*>& pairs, bool masked, bool half, cudaStream_t st, int part = 0);
 private:
  void solve_parts(std::vector<StereoTgvImpl*>& pairs, bool masked, bool half, cudaStream_t st, int part);
 public:
  // allocate fused buffers and refresh edge codes, each on the pair's own stream
  static void prepare(std::vector<StereoTgvImpl*>& pairs, bool masked);
  size_t graphs() const { return cache_.size(); }
  // iteration-kernel variant per pyramid level (finest first) of the last solve
  std::vector<int> last_variants;
  void note_variants(const std::vector<int>& v, int part);

 private:
  struct Entry {
    cudaGraphExec_t exec = nullptr;
    long long kernels = 0;  // kernel launches recorded in the graph (added to the launch count per replay)
    std::vector<PairPtrs> after;
    std::vector<ProfRec> prof;
    std::vector<cudaEvent_t> events;
    std::vector<std::pair<const StereoTgvImpl*, uint64_t>> owners;  // pairs and their generation
    uint64_t last_use = 0;
  };
  // Graphs of a pair captured under an older generation (an earlier mask, initialize or state
  // import) are destroyed when the pair is next solved, and at most kMaxGraphs are kept (the
  // least recently replayed go first), so a long-running server whose batch compositions keep
  // changing holds a bounded number of graph executables.
  static constexpr size_t kMaxGraphs = 64;
  void evict(const std::vector<StereoTgvImpl*>& pairs);
  void drop(std::map<std::vector<uintptr_t>, Entry>::iterator it);
  uint64_t use_clock_ = 0;
  std::map<std::vector<uintptr_t>, Entry> cache_;
  std::map<std::vector<int>, std::vector<int>> tuned_;
};

// process-wide counter of handle states (StereoTgvImpl::generation)
uint64_t next_generation();
// allocation-failure injection for tests (vfs_debug_fail_allocation)
std::atomic<int>& alloc_failure_countdown();

// Device bytes a pair of this geometry allocates: the solver pool, and with `fused`
// also the fused-path buffers.  Matches StereoTgvImpl::initialize / ensureFused.
size_t estimate_device_bytes(int width, int height, int nLevels, float fScale, int strideAlignment, bool fused);

class StereoTgvImpl {
 public:
  StereoTgvImpl(int blockWidth, int blockHeight, int strideAlignment);
  ~StereoTgvImpl();

  void initialize(const SolverParams& p);
  // a handle runs on its own non-blocking stream unless the caller sets one
  void setStream(cudaStream_t st) { stream_ = st ? st : own_stream(); }
  cudaStream_t stream() const { return stream_; }
  bool initialized() const { return initialized_; }

  void loadVectorFields(const float* tv_host, const float* cv_host);
  void copyMaskToDevice(const float* mask_host);
  void copyImagesU8(const uint8_t* i0, const uint8_t* i1, bool device_src);
  void copyImagesF32(const float* i0, const float* i1);
  void copyImagesU8C3(const uint8_t* i0, const uint8_t* i1);
  void solve(bool masked);
  void copyOut(const char* what, float* dst, bool to_host);
  // stream-ordered forms on a given stream (no synchronisation): the batched host-buffer solve
  void copyImagesU8On(const uint8_t* i0, const uint8_t* i1, cudaMemcpyKind kind, cudaStream_t st);
  void copyOutOn(const char* what, float* dst, cudaMemcpyKind kind, cudaStream_t st);
  void convertKB(float fx, float fy, float cx, float cy, float d1, float d2, float d3, float d4, float t1, float t2,
                 float t3);
  void flowToHSV(float flowscale);
  void debugGet(const char* name, int comps, float* out_host);

  SolverParams P;
  float baseline = 0.0f, focal = 0.0f;
  // ---- warm start (opt-in; the reference zeroes u, u-bar and warpUV at every solve,
  // stereotgv.cu:395-397) ---------------------------------------------------------
  // warm_level < 0: off.  Otherwise, once a frame has been solved, the next solve starts at
  // pyramid level min(warm_level, levels - 1) from the previous frame's disparity; the levels
  // above it are skipped.
  int warm_level = -1;
  bool have_prev = false;  // d_u holds the disparity of the last solved frame (full resolution)
  bool warmStart() const { return warm_level >= 0 && have_prev; }
  int topLevel() const {
    return (warm_level >= 0 && have_prev) ? std::min(warm_level, levels() - 1) : levels() - 1;
  }
  // State at the start of a solve whose first level is `top`: cold (top = levels - 1 and no
  // warm start) zeroes u, u-bar and warpUV as the reference does; warm brings the previous
  // disparity to level `top` (box downscale, values / fScale per level), sets u-bar = u and
  // zeroes warpUV (the first level derives it from u).
  void startState(int top, cudaStream_t st);

  // ---- state export / import (no counterpart in the reference) ------------------
  // The whole device state of the handle (both pools, which physical buffer holds each
  // ping-pong role, the warm-start flag), so that a handle initialised with the same geometry
  // continues bit for bit where the exported one stopped.  Host settings (limit range,
  // camera, solve path, stream) are not part of it.
  size_t stateBytes() const;
  void exportState(void* host, size_t bytes);
  void importState(const void* host, size_t bytes);
  // tensor weight from CUDA's expf / powf as the reference (1, default) or from the portable
  // exp / log of tgv_math.cuh that the CPU oracle restates bit for bit (0)
  int tensor_cuda_math = 1;
  bool visualizeResults = false;
  int blockWidth, blockHeight, strideAlignment;
  int width = 0, height = 0, stride = 0;
  std::vector<int> pW, pH, pS;
  SolvePath path = SolvePath::kReference;
  bool half_storage = false;  // fused path: p, q, v-bar and the warped image stored as half
  // d_i1warp holds half values at the level-0 stride (the last solve was the fused path with
  // half storage); copies of the warped image widen them to float
  bool i1warp_half = false;
  std::string last_error;

  // ---- fused-path state (allocated on first use) ------------------------------
  // p and q: two planes each (read one, write the other per iteration), float or
  // half; v-bar in half storage: its own ping-pong pair (float storage uses d_v_ /
  // d_v_s); edge codes per level for the masked and the plain form.
  void ensureFused();
  void* f_p = nullptr;
  void* f_q = nullptr;
  void* f_vh = nullptr;  // current half v-bar
  void* f_vhs = nullptr; // other half v-bar
  // half storage: the current level's coefficient records of the iteration (IterPair::abce, rv)
  float4* f_abce = nullptr;
  float2* f_rv = nullptr;
  std::vector<uint8_t*> code_masked, code_plain;
  bool codes_valid = false;
  // per level: the K-iterations-per-launch kernel reproduces the masked form exactly (false
  // only when the row has no padding and a pixel of column 0 is on; kernels_tb.cu)
  std::vector<uint8_t> tb_ok;
  // per level (masked form): no pixel of column 0 is on, so no pixel reads west of the image
  // (where the reference reads the previous row's last element); the TMA iteration kernel,
  // whose copies are two-dimensional, is used only there
  std::vector<uint8_t> tma_ok;
  // per one-iteration tile variant (0-2) and level: for each tile row, the first and last
  // tile column whose region (tile + west / north halo) holds a pixel that is on (masked
  // form; first > last for a row without any)
  std::vector<std::vector<uint16_t>> span_lo[kIterSpanSlots], span_hi[kIterSpanSlots];
  // per tile row, the run of tiles whose region is all interior pixels (IterArgs::in_lo / in_hi)
  std::vector<std::vector<uint16_t>> inner_lo[kIterSpanSlots], inner_hi[kIterSpanSlots];
  int f_parity = 0;      // which p / q plane holds the latest values
  int levels() const { return (int)pW.size(); }
  Geom geomAt(int level) const { return Geom{pW[level], pH[level], pS[level]}; }
  cudaTextureObject_t tex1(const float* p, int level, bool linear = true) { return t1(p, level, linear); }
  cudaTextureObject_t tex2(const float2* p, int level) { return t2(p, level); }
  // a plane holding one half per pixel at the level's stride (linear filtering)
  cudaTextureObject_t tex1h(const void* p, int level) {
    return tex.get(p, pW[level], pH[level], (size_t)pS[level] * sizeof(__half), TexCache::kHalf1, true);
  }
  size_t fullElems() const { return full_; }

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
  // Guard zones: kGuardBytes of kGuardByte after every device plane of both pools, written at
  // allocation; checkGuards() counts the zones a kernel has written into (out-of-bounds
  // stores), vfs_debug_check_guards in the C ABI.
  static constexpr size_t kGuardBytes = 256;
  static constexpr unsigned char kGuardByte = 0xA5;
  int checkGuards();
  TexCache tex;

  // ---- opt-in event timing of launch groups (bench / profiling) -----------
  bool profiling = false;
  void profReset();
  // Sum over records of `tag` (kProf*): count, total milliseconds, pixel-iterations.
  void profRead(int tag, long long* count, double* total_ms, double* pixel_iters);
  std::vector<ProfRec> profRecords() const { return prof_; }
  void setProfRecords(const std::vector<ProfRec>& r) { prof_ = r; }
  // while a graph is captured, profiling events are created here (owned by the graph)
  std::vector<cudaEvent_t>* capture_events = nullptr;
  FusedEngine engine;  // single-pair fused solves
  // renewed by every initialize and every rebuild of the edge codes (a new mask): the tile
  // spans and the multi-iteration levels baked into captured graphs follow the mask
  uint64_t generation = 0;

 private:
  void release();
  float* alloc(size_t bytes);
  void fillGuards(size_t from, cudaStream_t st);
  std::vector<char*> guards_;
  Geom geom(int level) const { return Geom{pW[level], pH[level], pS[level]}; }
  cudaTextureObject_t t1(const float* p, int level, bool linear = true) {
    return tex.get(p, pW[level], pH[level], (size_t)pS[level] * sizeof(float), 1, linear);
  }
  cudaTextureObject_t t2(const float2* p, int level) {
    return tex.get(p, pW[level], pH[level], (size_t)pS[level] * sizeof(float2), 2, true);
  }
  void solveReference(bool masked);

 public:
  cudaEvent_t profEvent();
  void profBegin(int tag, int level, int iters);
  // st: the stream the timed work is queued on (the handle's stream when 0)
  // launches: kernel launches in the group (0: one per iteration)
  void profBeginPx(int tag, long long px, int iters, cudaStream_t st = 0, int launches = 0);
  void profEnd(cudaStream_t st = 0);

 private:
  std::vector<ProfRec> prof_;
  std::vector<cudaEvent_t> evpool_;
  size_t evused_ = 0;

  cudaStream_t own_stream();
  bool initialized_ = false;
  cudaStream_t own_stream_ = nullptr;
  cudaStream_t stream_ = 0;
  char* fpool_ = nullptr;
  char* pool_ = nullptr;
  size_t pool_bytes_ = 0, pool_used_ = 0;
  size_t full_ = 0;  // elements of a full-resolution pitched plane
};

}  // namespace vfs
