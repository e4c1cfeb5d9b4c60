// extern "C" layer over StereoTgvImpl (declarations in include/vfs_b200.h).
// Every entry point converts exceptions into a status code and records the
// message on the handle; nothing here exits the process.
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <string>

#include "../../include/vfs_b200.h"
#include "hist.cuh"
#include "io.hpp"
#include "stereo_tgv.cuh"

struct vfs_batch {
  std::vector<vfs_stereo*> members;
  vfs::FusedEngine engine;
  cudaStream_t stream = 0;      // the batch's stream (its own unless set)
  cudaStream_t own = nullptr;
  cudaEvent_t done = nullptr;   // batch work finished (members' streams wait on it)
  cudaEvent_t start = nullptr;  // members' inputs ready (the concurrent streams wait on it)
  std::vector<cudaEvent_t> ready;  // member work finished (the batch stream waits on them)
  std::vector<cudaStream_t> lanes;     // concurrent mode: one stream per member slot
  std::vector<cudaEvent_t> lane_done;  // concurrent mode: per-slot completion
  std::vector<cudaEvent_t> fine_done;  // concurrent mode: per-slot end of the full-resolution part
  std::vector<cudaEvent_t> coarse_done;  // concurrent mode: per-slot end of the coarse part
  std::vector<cudaStream_t> fine_lanes;  // concurrent mode: streams of the full-resolution parts
  int fine_limit = -1;  // concurrent mode: pairs at full resolution at once (0: no limit, -1: auto)
  bool stagger_coarse = false;  // coarse parts also S at a time, one slot ahead of the fine parts
  int fine_priority = 4;  // 0: no priorities; 1: full-resolution parts on high-priority
                          // streams; 2: also the coarse parts of the first max_pairs pairs; 3:
                          // every part of pair k at the priority of its full-resolution round
                          // k / max_pairs; 4 (default): coarse parts above full-resolution parts
  std::map<int, std::vector<cudaStream_t>> graded_lanes;  // priority 3: per priority, one stream per slot
  int mode = VFS_BATCH_CONCURRENT;
  bool half = false;
  std::string err;
  ~vfs_batch() {
    engine.clear();
    for (auto e : ready) cudaEventDestroy(e);
    for (auto e : lane_done) cudaEventDestroy(e);
    for (auto e : fine_done) cudaEventDestroy(e);
    for (auto e : coarse_done) cudaEventDestroy(e);
    for (auto l : fine_lanes) cudaStreamDestroy(l);
    for (auto& g : graded_lanes)
      for (auto l : g.second) cudaStreamDestroy(l);
    for (auto l : lanes) cudaStreamDestroy(l);
    if (done) cudaEventDestroy(done);
    if (start) cudaEventDestroy(start);
    if (own) cudaStreamDestroy(own);
  }
};

struct vfs_stereo {
  vfs::StereoTgvImpl impl;
  std::string err;
  // SolveStereo scratch (device): 2 images, histogram and LUT
  uint8_t* d_eq = nullptr;
  unsigned int* d_hist = nullptr;
  size_t eq_bytes = 0;
  vfs_stereo(int bw, int bh, int sa) : impl(bw, bh, sa) {}
  ~vfs_stereo() {
    if (d_eq) cudaFree(d_eq);
  }
};

namespace {

thread_local std::string g_create_error;

template <class H, class F>
int guarded(H* s, F&& f) {
  if (!s) return VFS_ERR_ARG;
  try {
    f();
    return VFS_OK;
  } catch (const vfs::CudaError& e) {
    s->err = std::string("CUDA error ") + cudaGetErrorString(e.err) + " in " + e.what;
    (void)cudaGetLastError();
    return e.err == cudaErrorMemoryAllocation ? VFS_ERR_NOMEM : VFS_ERR_CUDA;
  } catch (const vfs::ArgError& e) {
    s->err = e.msg;
    return VFS_ERR_ARG;
  } catch (const std::bad_alloc&) {
    s->err = "host allocation failed";
    return VFS_ERR_NOMEM;
  } catch (...) {
    s->err = "unknown error";
    return VFS_ERR_CUDA;
  }
}

}  // namespace

namespace vfs {
// message of the last failure of a call that has no handle (read with vfs_last_error(NULL))
void set_global_error(const char* msg) { g_create_error = msg; }
}  // namespace vfs

extern "C" {

const char* vfs_status_string(int st) {
  switch (st) {
    case VFS_OK: return "ok";
    case VFS_ERR_ARG: return "invalid argument";
    case VFS_ERR_CUDA: return "CUDA error";
    case VFS_ERR_STATE: return "invalid call order";
    case VFS_ERR_NOMEM: return "out of device memory";
    case VFS_ERR_IO: return "file error";
    case VFS_ERR_TIMEOUT: return "device wait timed out";
    case VFS_ERR_BUSY: return "not enough free device memory";
    default: return "unknown status";
  }
}

const char* vfs_last_error(const vfs_stereo* s) { return s ? s->err.c_str() : g_create_error.c_str(); }

int vfs_version(void) { return 100; }

int vfs_create_ex(vfs_stereo** out, int bw, int bh, int sa) {
  if (!out) return VFS_ERR_ARG;
  *out = nullptr;
  if (bw <= 0 || bh <= 0 || sa <= 0) {
    g_create_error = "vfs_create_ex: block and stride alignment must be positive";
    return VFS_ERR_ARG;
  }
  vfs_stereo* s = new (std::nothrow) vfs_stereo(bw, bh, sa);
  if (!s) return VFS_ERR_NOMEM;
  *out = s;
  return VFS_OK;
}

int vfs_create(vfs_stereo** out) { return vfs_create_ex(out, 32, 1, 32); }

int vfs_destroy(vfs_stereo* s) {
  if (!s) return VFS_ERR_ARG;
  cudaStreamSynchronize(s->impl.stream());
  delete s;
  return VFS_OK;
}

int vfs_set_stream(vfs_stereo* s, void* st) {
  return guarded(s, [&] { s->impl.setStream((cudaStream_t)st); });
}

int vfs_synchronize(vfs_stereo* s) {
  return guarded(s, [&] { VFS_CUDA(cudaStreamSynchronize(s->impl.stream())); });
}

int vfs_initialize(vfs_stereo* s, int width, int height, float beta, float gamma, float alpha0, float alpha1,
                   float timestep_lambda, float lambda, int nLevels, float fScale, int nWarpIters,
                   int nSolverIters) {
  return guarded(s, [&] {
    vfs::SolverParams p;
    p.width = width;
    p.height = height;
    p.beta = beta;
    p.gamma = gamma;
    p.alpha0 = alpha0;
    p.alpha1 = alpha1;
    p.timestep_lambda = timestep_lambda;
    p.lambda = lambda;
    p.nLevels = nLevels;
    p.fScale = fScale;
    p.nWarpIters = nWarpIters;
    p.nSolverIters = nSolverIters;
    p.limitRange = s->impl.P.limitRange;
    s->impl.initialize(p);
  });
}

int vfs_set_limit_range(vfs_stereo* s, float lr) {
  return guarded(s, [&] {
    if (s->impl.P.limitRange != lr) s->impl.generation = vfs::next_generation();  // captured graphs hold it
    s->impl.P.limitRange = lr;
  });
}

int vfs_cached_graphs(const vfs_stereo* s) { return s ? (int)s->impl.engine.graphs() : VFS_ERR_ARG; }
int vfs_batch_cached_graphs(const vfs_batch* b) { return b ? (int)b->engine.graphs() : VFS_ERR_ARG; }
long long vfs_tuning_solves(void) { return vfs::tuning_solve_count(); }

int vfs_set_warm_start(vfs_stereo* s, int level) {
  return guarded(s, [&] {
    if (level < -1) throw vfs::ArgError{"vfs_set_warm_start: level must be -1 (off) or >= 0"};
    s->impl.warm_level = level;
  });
}

size_t vfs_state_bytes(const vfs_stereo* s) { return s ? s->impl.stateBytes() : 0; }

int vfs_export_state(vfs_stereo* s, void* host, size_t bytes) {
  return guarded(s, [&] { s->impl.exportState(host, bytes); });
}

int vfs_import_state(vfs_stereo* s, const void* host, size_t bytes) {
  return guarded(s, [&] { s->impl.importState(host, bytes); });
}

int vfs_debug_fail_allocation(int n) {
  if (n < 0) return VFS_ERR_ARG;
  vfs::alloc_failure_countdown().store(n);
  return VFS_OK;
}

int vfs_set_tensor_math(vfs_stereo* s, int mode) {
  return guarded(s, [&] {
    if (mode != VFS_TENSOR_MATH_CUDA && mode != VFS_TENSOR_MATH_PORTABLE)
      throw vfs::ArgError{"vfs_set_tensor_math: mode must be VFS_TENSOR_MATH_CUDA or VFS_TENSOR_MATH_PORTABLE"};
    const int cuda_math = mode == VFS_TENSOR_MATH_CUDA ? 1 : 0;
    if (s->impl.tensor_cuda_math != cuda_math) s->impl.generation = vfs::next_generation();
    s->impl.tensor_cuda_math = cuda_math;
  });
}

int vfs_set_camera(vfs_stereo* s, float baseline, float focal) {
  return guarded(s, [&] {
    s->impl.baseline = baseline;
    s->impl.focal = focal;
  });
}

int vfs_get_level_size(const vfs_stereo* cs, int level, int* w, int* h, int* st) {
  vfs_stereo* s = const_cast<vfs_stereo*>(cs);
  return guarded(s, [&] {
    if (!s->impl.initialized()) throw vfs::ArgError{"get_level_size before initialize"};
    if (level < 0 || level >= (int)s->impl.pW.size()) throw vfs::ArgError{"level out of range"};
    if (w) *w = s->impl.pW[level];
    if (h) *h = s->impl.pH[level];
    if (st) *st = s->impl.pS[level];
  });
}

int vfs_load_vector_fields(vfs_stereo* s, const float* tv, const float* cv) {
  return guarded(s, [&] { s->impl.loadVectorFields(tv, cv); });
}

int vfs_copy_mask_to_device(vfs_stereo* s, const float* mask) {
  return guarded(s, [&] { s->impl.copyMaskToDevice(mask); });
}

int vfs_copy_images_to_device_u8(vfs_stereo* s, const uint8_t* i0, const uint8_t* i1) {
  vfs::TraceRange r("vfs_copy_images_to_device");
  return guarded(s, [&] { s->impl.copyImagesU8(i0, i1, false); });
}

int vfs_copy_images_to_device_f32(vfs_stereo* s, const float* i0, const float* i1) {
  return guarded(s, [&] { s->impl.copyImagesF32(i0, i1); });
}

int vfs_copy_images_to_device_u8c3(vfs_stereo* s, const uint8_t* i0, const uint8_t* i1) {
  return guarded(s, [&] { s->impl.copyImagesU8C3(i0, i1); });
}

int vfs_copy_images_from_device_u8(vfs_stereo* s, const uint8_t* d0, const uint8_t* d1) {
  return guarded(s, [&] { s->impl.copyImagesU8(d0, d1, true); });
}

int vfs_solve_stereo_forward(vfs_stereo* s) {
  vfs::TraceRange r("vfs_solve_stereo_forward");
  return guarded(s, [&] { s->impl.solve(false); });
}

int vfs_solve_stereo_forward_masked(vfs_stereo* s) {
  vfs::TraceRange r("vfs_solve_stereo_forward_masked");
  return guarded(s, [&] { s->impl.solve(true); });
}

int vfs_debug_check_guards(vfs_stereo* s, int* bad_zones) {
  return guarded(s, [&] {
    if (!bad_zones) throw vfs::ArgError{"check guards: null output"};
    *bad_zones = s->impl.checkGuards();
  });
}

int vfs_copy_1d_disparity_to_host(vfs_stereo* s, float* u) {
  vfs::TraceRange r("vfs_copy_1d_disparity_to_host");
  return guarded(s, [&] { s->impl.copyOut("u", u, true); });
}

int vfs_copy_disparity_to_host(vfs_stereo* s, float* uv) {
  return guarded(s, [&] { s->impl.copyOut("warpUV", uv, true); });
}

int vfs_copy_warped_image_to_host(vfs_stereo* s, float* im) {
  return guarded(s, [&] { s->impl.copyOut("i1warp", im, true); });
}

int vfs_copy_1d_disparity_to_device(vfs_stereo* s, float* d_u) {
  return guarded(s, [&] { s->impl.copyOut("u", d_u, false); });
}

int vfs_copy_disparity_to_device(vfs_stereo* s, float* d_uv) {
  return guarded(s, [&] { s->impl.copyOut("warpUV", d_uv, false); });
}

int vfs_copy_stereo_to_host(vfs_stereo* s, float* depth, float* X, float fx, float fy, float cx, float cy, float d1,
                            float d2, float d3, float d4, float t1, float t2, float t3) {
  return guarded(s, [&] {
    s->impl.convertKB(fx, fy, cx, cy, d1, d2, d3, d4, t1, t2, t3);
    if (depth) s->impl.copyOut("depth", depth, true);
    if (X) s->impl.copyOut("X", X, true);
    VFS_CUDA(cudaStreamSynchronize(s->impl.stream()));
  });
}

int vfs_copy_disparity_vis_to_host(vfs_stereo* s, float* rgb, float flow_scale) {
  return guarded(s, [&] {
    s->impl.flowToHSV(flow_scale);
    s->impl.copyOut("rgb", rgb, true);
  });
}

int vfs_debug_get_buffer(vfs_stereo* s, const char* name, int comps, float* out) {
  return guarded(s, [&] {
    if (!name || !out) throw vfs::ArgError{"debug get: null argument"};
    s->impl.debugGet(name, comps, out);
  });
}

int vfs_set_solve_path(vfs_stereo* s, int path, int half_storage) {
  return guarded(s, [&] {
    if (path != VFS_PATH_REFERENCE && path != VFS_PATH_FUSED) throw vfs::ArgError{"unknown solve path"};
    if (path == VFS_PATH_REFERENCE && half_storage) throw vfs::ArgError{"half storage needs the fused path"};
    s->impl.path = path == VFS_PATH_FUSED ? vfs::SolvePath::kFused : vfs::SolvePath::kReference;
    s->impl.half_storage = half_storage != 0;
  });
}

int vfs_set_graph(vfs_stereo* s, int use_graph) {
  return guarded(s, [&] { s->impl.engine.use_graph = use_graph != 0; });
}

size_t vfs_estimate_device_bytes(int width, int height, int nLevels, float fScale, int sa, int fused) {
  return vfs::estimate_device_bytes(width, height, nLevels, fScale, sa, fused != 0);
}

int vfs_batch_create(vfs_batch** out) {
  if (!out) return VFS_ERR_ARG;
  *out = new (std::nothrow) vfs_batch();
  if (!*out) return VFS_ERR_NOMEM;
  if (cudaStreamCreateWithFlags(&(*out)->own, cudaStreamNonBlocking) != cudaSuccess) {
    (void)cudaGetLastError();
    delete *out;
    *out = nullptr;
    return VFS_ERR_CUDA;
  }
  (*out)->stream = (*out)->own;
  return VFS_OK;
}

int vfs_batch_destroy(vfs_batch* b) {
  if (!b) return VFS_ERR_ARG;
  cudaStreamSynchronize(b->stream);
  delete b;
  return VFS_OK;
}

const char* vfs_batch_last_error(const vfs_batch* b) { return b ? b->err.c_str() : ""; }

int vfs_batch_set_stream(vfs_batch* b, void* st) {
  return guarded(b, [&] {
    VFS_CUDA(cudaStreamSynchronize(b->stream));
    b->stream = st ? (cudaStream_t)st : b->own;
    b->engine.clear();
  });
}

int vfs_batch_add(vfs_batch* b, vfs_stereo* s) {
  return guarded(b, [&] {
    if (!s) throw vfs::ArgError{"batch add: null handle"};
    if ((int)b->members.size() >= vfs::kMaxPairs) throw vfs::ArgError{"batch is full"};
    for (auto* m : b->members)
      if (m == s) throw vfs::ArgError{"batch add: handle already in the batch"};
    if (!s->impl.initialized()) throw vfs::ArgError{"batch add: handle not initialized"};
    cudaEvent_t e;
    VFS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ready.push_back(e);
    b->members.push_back(s);
    b->engine.clear();
  });
}

int vfs_batch_clear(vfs_batch* b) {
  return guarded(b, [&] {
    VFS_CUDA(cudaStreamSynchronize(b->stream));
    b->members.clear();
    b->engine.clear();
    for (auto e : b->ready) cudaEventDestroy(e);
    b->ready.clear();
  });
}

int vfs_batch_size(const vfs_batch* b) { return b ? (int)b->members.size() : VFS_ERR_ARG; }

int vfs_batch_set_storage(vfs_batch* b, int half) {
  return guarded(b, [&] { b->half = half != 0; });
}

int vfs_batch_set_graph(vfs_batch* b, int use_graph) {
  return guarded(b, [&] { b->engine.use_graph = use_graph != 0; });
}

int vfs_batch_set_autotune(vfs_batch* b, int on) {
  return guarded(b, [&] { b->engine.autotune = on != 0; });
}

int vfs_set_autotune(vfs_stereo* s, int on) {
  return guarded(s, [&] { s->impl.engine.autotune = on != 0; });
}

int vfs_set_iteration_variant(vfs_stereo* s, int variant) {
  return guarded(s, [&] {
    if (variant != -1 && !vfs::iter_variant_valid(variant)) throw vfs::ArgError{"iteration variant out of range or retired"};
    s->impl.engine.forced_variant = variant;
  });
}

namespace {
std::vector<int> checked_levels(const int* variants, int n) {
  if (n < 0 || n > 32 || (n > 0 && !variants)) throw vfs::ArgError{"invalid per-level variant list"};
  std::vector<int> v(variants, variants + n);
  for (int x : v)
    if (!vfs::iter_variant_valid(x)) throw vfs::ArgError{"iteration variant out of range or retired"};
  return v;
}
}  // namespace

int vfs_set_iteration_variants(vfs_stereo* s, const int* variants, int n_levels) {
  return guarded(s, [&] { s->impl.engine.forced_levels = checked_levels(variants, n_levels); });
}

int vfs_batch_set_iteration_variants(vfs_batch* b, const int* variants, int n_levels) {
  return guarded(b, [&] { b->engine.forced_levels = checked_levels(variants, n_levels); });
}

int vfs_get_iteration_variants(vfs_stereo* s, int* variants, int max_levels, int* count) {
  return guarded(s, [&] {
    const std::vector<int>& v = s->impl.engine.last_variants;
    if (count) *count = (int)v.size();
    for (int l = 0; l < max_levels && l < (int)v.size(); l++) variants[l] = v[l];
  });
}

int vfs_batch_set_iteration_variant(vfs_batch* b, int variant) {
  return guarded(b, [&] {
    if (variant != -1 && !vfs::iter_variant_valid(variant)) throw vfs::ArgError{"iteration variant out of range or retired"};
    b->engine.forced_variant = variant;
  });
}

int vfs_batch_set_fine_concurrency(vfs_batch* b, int max_pairs) {
  return guarded(b, [&] {
    if (max_pairs < -1) throw vfs::ArgError{"fine concurrency must be >= -1"};
    b->fine_limit = max_pairs;
  });
}

int vfs_batch_set_pipeline(vfs_batch* b, int stagger_coarse, int priority) {
  return guarded(b, [&] {
    if (priority < 0 || priority > 4) throw vfs::ArgError{"pipeline priority must be 0 to 4"};
    b->stagger_coarse = stagger_coarse != 0;
    b->fine_priority = priority;
  });
}

int vfs_batch_set_mode(vfs_batch* b, int mode) {
  return guarded(b, [&] {
    if (mode != VFS_BATCH_CONCURRENT && mode != VFS_BATCH_ONE_LAUNCH) throw vfs::ArgError{"unknown batch mode"};
    b->mode = mode;
  });
}

}  // extern "C"

namespace {

// Host buffers of a batched solve from and to host memory (null: device-resident inputs
// already copied by the caller, outputs left on the device).
struct BatchHostIO {
  const uint8_t* const* i0 = nullptr;
  const uint8_t* const* i1 = nullptr;
  float* const* u = nullptr;
  bool device = false;  // the buffers are in device memory (copies stay on the device)
};

void batch_solve(vfs_batch* b, int masked, const BatchHostIO* io) {
  vfs::TraceRange trace("vfs_batch_solve");
  if (b->members.empty()) throw vfs::ArgError{"batch solve: empty batch"};
  std::vector<vfs::StereoTgvImpl*> pairs;
  for (auto* m : b->members) pairs.push_back(&m->impl);
  if (io) {
    for (size_t k = 0; k < pairs.size(); k++)
      if (!io->i0[k] || !io->i1[k] || !io->u[k]) throw vfs::ArgError{"batch solve: null host buffer"};
  }
  // per-pair preparation on each member's own stream, then order the batch stream
  // after every member's queued work and every member's stream after the batch
  vfs::FusedEngine::prepare(pairs, masked != 0);
  if (!b->done) VFS_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
  for (size_t k = 0; k < pairs.size(); k++) {
    if (pairs[k]->stream() == b->stream) continue;
    VFS_CUDA(cudaEventRecord(b->ready[k], pairs[k]->stream()));
    VFS_CUDA(cudaStreamWaitEvent(b->stream, b->ready[k], 0));
  }
  if (b->mode == VFS_BATCH_ONE_LAUNCH) {
    if (io)
      for (size_t k = 0; k < pairs.size(); k++)
        pairs[k]->copyImagesU8On(io->i0[k], io->i1[k], io->device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, b->stream);
    b->engine.solve(pairs, masked != 0, b->half, b->stream);
    if (io)
      for (size_t k = 0; k < pairs.size(); k++)
        pairs[k]->copyOutOn("u", io->u[k], io->device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, b->stream);
  } else {
    // fork: every pair's upload, solve (its own graph) and download on its own slot
    // stream, then join; one pair's copies overlap the other pairs' solves
    if (!b->start) VFS_CUDA(cudaEventCreateWithFlags(&b->start, cudaEventDisableTiming));
    while (b->lanes.size() < pairs.size()) {
      cudaStream_t l;
      VFS_CUDA(cudaStreamCreateWithFlags(&l, cudaStreamNonBlocking));
      b->lanes.push_back(l);
      cudaEvent_t e;
      VFS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      b->lane_done.push_back(e);
      VFS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      b->fine_done.push_back(e);
      VFS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      b->coarse_done.push_back(e);
      int lo = 0, hi = 0;  // numerically lower priority values are higher priorities
      VFS_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
      VFS_CUDA(cudaStreamCreateWithPriority(&l, cudaStreamNonBlocking, hi));
      b->fine_lanes.push_back(l);
    }
    const int n = (int)pairs.size();
    // With a limit S on the pairs at full resolution, each pair's solve is enqueued as two
    // graphs: the coarse levels of every pair start together, and pair k's full-resolution
    // level waits for pair k - S's, so that at most S full-resolution working sets compete
    // for L2 while the other pairs run their coarse levels.
    int S = b->fine_limit;
    if (S < 0) {
      // auto: as many full-resolution working sets as fit in three quarters of L2, at least
      // two (per pixel: the iteration's reads and the other ping-pong planes it writes)
      int dev = 0, l2 = 0;
      VFS_CUDA(cudaGetDevice(&dev));
      VFS_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
      double ws = 0;
      for (auto* p : pairs) ws = std::max(ws, (double)p->width * p->height * (b->half ? 69.0 : 101.0));
      // no split when fewer than two working sets fit (the limit then only serialises)
      S = ws > 0 ? (int)(0.75 * l2 / ws) : 0;
      if (S < 2) S = 0;
    }
    const bool split = S > 0 && S < n;
    int prio_lo = 0, prio_hi = 0;
    VFS_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    // priority 3: pair k's coarse and full-resolution parts run at the priority of its
    // full-resolution round k / S (round 0 the highest), so that the GPU prefers the work of the
    // earliest round and the later rounds' coarse levels fill the gaps its launches leave
    // priority 4: the coarse parts, latency-bound chains of small launches, run above the
    // full-resolution parts (the first round's coarse parts highest), so that every pair's
    // chain advances at its own pace and the full-resolution launches fill the rest of the GPU
    const bool graded = split && (b->fine_priority == 3 || b->fine_priority == 4);
    const bool coarse_first = b->fine_priority == 4;
    auto round_prio = [&](int k) {
      if (coarse_first) return std::min(prio_lo, prio_hi + (k < S ? 0 : 1));
      return std::min(prio_lo, prio_hi + k / S);
    };
    auto graded_lane = [&](int k) -> cudaStream_t {
      std::vector<cudaStream_t>& v = b->graded_lanes[round_prio(k)];
      while ((int)v.size() <= k) {
        cudaStream_t l;
        VFS_CUDA(cudaStreamCreateWithPriority(&l, cudaStreamNonBlocking, round_prio(k)));
        v.push_back(l);
      }
      return v[k];
    };
    // prio: the priority the launches of this part carry (0: none)
    auto run = [&](int k, int part, int concurrency, cudaStream_t lane, int prio = 0) {
      struct PrioScope {
        int old;
        PrioScope(int p) : old(vfs::launch_priority()) { vfs::launch_priority() = p; }
        ~PrioScope() { vfs::launch_priority() = old; }
      } prio_scope(prio);
      std::vector<vfs::StereoTgvImpl*> one{pairs[k]};
      vfs::FusedEngine& eng = pairs[k]->engine;
      const bool g = eng.use_graph, t = eng.autotune;
      const int fv = eng.forced_variant, cc = eng.concurrency;
      const std::vector<int> fl = eng.forced_levels;
      eng.use_graph = b->engine.use_graph;
      eng.autotune = b->engine.autotune;
      eng.forced_variant = b->engine.forced_variant;
      eng.forced_levels = b->engine.forced_levels;
      eng.concurrency = concurrency;
      auto restore = [&] {
        eng.use_graph = g;
        eng.autotune = t;
        eng.forced_variant = fv;
        eng.forced_levels = fl;
        eng.concurrency = cc;
      };
      try {
        eng.solve(one, masked != 0, b->half, lane, part);
      } catch (...) {
        restore();
        throw;
      }
      restore();
    };
    VFS_CUDA(cudaEventRecord(b->start, b->stream));
    for (int k = 0; k < n; k++) {
      VFS_CUDA(cudaStreamWaitEvent(b->lanes[k], b->start, 0));
      // staggered coarse parts: pair k's coarse levels follow pair k - S's
      if (split && b->stagger_coarse && k >= S) VFS_CUDA(cudaStreamWaitEvent(b->lanes[k], b->coarse_done[k - S], 0));
      // the first S pairs' coarse parts on the high-priority streams (their full-resolution
      // parts follow there), so that full-resolution work starts early
      cudaStream_t cl = graded ? graded_lane(k)
                               : (split && b->fine_priority >= 2 && k < S) ? b->fine_lanes[k] : b->lanes[k];
      if (cl != b->lanes[k]) VFS_CUDA(cudaStreamWaitEvent(cl, b->start, 0));
      if (io)
        pairs[k]->copyImagesU8On(io->i0[k], io->i1[k], io->device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                 cl);
      run(k, split ? 1 : 0, n, cl, graded ? round_prio(k) : cl != b->lanes[k] ? prio_hi : 0);
      if (split) {
        VFS_CUDA(cudaEventRecord(b->coarse_done[k], cl));
        continue;
      }
      if (io)
        pairs[k]->copyOutOn("u", io->u[k], io->device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, b->lanes[k]);
      VFS_CUDA(cudaEventRecord(b->lane_done[k], b->lanes[k]));
      VFS_CUDA(cudaStreamWaitEvent(b->stream, b->lane_done[k], 0));
    }
    if (split) {
      for (int k = 0; k < n; k++) {
        cudaStream_t fl = coarse_first ? b->lanes[k]
                          : graded     ? graded_lane(k)
                          : b->fine_priority ? b->fine_lanes[k] : b->lanes[k];
        VFS_CUDA(cudaStreamWaitEvent(fl, b->coarse_done[k], 0));
        if (k >= S) VFS_CUDA(cudaStreamWaitEvent(fl, b->fine_done[k - S], 0));
        run(k, 2, S, fl, coarse_first ? 0 : graded ? round_prio(k) : b->fine_priority >= 1 ? prio_hi : 0);
        VFS_CUDA(cudaEventRecord(b->fine_done[k], fl));
        if (io) pairs[k]->copyOutOn("u", io->u[k], io->device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, fl);
        VFS_CUDA(cudaEventRecord(b->lane_done[k], fl));
        VFS_CUDA(cudaStreamWaitEvent(b->stream, b->lane_done[k], 0));
        // the next solve's parts of this slot follow this one's end
        VFS_CUDA(cudaStreamWaitEvent(b->lanes[k], b->lane_done[k], 0));
        VFS_CUDA(cudaStreamWaitEvent(b->fine_lanes[k], b->lane_done[k], 0));
      }
    }
  }
  VFS_CUDA(cudaEventRecord(b->done, b->stream));
  for (auto* p : pairs)
    if (p->stream() != b->stream) VFS_CUDA(cudaStreamWaitEvent(p->stream(), b->done, 0));
  if (io && !io->device) VFS_CUDA(cudaStreamSynchronize(b->stream));
}

}  // namespace

extern "C" {

int vfs_batch_solve(vfs_batch* b, int masked) {
  return guarded(b, [&] { batch_solve(b, masked, nullptr); });
}

int vfs_batch_solve_host(vfs_batch* b, const uint8_t* const* i0, const uint8_t* const* i1, float* const* u_out,
                         int masked) {
  return guarded(b, [&] {
    if (!i0 || !i1 || !u_out) throw vfs::ArgError{"batch solve: null host buffer list"};
    BatchHostIO io{i0, i1, u_out, false};
    batch_solve(b, masked, &io);
  });
}

int vfs_batch_solve_device(vfs_batch* b, const uint8_t* const* d_i0, const uint8_t* const* d_i1, float* const* d_u_out,
                           int masked) {
  return guarded(b, [&] {
    if (!d_i0 || !d_i1 || !d_u_out) throw vfs::ArgError{"batch solve: null device buffer list"};
    BatchHostIO io{d_i0, d_i1, d_u_out, true};
    batch_solve(b, masked, &io);
  });
}

int vfs_equalize_hist_u8(const uint8_t* d_src, uint8_t* d_dst, size_t n, void* cuda_stream) {
  if (n == 0) return VFS_OK;
  if (!d_src || !d_dst) return VFS_ERR_ARG;
  if (n > 0xFFFFFFFFull) return VFS_ERR_ARG;  // 32-bit histogram counters
  cudaStream_t st = (cudaStream_t)cuda_stream;
  void* scratch = nullptr;
  if (cudaMallocAsync(&scratch, 256 * sizeof(unsigned int) + 256, st) != cudaSuccess) {
    (void)cudaGetLastError();
    return VFS_ERR_NOMEM;
  }
  int rc = VFS_OK;
  try {
    vfs::launch_equalize_hist(d_src, d_dst, n, (unsigned int*)scratch, (uint8_t*)scratch + 256 * sizeof(unsigned int),
                              st);
  } catch (const vfs::CudaError&) {
    (void)cudaGetLastError();
    rc = VFS_ERR_CUDA;
  }
  if (cudaFreeAsync(scratch, st) != cudaSuccess) {
    (void)cudaGetLastError();
    rc = VFS_ERR_CUDA;
  }
  return rc;
}

long long vfs_launch_count(void) { return vfs::launch_counter().load(); }

int vfs_device_status(int* status) {
  try {
    int v = vfs::tma_status_take();
    if (status) *status = v;
    return VFS_OK;
  } catch (const vfs::CudaError& e) {
    (void)cudaGetLastError();
    vfs::set_global_error(cudaGetErrorString(e.err));
    return VFS_ERR_CUDA;
  }
}

int vfs_set_launch_overlap(int on) {
  vfs::pdl_enabled().store(on != 0);
  return VFS_OK;
}

int vfs_profile_enable(vfs_stereo* s, int on) {
  return guarded(s, [&] { s->impl.profiling = on != 0; });
}

int vfs_profile_reset(vfs_stereo* s) {
  return guarded(s, [&] {
    VFS_CUDA(cudaStreamSynchronize(s->impl.stream()));
    s->impl.profReset();
  });
}

int vfs_profile_read(vfs_stereo* s, int kind, long long* n, double* ms, double* pi) {
  return guarded(s, [&] {
    if (kind < 0 || kind >= vfs::kProfTags) throw vfs::ArgError{"profile kind out of range"};
    s->impl.profRead(kind, n, ms, pi);
  });
}

// One process-wide reference event, so that records of different handles (solved on
// different streams) can be placed on one time axis.
static cudaEvent_t g_prof_epoch = nullptr;

int vfs_profile_epoch(void* cuda_stream) {
  cudaError_t e = cudaSuccess;
  if (!g_prof_epoch) e = cudaEventCreate(&g_prof_epoch);
  if (e == cudaSuccess) e = cudaEventRecord(g_prof_epoch, (cudaStream_t)cuda_stream);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    vfs::set_global_error(cudaGetErrorString(e));
    return VFS_ERR_CUDA;
  }
  return VFS_OK;
}

int vfs_profile_intervals(vfs_stereo* s, int kind, int max_records, double* start_ms, double* end_ms,
                          double* pixel_iterations, double* launches, int* count) {
  return guarded(s, [&] {
    if (kind < 0 || kind >= vfs::kProfTags) throw vfs::ArgError{"profile kind out of range"};
    if (!g_prof_epoch) throw vfs::ArgError{"vfs_profile_epoch() has not been recorded"};
    if (max_records < 0 || !count) throw vfs::ArgError{"invalid output"};
    VFS_CUDA(cudaEventSynchronize(g_prof_epoch));
    int n = 0;
    for (const auto& r : s->impl.profRecords()) {
      if (r.tag != kind) continue;
      if (n < max_records) {
        VFS_CUDA(cudaEventSynchronize(r.b));
        float a = 0, b = 0;
        VFS_CUDA(cudaEventElapsedTime(&a, g_prof_epoch, r.a));
        VFS_CUDA(cudaEventElapsedTime(&b, g_prof_epoch, r.b));
        if (start_ms) start_ms[n] = a;
        if (end_ms) end_ms[n] = b;
        if (pixel_iterations) pixel_iterations[n] = (double)r.px * r.iters;
        if (launches) launches[n] = (double)r.launches;
      }
      n++;
    }
    *count = n;
  });
}

// ---- reference DLL entry points (dllhook/vfs.cpp) --------------------------------
vfs_stereo* Create(void) {
  vfs_stereo* s = nullptr;
  vfs_create(&s);
  return s;
}

void Init(vfs_stereo* s, int w, int h, float beta, float gamma, float alpha0, float alpha1, float tsl, float lambda,
          int nLevel, float fScale, int nWarpIters, int nSolverIters, float focal, float baseline,
          const char* maskFile, const char* tvFile, const char* cvFile) {
  guarded(s, [&] {
    vfs::SolverParams p;
    p.width = w;
    p.height = h;
    p.beta = beta;
    p.gamma = gamma;
    p.alpha0 = alpha0;
    p.alpha1 = alpha1;
    p.timestep_lambda = tsl;
    p.lambda = lambda;
    p.nLevels = nLevel;
    p.fScale = fScale;
    p.nWarpIters = nWarpIters;
    p.nSolverIters = nSolverIters;
    p.limitRange = s->impl.P.limitRange;
    s->impl.initialize(p);
    s->impl.baseline = baseline;
    s->impl.focal = focal;
    std::string err;
    int mw, mh;
    std::vector<uint8_t> m8;
    if (!maskFile || !vfs::read_gray8(maskFile, mw, mh, m8, err)) throw vfs::ArgError{"Init: mask: " + err};
    if (mw != w || mh != h) throw vfs::ArgError{"Init: mask size differs from the solver size"};
    std::vector<float> mask((size_t)w * h);
    for (size_t i = 0; i < mask.size(); i++) mask[i] = (float)(m8[i] * (1.0 / 255.0));  // convertTo(CV_32F, 1/255)
    s->impl.copyMaskToDevice(mask.data());
    int tw, th, cw, ch;
    std::vector<float> tv, cv;
    if (!tvFile || !vfs::read_flo(tvFile, tw, th, tv, err)) throw vfs::ArgError{"Init: translation field: " + err};
    if (!cvFile || !vfs::read_flo(cvFile, cw, ch, cv, err)) throw vfs::ArgError{"Init: calibration field: " + err};
    if (tw != w || th != h || cw != w || ch != h) throw vfs::ArgError{"Init: vector field size differs"};
    s->impl.loadVectorFields(tv.data(), cv.data());
  });
}

void SolveStereo(vfs_stereo* s, unsigned char* fs1, unsigned char* fs2, unsigned char* output, int w, int h,
                 float maxDepth) {
  guarded(s, [&] {
    auto& I = s->impl;
    if (!I.initialized()) throw vfs::ArgError{"SolveStereo before Init"};
    if (!fs1 || !fs2) throw vfs::ArgError{"SolveStereo: null image"};
    if (w != I.width || h != I.height) throw vfs::ArgError{"SolveStereo: image size differs from Init"};
    size_t n = (size_t)w * h;
    size_t need = 2 * n + 256 * sizeof(unsigned int) + 256 + 1024;
    if (s->eq_bytes < need) {
      if (s->d_eq) cudaFree(s->d_eq);
      s->d_eq = nullptr;
      VFS_CUDA(cudaMalloc(&s->d_eq, need));
      s->eq_bytes = need;
    }
    uint8_t* e0 = s->d_eq;
    uint8_t* e1 = s->d_eq + n;
    unsigned int* hist = (unsigned int*)(s->d_eq + ((2 * n + 255) & ~(size_t)255));
    uint8_t* lut = (uint8_t*)(hist + 256);
    cudaStream_t st = I.stream();
    VFS_CUDA(cudaMemcpyAsync(e0, fs1, n, cudaMemcpyHostToDevice, st));
    VFS_CUDA(cudaMemcpyAsync(e1, fs2, n, cudaMemcpyHostToDevice, st));
    vfs::launch_equalize_hist(e0, e0, n, hist, lut, st);
    vfs::launch_equalize_hist(e1, e1, n, hist, lut, st);
    I.copyImagesU8(e0, e1, true);
    I.solve(true);
    if (output) {
      std::vector<float> u(n);
      I.copyOut("u", u.data(), true);
      // depth from the 1-D disparity with the focal length and baseline given to
      // Init: Z = focal * |baseline| / u, written as round(255 * Z / maxDepth)
      // clamped to 0..255 (0 where u <= 0).
      for (size_t i = 0; i < n; i++) {
        float z = u[i] > 0.0f ? I.focal * std::fabs(I.baseline) / u[i] : 0.0f;
        float v = maxDepth > 0.0f ? 255.0f * z / maxDepth : 0.0f;
        output[i] = (uint8_t)(v <= 0.0f ? 0 : v >= 255.0f ? 255 : (int)std::lround(v));
      }
    } else {
      VFS_CUDA(cudaStreamSynchronize(st));
    }
  });
}

}  // extern "C"
