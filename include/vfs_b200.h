/*
 * vfs_b200 — C ABI of the B200 variational fisheye stereo (TGV-L1) solver.
 *
 * Every function returns an int status: VFS_OK (0) or a negative VFS_ERR_* code;
 * nothing in the library exits the process.  vfs_status_string() names a code and
 * vfs_last_error() returns the message of the last failure on a handle.
 *
 * Threading: a handle must be used by one host thread at a time.  All device work
 * of a handle is ordered on its CUDA stream (vfs_set_stream); host-buffer entry
 * points synchronise that stream before they return, device-pointer entry points do
 * not.
 *
 * Images, masks and vector fields are tightly packed row-major width x height arrays
 * (2 interleaved floats per pixel for vector fields), the raw-pointer equivalent of the
 * cv::Mat arguments of the reference class.
 */
#ifndef VFS_B200_H
#define VFS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VFS_OK 0
#define VFS_ERR_ARG (-1)      /* invalid argument or size */
#define VFS_ERR_CUDA (-2)     /* a CUDA runtime call failed */
#define VFS_ERR_STATE (-3)    /* call order violated (e.g. solve before initialize) */
#define VFS_ERR_NOMEM (-4)    /* device allocation failed */
#define VFS_ERR_IO (-5)       /* file could not be read or parsed */
#define VFS_ERR_TIMEOUT (-6)  /* a device-side wait ran out of iterations */
#define VFS_ERR_BUSY (-7)     /* admission refused: not enough free device memory */

typedef struct vfs_stereo vfs_stereo;

const char* vfs_status_string(int status);
const char* vfs_last_error(const vfs_stereo* s);
int vfs_version(void); /* 100 * major + minor */

/* StereoTgv::StereoTgv() (stereotgv/stereotgv.cu:32-36; dllhook/vfs.cpp:3-6 Create). */
int vfs_create(vfs_stereo** out);
/* StereoTgv::StereoTgv(blockWidth, blockHeight, strideAlignment) (stereotgv.cu:38-42).
 * strideAlignment sets the row pitch in elements; blockWidth sets the column extent of
 * the reference's tensor launch (calcTensor.cu:81,227). */
int vfs_create_ex(vfs_stereo** out, int blockWidth, int blockHeight, int strideAlignment);
int vfs_destroy(vfs_stereo* s);
/* Select the CUDA stream (a cudaStream_t) used for all device work of the handle. */
int vfs_set_stream(vfs_stereo* s, void* cuda_stream);
int vfs_synchronize(vfs_stereo* s);

/* StereoTgv::initialize (stereotgv/stereotgv.h:107-109, stereotgv.cu:44-168). */
int vfs_initialize(vfs_stereo* s, int width, int height, float beta, float gamma, float alpha0,
                   float alpha1, float timestep_lambda, float lambda, int nLevels, float fScale,
                   int nWarpIters, int nSolverIters);
/* Public fields of the reference class: limitRange (stereotgv.h:45, default 1.0),
 * baseline / focal (stereotgv.h:31-32, set by dllhook/vfs.cpp:15-16). */
int vfs_set_limit_range(vfs_stereo* s, float limit_range);
int vfs_set_camera(vfs_stereo* s, float baseline, float focal);

/* Arithmetic of the diffusion-tensor weight exp(-beta |grad I|^gamma) (no counterpart in the
 * reference, which always calls CUDA's expf / powf there: calcTensor.cu:60-64).
 * VFS_TENSOR_MATH_CUDA (the default) makes the same calls, so a solve reproduces the
 * reference's CUDA build.  VFS_TENSOR_MATH_PORTABLE uses an exp / log built only from
 * correctly rounded IEEE operations, which a CPU restatement reproduces bit for bit; the two
 * weights agree to 1.5e-6 relative.  Applies to both solve paths from the next solve on. */
/* Warm start (no counterpart in the reference, which starts every solve from zero:
 * stereotgv.cu:395-397).  level < 0 (the default): off.  level >= 0: once the handle has solved
 * a frame, the next solve starts at pyramid level min(level, nLevels - 1), 0 being full
 * resolution, from the previous frame's disparity (box-downscaled to that level); the levels
 * above it are not solved.  level = nLevels - 1 keeps every level and only changes the starting
 * point.  initialize and loadVectorFields forget the previous frame. */
int vfs_set_warm_start(vfs_stereo* s, int level);

/* Number of CUDA graph executables a handle's fused solves keep cached (no counterpart in the
 * reference).  Graphs captured for an older mask or initialize are destroyed on the next
 * solve, and at most 64 are kept (vfs_batch_cached_graphs: the same for a batch). */
int vfs_cached_graphs(const vfs_stereo* s);
/* Number of fused solves this process has run while timing the iteration-kernel variants (the
 * first solve of a new setting; no counterpart in the reference).  A one-pair solve reuses
 * every pyramid level tuned before for the same level size, form and storage (the choice made
 * for a pair alone or with other pairs in flight, the same setting first), so a server whose
 * batch compositions change tunes only for level sizes it has not seen. */
long long vfs_tuning_solves(void);

/* Whole-state export / import (no counterpart in the reference): the handle's device state
 * (image pyramid, mask, fields, every solver buffer with the stale values the reference keeps
 * between frames, and the warm-start disparity), so that a handle initialised with the same
 * size, levels and scale continues bit for bit where the exported one stopped; a camera
 * stream's state can thus leave the GPU while the stream is idle.  Host-side settings (limit
 * range, camera, solve path, stream) are not part of it.  vfs_state_bytes gives the size (0 before
 * initialize); both calls synchronise the handle's stream. */
size_t vfs_state_bytes(const vfs_stereo* s);
int vfs_export_state(vfs_stereo* s, void* host, size_t bytes);
int vfs_import_state(vfs_stereo* s, const void* host, size_t bytes);

/* Test hook (no counterpart in the reference): with n > 0 the n-th following device-pool
 * allocation of any handle fails as if the GPU were out of memory (the call returns
 * VFS_ERR_NOMEM and leaves nothing allocated); 0 turns it off. */
int vfs_debug_fail_allocation(int n);
/* Test hook (no counterpart in the reference): every device plane of a handle is followed by
 * a 256-byte guard zone of 0xA5 bytes, written when the plane is allocated.  *bad_zones is the
 * number of zones that no longer hold the pattern, i.e. that a kernel has stored into past the
 * end of a plane (0 when every store stayed in bounds).  Synchronises the handle's stream. */
int vfs_debug_check_guards(vfs_stereo* s, int* bad_zones);

#define VFS_TENSOR_MATH_CUDA 0
#define VFS_TENSOR_MATH_PORTABLE 1
int vfs_set_tensor_math(vfs_stereo* s, int mode);
/* Pyramid geometry of an initialized handle: level sizes and pitches (elements). */
int vfs_get_level_size(const vfs_stereo* s, int level, int* width, int* height, int* stride);

/* StereoTgv::loadVectorFields(translation, calibration) (stereotgv.h:110,
 * stereotgv.cu:171-199): two H x W x 2 float32 fields in host memory. */
int vfs_load_vector_fields(vfs_stereo* s, const float* translation, const float* calibration);
/* StereoTgv::copyMaskToDevice (stereotgv.h:115, stereotgv.cu:241-252): H x W float32, 0 = off. */
int vfs_copy_mask_to_device(vfs_stereo* s, const float* mask);

/* StereoTgv::copyImagesToDevice(uchar*, uchar*) (stereotgv.h:112, stereotgv.cu:201-213). */
int vfs_copy_images_to_device_u8(vfs_stereo* s, const uint8_t* i0, const uint8_t* i1);
/* StereoTgv::copyImagesToDevice(cv::Mat, cv::Mat) for CV_32F and CV_8UC3 (stereotgv.cu:215-239). */
int vfs_copy_images_to_device_f32(vfs_stereo* s, const float* i0, const float* i1);
int vfs_copy_images_to_device_u8c3(vfs_stereo* s, const uint8_t* i0_rgb, const uint8_t* i1_rgb);
/* Same as the u8 copy with the images already in device memory (tight W x H); stream-ordered. */
int vfs_copy_images_from_device_u8(vfs_stereo* s, const uint8_t* d_i0, const uint8_t* d_i1);

/* StereoTgv::solveStereoForward / solveStereoForwardMasked (stereotgv.h:116-117,
 * stereotgv.cu:256-387 and 389-515).  Stream-ordered: returns after enqueueing. */
int vfs_solve_stereo_forward(vfs_stereo* s);
int vfs_solve_stereo_forward_masked(vfs_stereo* s);

/* StereoTgv::copy1DDisparityToHost (stereotgv.cu:533-540): W x H float32. */
int vfs_copy_1d_disparity_to_host(vfs_stereo* s, float* u);
/* StereoTgv::copyDisparityToHost (stereotgv.cu:542-549): W x H x 2 float32. */
int vfs_copy_disparity_to_host(vfs_stereo* s, float* warp_uv);
/* StereoTgv::copyWarpedImageToHost (stereotgv.cu:561-568): W x H float32. */
int vfs_copy_warped_image_to_host(vfs_stereo* s, float* image);
/* Device-pointer outputs (tight W x H / W x H x 2), stream-ordered. */
int vfs_copy_1d_disparity_to_device(vfs_stereo* s, float* d_u);
int vfs_copy_disparity_to_device(vfs_stereo* s, float* d_warp_uv);
/* StereoTgv::copyStereoToHost (stereotgv.h:118-120, stereotgv.cu:517-531; kernel
 * conversion.cu:3-69): depth W x H and X W x H x 3 from the 2-D disparity, with the
 * reference's argument order (focalx, focaly, cx, cy, d1..d4, t1..t3). */
int vfs_copy_stereo_to_host(vfs_stereo* s, float* depth, float* X, float focalx, float focaly,
                            float cx, float cy, float d1, float d2, float d3, float d4, float t1,
                            float t2, float t3);
/* StereoTgv::copyDisparityVisToHost (stereotgv.cu:551-559; flowToHsv.cu:4-110): W x H x 3. */
int vfs_copy_disparity_vis_to_host(vfs_stereo* s, float* rgb, float flow_scale);

/* Inspection of internal state for tests: copy the level-0 view (W x H x comps) of a
 * named solver buffer ("u", "u_", "warpUV", "a", "b", "c", "etau", "Iu", "Iz", "i1warp",
 * "tv2", "p", "q", "Tp", ...) to host memory. */
int vfs_debug_get_buffer(vfs_stereo* s, const char* name, int comps, float* out);

/* ---- fast path (no counterpart in the reference) ---------------------------------
 * vfs_set_solve_path selects how vfs_solve_stereo_forward[_masked] runs:
 *   VFS_PATH_REFERENCE: one kernel per reference kernel, in the reference's order;
 *   VFS_PATH_FUSED: one fused kernel per primal-dual iteration plus fused per-warp and
 *   per-level kernels, replayed as a CUDA graph.  With float storage the fused path gives
 *   bit-identical results; with half storage (half_storage = 1) p, q, v-bar and the warped
 *   image are kept as IEEE half in memory (all arithmetic stays float; the warped image is
 *   widened to float when it is copied out). */
#define VFS_PATH_REFERENCE 0
#define VFS_PATH_FUSED 1
int vfs_set_solve_path(vfs_stereo* s, int path, int half_storage);
int vfs_set_graph(vfs_stereo* s, int use_graph);

/* Device memory a handle of this geometry allocates (solver state, plus the fused-path
 * buffers when fused != 0), without allocating: for admission control.  0 for invalid
 * geometry.  (No counterpart in the reference.) */
size_t vfs_estimate_device_bytes(int width, int height, int nLevels, float fScale, int strideAlignment,
                                 int fused);

/* Batched solves: several handles (pairs, possibly of different sizes) solved together by
 * the fused path, replayed from CUDA graphs (see vfs_batch_set_mode for how the pairs share
 * launches).
 * Pairs of a batch need equal nWarpIters, nSolverIters and timestep_lambda.  The batch
 * does not own the handles; vfs_batch_add moves the handle onto the batch's stream.  At
 * most VFS_BATCH_MAX pairs. */
#define VFS_BATCH_MAX 24
typedef struct vfs_batch vfs_batch;
int vfs_batch_create(vfs_batch** out);
int vfs_batch_cached_graphs(const vfs_batch* b);
int vfs_batch_destroy(vfs_batch* b);
const char* vfs_batch_last_error(const vfs_batch* b);
int vfs_batch_set_stream(vfs_batch* b, void* cuda_stream);
int vfs_batch_add(vfs_batch* b, vfs_stereo* s);
int vfs_batch_clear(vfs_batch* b);
int vfs_batch_size(const vfs_batch* b);
int vfs_batch_set_storage(vfs_batch* b, int half_storage);
int vfs_batch_set_graph(vfs_batch* b, int use_graph);
int vfs_batch_solve(vfs_batch* b, int masked);
/* One batched solve from and to host memory: the reference's per-frame sequence
 * copyImagesToDevice(uchar*, uchar*) -> solveStereoForward[Masked] -> copy1DDisparityToHost
 * (stereotgv.cu:201-213, 256-515, 533-540) for every pair of the batch in one call.  Pair k
 * reads its tight W x H u8 images from i0[k] and i1[k] and writes its tight W x H float32
 * disparity to u_out[k].  Each pair's upload, solve and download are queued on that pair's
 * lane, so the copies of one pair overlap the solves of the others.  Returns when every
 * output is in host memory.  Page-locked host buffers are copied asynchronously by the copy
 * engines; pageable ones work but are staged by the CUDA driver. */
int vfs_batch_solve_host(vfs_batch* b, const uint8_t* const* i0, const uint8_t* const* i1,
                         float* const* u_out, int masked);
/* The same with the images and disparities in device memory (e.g. frames decoded on the GPU):
 * tight W x H u8 inputs and W x H float32 outputs.  Stream-ordered on the batch's stream:
 * returns after enqueueing. */
int vfs_batch_solve_device(vfs_batch* b, const uint8_t* const* d_i0, const uint8_t* const* d_i1,
                           float* const* d_u_out, int masked);
/* The fused path picks the tile height of its iteration kernel per pyramid level by timing
 * the variants on the first solve of each batch composition (on by default); the timing
 * launches do not change results.  Off: the default 31 x 8 tiles everywhere. */
int vfs_batch_set_autotune(vfs_batch* b, int on);
/* How a batch runs its pairs:
 *   VFS_BATCH_CONCURRENT (default): each pair replays its own CUDA graph of one-pair fused
 *     kernels on one of the batch's internal streams; the pairs run concurrently.
 *   VFS_BATCH_ONE_LAUNCH: one launch per step and pyramid level covers every pair (the pair
 *     is found per block from the launch's tile ranges).
 * Both give identical results; concurrent graphs measure faster on B200. */
#define VFS_BATCH_CONCURRENT 0
#define VFS_BATCH_ONE_LAUNCH 1
int vfs_batch_set_mode(vfs_batch* b, int mode);
/* Concurrent mode: run at most max_pairs pairs' full-resolution level at a time (0: no
 * limit; -1, the default: as many full-resolution working sets as fit in three quarters of
 * the L2 cache, and no limit when that is fewer than 2).  Each pair's solve is then two graphs: all pairs' coarser levels
 * start together, and pair k's full-resolution level follows pair k - max_pairs's, so that the
 * full-resolution working sets in flight stay in L2 (on B200, 8 pairs of 848 x 800 with FP16
 * storage: 15.3 ms per batch with 2 at a time against 17.2 ms without a limit).  Results are
 * unchanged. */
int vfs_batch_set_fine_concurrency(vfs_batch* b, int max_pairs);
/* With a full-resolution limit: stagger_coarse = 1 also runs the coarser levels max_pairs
 * pairs at a time (pair k's after pair k - max_pairs's); priority = 1 runs the
 * full-resolution parts on high-priority streams, priority = 2 also the first max_pairs
 * pairs' coarser levels, so that full-resolution work starts while the other pairs' coarse
 * levels run; priority = 3 runs all of pair k's work at the priority of its full-resolution
 * round k / max_pairs (the first round highest); priority = 4, the default, runs the coarser
 * levels above the full-resolution levels (the first round's coarser levels highest), so that
 * every pair's chain of small coarse launches advances while the full-resolution launches
 * fill the rest of the GPU; 0 uses no priorities.  Results are unchanged. */
int vfs_batch_set_pipeline(vfs_batch* b, int stagger_coarse, int priority);
int vfs_set_autotune(vfs_stereo* s, int on);
/* Force one variant of the fused iteration kernel at every pyramid level (-1: the tuned or
 * default choice).  0-2, 19: 32 x (TH + 1)-thread blocks, TH = 4, 8, 16, 15, exchanging
 * the west / north neighbours' T p and q through shared memory; 6-9: several iterations per
 * launch with the tile's region held in shared memory (6: 3 iterations on 64 x 24 tiles, 7: 5
 * on 32 x 24, 8: 3 on 23 x 23, 9: 5 on 17 x 17, 12: 7 on 11 x 11, 13: 9 on 5 x 5); 14-15: the
 * whole level in the shared memory of a thread-block cluster of 16 / 8 CTAs, up to 64
 * iterations per launch (levels whose state fits: about 3200 pixels per CTA with half
 * storage), two cluster barriers per iteration; 18: the 8-row tiles of variant 1 with the
 * block's region of every input plane brought into shared memory by bulk tensor copies.
 * 6-18 apply to one-pair launches (other launches, and levels where they do not apply, use
 * variant 1).  3-5, 10, 11, 16 and 17 are retired and rejected with VFS_ERR_ARG.  Every
 * variant gives the same results; this selects speed only.  (No counterpart in the
 * reference.) */
#define VFS_ITER_VARIANTS 20
int vfs_set_iteration_variant(vfs_stereo* s, int variant);
/* Force one variant per pyramid level (finest first; levels beyond n_levels use variant 1),
 * e.g. to pin a tuned choice; n_levels = 0 clears it. */
int vfs_set_iteration_variants(vfs_stereo* s, const int* variants, int n_levels);
int vfs_batch_set_iteration_variants(vfs_batch* b, const int* variants, int n_levels);
/* The variant each pyramid level (finest first) used in the handle's last fused solve
 * (tuned, default or forced); *count receives the number of levels. */
int vfs_get_iteration_variants(vfs_stereo* s, int* variants, int max_levels, int* count);
int vfs_batch_set_iteration_variant(vfs_batch* b, int variant);

/* Histogram equalisation of n 8-bit pixels in device memory (d_dst may equal d_src), as
 * cv::equalizeHist, which the reference's SolveStereo applies to both images on the host
 * (dllhook/vfs.cpp:36-37).  Stream-ordered on cuda_stream; its 1280 bytes of scratch are
 * allocated and freed on that stream (cudaMallocAsync / cudaFreeAsync). */
int vfs_equalize_hist_u8(const uint8_t* d_src, uint8_t* d_dst, size_t n, void* cuda_stream);

/* Histogram equalisation that allocates nothing (no counterpart in the reference).
 * For callers that cannot allocate device memory where they call it: real-time camera
 * threads with a latency budget, where cudaMalloc / cudaFree can synchronise the whole device
 * and stall for an unbounded time; and hosts that hand all of the GPU's memory to their own
 * allocator or pool up front, so that a library allocation would fail or break the budget.
 * It equalises `count` images of n pixels each, stored back to back at d_src (results at
 * d_dst, which may equal d_src), like vfs_equalize_hist_u8.
 * Limits: count <= VFS_NOALLOC_MAX_IMAGES (16) and n <= 2^32 - 1; larger requests return
 * VFS_ERR_ARG with a message in vfs_last_error(NULL).  The scratch is a 20 KiB array that
 * each GPU loading the library keeps until exit, shared by every call on that GPU; each call
 * clears the histograms it uses.  Calls whose work overlaps on the GPU (different streams,
 * or host threads without ordering) race on the array, so order them on one stream.
 * The first call on a device (and the first after cudaDeviceReset or under another CUDA
 * context) looks up the array's device address with cudaGetSymbolAddress and caches it. */
#define VFS_NOALLOC_MAX_IMAGES 16
int vfs_equalize_hist_u8_noalloc(const uint8_t* d_src, uint8_t* d_dst, size_t n, int count,
                                 void* cuda_stream);

/* Measurement hooks (no counterpart in the reference).  vfs_launch_count() is the number
 * of kernels this library has launched in the process.  With profiling on, each group of
 * inner primal-dual kernels (one iteration in the drop-in path, one fused launch of several
 * iterations in the fused path) is bracketed by CUDA events on the handle's stream;
 * vfs_profile_read() sums the records of a group kind (0 = drop-in inner iteration,
 * 1 = fused inner launch, 2 = fused per-warp prologue, 3 = fused epilogue). */
long long vfs_launch_count(void);

/* Device-side status of the current device (no counterpart in the reference): *status = 1 if
 * a kernel of the TMA-staged iteration variant gave up a bounded wait for its copies since the
 * last call (its block then wrote nothing), else 0; the flag is cleared.  Synchronous. */
int vfs_device_status(int* status);
/* Process-wide: launch the fused iteration kernels with programmatic dependent launch
 * (on = 1, the default), so that each launch is scheduled while the previous one drains;
 * every such kernel waits for its predecessor's results before reading memory, so the
 * results are the same either way.  Graphs captured before a change keep the old setting. */
int vfs_set_launch_overlap(int on);
int vfs_profile_enable(vfs_stereo* s, int on);
int vfs_profile_reset(vfs_stereo* s);
int vfs_profile_read(vfs_stereo* s, int kind, long long* launches, double* total_ms,
                     double* pixel_iterations);
/* vfs_profile_epoch() records one process-wide reference event on a stream (NULL: the
 * legacy default stream).  vfs_profile_intervals() then returns, for the handle's records
 * of a kind, their start and end in ms after that event, their pixel-iterations and their
 * kernel launches (up to max_records of them; *count receives the number of records).  Records of handles
 * solved concurrently on different streams overlap; their union is the time during which
 * at least one such group ran.  A graph replay re-records the events captured with it, so
 * after several replays the records describe the last one. */
int vfs_profile_epoch(void* cuda_stream);
int vfs_profile_intervals(vfs_stereo* s, int kind, int max_records, double* start_ms, double* end_ms,
                          double* pixel_iterations, double* launches, int* count);

/* ---- reference DLL entry points (dllhook/vfs.h:37-44) -------------------------------
 * Create / Init / SolveStereo with the reference's names and argument lists.  Init reads
 * the mask (8-bit PNG or binary PGM, scaled by 1/255) and the two Middlebury .flo fields.
 * SolveStereo equalises both images' histograms on the device (the reference calls
 * cv::equalizeHist), solves the masked problem and, unlike the reference (which leaves
 * it unwritten, dllhook/vfs.cpp:42-47), fills `output` with depth8 = clamp(255 * Z /
 * maxDepth) using the focal/baseline set by Init.  Errors are reported by
 * vfs_last_error() on the handle. */
vfs_stereo* Create(void);
void Init(vfs_stereo* vfs, int stereoWidth, int stereoHeight, float beta, float gamma,
          float alpha0, float alpha1, float timeStepLambda, float lambda, int nLevel,
          float fScale, int nWarpIters, int nSolverIters, float focal, float baseline,
          const char* fisheyeMaskFilename, const char* translationVectorFilename,
          const char* calibrationVectorFilename);
void SolveStereo(vfs_stereo* vfs, unsigned char* fs1, unsigned char* fs2, unsigned char* output,
                 int stereoWidth, int stereoHeight, float maxDepth);

#ifdef __cplusplus
}
#endif
#endif /* VFS_B200_H */
