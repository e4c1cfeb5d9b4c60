"""Python mirror of the reference ``StereoTgv`` class (stereotgv/stereotgv.h:14-124).

Method names, argument order and meaning follow the reference; ``cv::Mat`` arguments become
numpy arrays (H x W, H x W x 2 or H x W x 3) and ``cv::Mat&`` outputs become return values.
Device-resident inputs and outputs are also accepted as torch CUDA tensors through the
``*_device`` methods.  All work runs in the CUDA library (vfs_b200/_lib); failures raise
:class:`VfsError` with the library's status and message.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from ._native import VfsError, check, check_batch, lib

__all__ = ["StereoTgv", "StereoBatch", "VfsError"]

PATH_REFERENCE = 0
PATH_FUSED = 1


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _stream_ptr(stream):
    """cudaStream_t of a torch.cuda.Stream or a raw integer handle (None: the default stream)."""
    raw = getattr(stream, "cuda_stream", stream)
    return ctypes.c_void_p(int(raw) if raw else 0)


class StereoTgv:
    """Variational fisheye stereo solver on one GPU (one camera pair)."""

    def __init__(self, blockWidth: int = 32, blockHeight: int = 1, strideAlignment: int = 32):
        self._L = lib()
        h = ctypes.c_void_p()
        st = self._L.vfs_create_ex(ctypes.byref(h), blockWidth, blockHeight, strideAlignment)
        if st != 0:
            raise VfsError(st, (self._L.vfs_last_error(None) or b"").decode())
        self._h = h
        self.BlockWidth, self.BlockHeight, self.StrideAlignment = blockWidth, blockHeight, strideAlignment
        self._limit_range = 1.0  # stereotgv.h:45
        self.baseline = 0.0
        self.focal = 0.0
        self.width = self.height = 0
        self._stream = None

    def close(self) -> None:
        """Destroy the handle now (frees its device memory); the object is unusable after."""
        h = getattr(self, "_h", None)
        if h:
            self._L.vfs_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # ---- configuration ---------------------------------------------------
    @property
    def limitRange(self) -> float:
        return self._limit_range

    @limitRange.setter
    def limitRange(self, v: float) -> None:
        self._limit_range = float(v)
        check(self._h, self._L.vfs_set_limit_range(self._h, self._limit_range))

    def set_warm_start(self, level: int) -> None:
        """Start each solve after the first from the previous frame's disparity at pyramid level
        ``level`` (0 = full resolution; levels above it are skipped); -1 turns it off."""
        check(self._h, self._L.vfs_set_warm_start(self._h, int(level)))

    def export_state(self) -> np.ndarray:
        """The handle's whole device state as a byte array (see vfs_export_state)."""
        n = int(self._L.vfs_state_bytes(self._h))
        if n == 0:
            raise VfsError(-3, "export_state before initialize")
        buf = np.empty(n, np.uint8)
        check(self._h, self._L.vfs_export_state(self._h, buf.ctypes.data_as(ctypes.c_void_p), n))
        return buf

    def import_state(self, state: np.ndarray) -> None:
        """Restore a state exported from a handle of the same size, levels and scale."""
        buf = np.ascontiguousarray(state, np.uint8)
        check(self._h, self._L.vfs_import_state(self._h, buf.ctypes.data_as(ctypes.c_void_p), buf.size))

    def set_tensor_math(self, portable: bool) -> None:
        """Tensor weight from CUDA's expf / powf as the reference (False, the default) or from
        the portable exp / log that the CPU oracle restates bit for bit (True)."""
        check(self._h, self._L.vfs_set_tensor_math(self._h, 1 if portable else 0))

    def set_stream(self, stream) -> None:
        """Run on a torch.cuda.Stream (or a raw cudaStream_t integer)."""
        raw = getattr(stream, "cuda_stream", stream)
        self._stream = stream
        check(self._h, self._L.vfs_set_stream(self._h, ctypes.c_void_p(int(raw) if raw else 0)))

    def synchronize(self) -> None:
        check(self._h, self._L.vfs_synchronize(self._h))

    def check_guards(self) -> int:
        """Number of the guard zones after the handle's device planes that a kernel has
        stored into (0: every store stayed in bounds)."""
        n = ctypes.c_int(-1)
        check(self._h, self._L.vfs_debug_check_guards(self._h, ctypes.byref(n)))
        return n.value

    def set_solve_path(self, fused: bool, half_storage: bool = False) -> None:
        """Select the drop-in path (one kernel per reference kernel) or the fused path
        (optionally with p, q, v-bar and the warped image stored as half)."""
        check(self._h, self._L.vfs_set_solve_path(self._h, PATH_FUSED if fused else PATH_REFERENCE,
                                                  int(half_storage)))

    def set_graph(self, on: bool) -> None:
        check(self._h, self._L.vfs_set_graph(self._h, int(on)))

    def set_autotune(self, on: bool) -> None:
        check(self._h, self._L.vfs_set_autotune(self._h, int(on)))

    def set_iteration_variant(self, variant: int) -> None:
        """Force one variant (0..19, the retired numbers excepted) of the fused iteration kernel,
        or -1 for the tuned choice."""
        check(self._h, self._L.vfs_set_iteration_variant(self._h, int(variant)))

    def set_iteration_variants(self, variants) -> None:
        """Force one variant per pyramid level (finest first); an empty list clears it."""
        arr = (ctypes.c_int * max(1, len(variants)))(*variants)
        check(self._h, self._L.vfs_set_iteration_variants(self._h, arr, len(variants)))

    def iteration_variants(self):
        """Iteration-kernel variant per pyramid level (finest first) of the last fused solve."""
        out = (ctypes.c_int * 16)()
        n = ctypes.c_int()
        check(self._h, self._L.vfs_get_iteration_variants(self._h, out, 16, ctypes.byref(n)))
        return [out[i] for i in range(min(n.value, 16))]

    # ---- reference methods -------------------------------------------------
    def initialize(self, width, height, beta, gamma, alpha0, alpha1, timestep_lambda, lambda_,
                   nLevels, fScale, nWarpIters, nSolverIters) -> int:
        check(self._h, self._L.vfs_initialize(self._h, int(width), int(height), beta, gamma, alpha0, alpha1,
                                              timestep_lambda, lambda_, int(nLevels), fScale, int(nWarpIters),
                                              int(nSolverIters)))
        self.width, self.height = int(width), int(height)
        check(self._h, self._L.vfs_set_camera(self._h, float(self.baseline), float(self.focal)))
        return 0

    def level_sizes(self):
        out = []
        w, h, s = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        lvl = 0
        while True:
            st = self._L.vfs_get_level_size(self._h, lvl, ctypes.byref(w), ctypes.byref(h), ctypes.byref(s))
            if st != 0:
                break
            out.append((w.value, h.value, s.value))
            lvl += 1
        return out

    def loadVectorFields(self, translationVector: np.ndarray, calibrationVector: np.ndarray) -> int:
        tv = np.ascontiguousarray(translationVector, np.float32)
        cv = np.ascontiguousarray(calibrationVector, np.float32)
        self._check_shape(tv, (self.height, self.width, 2), "translationVector")
        self._check_shape(cv, (self.height, self.width, 2), "calibrationVector")
        check(self._h, self._L.vfs_load_vector_fields(self._h, _ptr(tv), _ptr(cv)))
        return 0

    def copyMaskToDevice(self, mask: np.ndarray) -> int:
        m = np.ascontiguousarray(mask, np.float32)
        self._check_shape(m, (self.height, self.width), "mask")
        check(self._h, self._L.vfs_copy_mask_to_device(self._h, _ptr(m)))
        return 0

    def copyImagesToDevice(self, i0, i1) -> int:
        """u8 (H x W), float32 (H x W) or u8 colour (H x W x 3) images, as the reference overloads."""
        a = np.asarray(i0)
        b = np.asarray(i1)
        if a.dtype != b.dtype or a.shape != b.shape:
            raise VfsError(-1, "copyImagesToDevice: images differ in type or shape")
        if a.dtype == np.uint8 and a.ndim == 2:
            self._check_shape(a, (self.height, self.width), "image")
            a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
            check(self._h, self._L.vfs_copy_images_to_device_u8(self._h, _ptr(a), _ptr(b)))
        elif a.dtype == np.uint8 and a.ndim == 3 and a.shape[2] == 3:
            self._check_shape(a, (self.height, self.width, 3), "image")
            a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
            check(self._h, self._L.vfs_copy_images_to_device_u8c3(self._h, _ptr(a), _ptr(b)))
        elif a.dtype == np.float32 and a.ndim == 2:
            self._check_shape(a, (self.height, self.width), "image")
            a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
            check(self._h, self._L.vfs_copy_images_to_device_f32(self._h, _ptr(a), _ptr(b)))
        else:
            raise VfsError(-1, f"copyImagesToDevice: unsupported image type {a.dtype} {a.shape}")
        return 0

    def copy_images_from_device(self, d_i0, d_i1) -> None:
        """Images already on the GPU: tight H x W uint8 torch tensors (stream-ordered)."""
        for t in (d_i0, d_i1):
            if not (t.is_cuda and t.is_contiguous() and tuple(t.shape) == (self.height, self.width)):
                raise VfsError(-1, "copy_images_from_device: need contiguous H x W uint8 CUDA tensors")
        check(self._h, self._L.vfs_copy_images_from_device_u8(self._h, ctypes.c_void_p(d_i0.data_ptr()),
                                                              ctypes.c_void_p(d_i1.data_ptr())))

    def solveStereoForward(self) -> int:
        check(self._h, self._L.vfs_solve_stereo_forward(self._h))
        return 0

    def solveStereoForwardMasked(self) -> int:
        check(self._h, self._L.vfs_solve_stereo_forward_masked(self._h))
        return 0

    def copy1DDisparityToHost(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        check(self._h, self._L.vfs_copy_1d_disparity_to_host(self._h, _ptr(out)))
        return out

    def copyDisparityToHost(self) -> np.ndarray:
        out = np.empty((self.height, self.width, 2), np.float32)
        check(self._h, self._L.vfs_copy_disparity_to_host(self._h, _ptr(out)))
        return out

    def copyWarpedImageToHost(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        check(self._h, self._L.vfs_copy_warped_image_to_host(self._h, _ptr(out)))
        return out

    def copy_1d_disparity_to_device(self, d_out) -> None:
        if not (d_out.is_cuda and d_out.is_contiguous() and tuple(d_out.shape) == (self.height, self.width)):
            raise VfsError(-1, "copy_1d_disparity_to_device: need a contiguous H x W float32 CUDA tensor")
        check(self._h, self._L.vfs_copy_1d_disparity_to_device(self._h, ctypes.c_void_p(d_out.data_ptr())))

    def copyStereoToHost(self, focalx, focaly, cx, cy, d1, d2, d3, d4, t1, t2, t3) -> Tuple[np.ndarray, np.ndarray]:
        depth = np.empty((self.height, self.width), np.float32)
        X = np.empty((self.height, self.width, 3), np.float32)
        check(self._h, self._L.vfs_copy_stereo_to_host(self._h, _ptr(depth), _ptr(X), focalx, focaly, cx, cy,
                                                       d1, d2, d3, d4, t1, t2, t3))
        return depth, X

    def copyDisparityVisToHost(self, flowScale: float) -> np.ndarray:
        out = np.empty((self.height, self.width, 3), np.float32)
        check(self._h, self._L.vfs_copy_disparity_vis_to_host(self._h, _ptr(out), flowScale))
        return out

    # ---- measurement hooks ---------------------------------------------------
    @staticmethod
    def launch_count() -> int:
        return int(lib().vfs_launch_count())

    def profile(self, on: bool) -> None:
        check(self._h, self._L.vfs_profile_enable(self._h, int(on)))

    def profile_reset(self) -> None:
        check(self._h, self._L.vfs_profile_reset(self._h))

    def profile_read(self, kind: int):
        """(launches, total_ms, pixel_iterations) of a timed launch group kind."""
        n, ms, pi = ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double()
        check(self._h, self._L.vfs_profile_read(self._h, kind, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(pi)))
        return n.value, ms.value, pi.value

    @staticmethod
    def profile_epoch(stream=None) -> None:
        """Record the process-wide reference event of profile_intervals() on a stream."""
        L = lib()
        st = L.vfs_profile_epoch(_stream_ptr(stream))
        if st != 0:
            raise VfsError(st, L.vfs_last_error(None).decode(errors="replace"))

    def profile_intervals(self, kind: int) -> np.ndarray:
        """(start_ms, end_ms, pixel_iterations, launches) rows of the records of a kind,
        relative to the last profile_epoch()."""
        n = ctypes.c_int()
        check(self._h, self._L.vfs_profile_intervals(self._h, kind, 0, None, None, None, None, ctypes.byref(n)))
        out = np.zeros((4, n.value), np.float64)
        if n.value:
            check(self._h, self._L.vfs_profile_intervals(self._h, kind, n.value, _ptr(out[0]), _ptr(out[1]),
                                                         _ptr(out[2]), _ptr(out[3]), ctypes.byref(n)))
        return out.T.copy()

    def debug_buffer(self, name: str, comps: int = 1) -> np.ndarray:
        out = np.empty((self.height, self.width, comps), np.float32)
        check(self._h, self._L.vfs_debug_get_buffer(self._h, name.encode(), comps, _ptr(out)))
        return out[:, :, 0] if comps == 1 else out

    @staticmethod
    def _check_shape(a: np.ndarray, shape, what: str) -> None:
        if tuple(a.shape) != tuple(shape):
            raise VfsError(-1, f"{what}: expected shape {tuple(shape)}, got {tuple(a.shape)}")


class StereoBatch:
    """Several :class:`StereoTgv` pairs solved together by the fused path: by default each
    pair replays its own CUDA graph on one of the batch's streams (the pairs run concurrently,
    at most an L2-sized number of them at full resolution at a time); ``set_mode(True)``
    makes one launch per step and level cover every pair."""

    def __init__(self, half_storage: bool = False, stream=None):
        self._L = lib()
        h = ctypes.c_void_p()
        st = self._L.vfs_batch_create(ctypes.byref(h))
        if st != 0:
            raise VfsError(st, "vfs_batch_create failed")
        self._h = h
        self.members = []
        self.set_storage(half_storage)
        if stream is not None:
            self.set_stream(stream)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                self._L.vfs_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def set_stream(self, stream) -> None:
        """Run the batched work on this stream; members keep their own streams and are
        ordered before / after each batch solve with events."""
        raw = getattr(stream, "cuda_stream", stream)
        self._stream = stream
        check_batch(self._h, self._L.vfs_batch_set_stream(self._h, ctypes.c_void_p(int(raw) if raw else 0)))

    def set_storage(self, half_storage: bool) -> None:
        check_batch(self._h, self._L.vfs_batch_set_storage(self._h, int(half_storage)))

    def set_graph(self, on: bool) -> None:
        check_batch(self._h, self._L.vfs_batch_set_graph(self._h, int(on)))

    def set_autotune(self, on: bool) -> None:
        check_batch(self._h, self._L.vfs_batch_set_autotune(self._h, int(on)))

    def set_iteration_variant(self, variant: int) -> None:
        """Force one variant (0..19, the retired numbers excepted) of the fused iteration kernel,
        or -1 for the tuned choice."""
        check_batch(self._h, self._L.vfs_batch_set_iteration_variant(self._h, int(variant)))

    def set_iteration_variants(self, variants) -> None:
        """Force one variant per pyramid level (finest first); an empty list clears it."""
        arr = (ctypes.c_int * max(1, len(variants)))(*variants)
        check_batch(self._h, self._L.vfs_batch_set_iteration_variants(self._h, arr, len(variants)))

    def set_mode(self, one_launch: bool) -> None:
        """False (default): pairs run concurrently, each from its own CUDA graph; True: one
        launch per step and level covers all pairs."""
        check_batch(self._h, self._L.vfs_batch_set_mode(self._h, int(one_launch)))

    def set_fine_concurrency(self, max_pairs: int) -> None:
        """Concurrent mode: at most max_pairs pairs at full resolution at a time (0: no limit)."""
        check_batch(self._h, self._L.vfs_batch_set_fine_concurrency(self._h, int(max_pairs)))

    def set_pipeline(self, stagger_coarse: bool, priority: int) -> None:
        """With a full-resolution limit: stagger the coarse levels too; priority 1 runs the
        full-resolution parts on high-priority streams, 2 also the first pairs' coarse levels,
        3 every part of pair k at the priority of its full-resolution round, 4 (default) the
        coarse levels above the full-resolution levels; 0 no priorities."""
        check_batch(self._h, self._L.vfs_batch_set_pipeline(self._h, int(stagger_coarse), int(priority)))

    def add(self, solver: "StereoTgv") -> None:
        check_batch(self._h, self._L.vfs_batch_add(self._h, solver.handle))
        self.members.append(solver)

    def clear(self) -> None:
        check_batch(self._h, self._L.vfs_batch_clear(self._h))
        self.members = []

    def solve(self, masked: bool = True) -> None:
        check_batch(self._h, self._L.vfs_batch_solve(self._h, int(masked)))

    def solve_device(self, images, outputs, masked: bool = True) -> None:
        """One solve of every pair from and to device memory: ``images[k] = (i0, i1)``, tight
        H x W uint8 CUDA tensors of pair k, and ``outputs[k]`` H x W float32 CUDA tensors.
        Stream-ordered on the batch's stream."""
        n = len(self.members)
        if len(images) != n or len(outputs) != n:
            raise VfsError(-1, f"solve_device: {len(images)} image pairs and {len(outputs)} outputs for a batch of {n}")
        for m, (a, b), o in zip(self.members, images, outputs):
            for t in (a, b, o):
                if not (t.is_cuda and t.is_contiguous() and tuple(t.shape) == (m.height, m.width)):
                    raise VfsError(-1, "solve_device: need contiguous H x W CUDA tensors")
        P = ctypes.c_void_p * n
        i0 = P(*[a.data_ptr() for a, _ in images])
        i1 = P(*[b.data_ptr() for _, b in images])
        uo = P(*[o.data_ptr() for o in outputs])
        check_batch(self._h, self._L.vfs_batch_solve_device(self._h, i0, i1, uo, int(masked)))

    def solve_host(self, images, outputs=None, masked: bool = True):
        """One solve of every pair from and to host memory: ``images[k] = (i0, i1)``, tight
        H x W uint8 arrays of pair k; the disparities go to ``outputs[k]`` (H x W float32,
        allocated when not given).  Page-locked arrays (e.g. from ``torch.pin_memory``)
        are copied asynchronously.  Returns the outputs once they are in host memory."""
        n = len(self.members)
        if len(images) != n:
            raise VfsError(-1, f"solve_host: {len(images)} image pairs for a batch of {n}")
        if outputs is None:
            outputs = [np.empty((m.height, m.width), np.float32) for m in self.members]
        keep = []
        for m, (a, b), o in zip(self.members, images, outputs):
            for x, dt in ((a, np.uint8), (b, np.uint8), (o, np.float32)):
                if not (isinstance(x, np.ndarray) and x.dtype == dt and x.flags.c_contiguous
                        and x.shape == (m.height, m.width)):
                    raise VfsError(-1, "solve_host: need contiguous H x W uint8 images and float32 outputs")
            keep += [a, b, o]
        P = ctypes.c_void_p * n
        i0 = P(*[a.ctypes.data for a, _ in images])
        i1 = P(*[b.ctypes.data for _, b in images])
        uo = P(*[o.ctypes.data for o in outputs])
        check_batch(self._h, self._L.vfs_batch_solve_host(self._h, i0, i1, uo, int(masked)))
        return outputs

    def __len__(self):
        return len(self.members)
