"""The allocation-free equalisation entry point against the allocating one.

vfs_equalize_hist_u8_noalloc serves callers that cannot allocate device memory where they
call it (inside a stream capture or a graph being recorded, on real-time camera threads where
cudaMalloc / cudaFree may stall on device-wide synchronisation, or with device memory already
reserved by another allocator).  It keeps its scratch in a device array of the library, so two
calls in a row must each start from a cleared histogram: the second call here equalises
different images and must still match the allocating entry point exactly (the result is
integer / byte work).  This file runs last (pytest collects it after the other test files).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _eq_alloc(L, src, st):
    import torch
    out = torch.empty_like(src)
    rc = L.vfs_equalize_hist_u8(ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(out.data_ptr()), src.numel(),
                                ctypes.c_void_p(st.cuda_stream))
    assert rc == 0
    return out


def test_noalloc_matches_allocating_entry_point_twice(gpu):
    import torch
    from vfs_b200._native import lib
    L = lib()
    st = torch.cuda.current_stream()
    rng = np.random.default_rng(99)
    h, w = 400, 424
    for call in range(2):
        if call == 0:
            imgs = [rng.integers(0, 256, (h, w), dtype=np.uint8),
                    np.clip(rng.normal(80, 15, (h, w)), 0, 255).astype(np.uint8)]
        else:
            imgs = [np.clip(rng.normal(170, 30, (h, w)), 0, 255).astype(np.uint8),
                    rng.integers(100, 110, (h, w), dtype=np.uint8)]
        src = torch.from_numpy(np.stack(imgs)).cuda()
        dst = torch.empty_like(src)
        rc = L.vfs_equalize_hist_u8_noalloc(ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()), h * w,
                                            2, ctypes.c_void_p(st.cuda_stream))
        assert rc == 0, (L.vfs_last_error(None) or b"").decode()
        torch.cuda.synchronize()
        for k in range(2):
            ref = _eq_alloc(L, src[k].contiguous(), st)
            torch.cuda.synchronize()
            assert torch.equal(dst[k], ref), (call, k)


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    from vfs_b200._native import lib
    L = lib()
    rc = L.vfs_equalize_hist_u8_noalloc(ctypes.c_void_p(0), ctypes.c_void_p(0), 100, 17, ctypes.c_void_p(0))
    assert rc == -1
    assert b"VFS_NOALLOC_MAX_IMAGES" in (L.vfs_last_error(None) or b"")
    rc = L.vfs_equalize_hist_u8_noalloc(ctypes.c_void_p(0), ctypes.c_void_p(0), 1 << 33, 1, ctypes.c_void_p(0))
    assert rc == -1
