"""The allocation-free equalisation entry point against the allocating one.

vfs_equalize_hist_u8_noalloc is for callers that cannot allocate device memory where they
call it: real-time camera threads, where cudaMalloc / cudaFree can synchronise the device and
stall, and hosts whose device memory is handed to their own allocator up front.  It keeps its
scratch in a device array of the library that every call shares, so two calls in a row must
each start from a cleared histogram: the second call here equalises different images and must
still match the allocating entry point exactly (the result is integer / byte work).  This
file runs last (pytest collects it after the other test files).
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


def test_noalloc_in_place_and_unaligned_images(gpu):
    """count = 3 images of an odd size (later images start off a 16-byte boundary, which takes
    the scalar histogram loop) equalised in place (d_dst == d_src), twice in a row."""
    import torch
    from vfs_b200._native import lib
    L = lib()
    st = torch.cuda.current_stream()
    rng = np.random.default_rng(7)
    h, w = 401, 423
    for call in range(2):
        imgs = np.stack([np.clip(rng.normal(60 + 50 * k + 20 * call, 12 + 5 * k, (h, w)), 0, 255).astype(np.uint8)
                         for k in range(3)])
        src = torch.from_numpy(imgs).cuda()
        refs = [_eq_alloc(L, src[k].contiguous(), st) for k in range(3)]
        buf = src.clone()
        rc = L.vfs_equalize_hist_u8_noalloc(ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(buf.data_ptr()), h * w,
                                            3, ctypes.c_void_p(st.cuda_stream))
        assert rc == 0, (L.vfs_last_error(None) or b"").decode()
        torch.cuda.synchronize()
        for k in range(3):
            assert torch.equal(buf[k], refs[k]), (call, k)
