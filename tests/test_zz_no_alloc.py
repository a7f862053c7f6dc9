"""imops_demosaic_amaze_noalloc: AMaZE for callers that cannot allocate
device memory (graph capture, host-owned allocators, latency-critical
paths).  Its output must equal imops_demosaic_amaze's bit for bit, also on
the second of two calls in a row (the kernel's shared memory then still
holds the previous call's data).

This file is named so pytest collects it last; it also passes when run
alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(fn, mosaic, out, stream):
    H, W = mosaic.shape
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                   ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]
    return fn(ctypes.c_void_p(mosaic.data_ptr()), W, H, b"RGGB", 1, 0, 1.0, ctypes.c_void_p(out.data_ptr()),
              ctypes.c_void_p(stream.cuda_stream))


def test_noalloc_matches_allocating_entry_twice(gpu):
    import torch

    import imops_b200 as im
    from imops_b200 import synthetic

    lib = im.lib()
    stream = torch.cuda.current_stream()
    frames = [synthetic.mosaic_f32(1024, 1536, seed=41) * np.float32(1.2),  # 204 tiles: persistent grid, tiles per CTA > 1
              np.random.default_rng(42).random((320, 400), dtype=np.float32)]
    for m_np in frames:
        m = torch.from_numpy(m_np).to(gpu)
        ref = torch.empty((*m.shape, 3), device=gpu)
        got = torch.full((*m.shape, 3), float("nan"), device=gpu)
        assert _call(lib.imops_demosaic_amaze, m, ref, stream) == 0, im.last_error()
        assert _call(lib.imops_demosaic_amaze_noalloc, m, got, stream) == 0, im.last_error()
        torch.cuda.synchronize()
        assert torch.equal(got, ref)


def test_noalloc_rejects_reference_panic_sizes(gpu):
    import torch

    import imops_b200 as im

    m = torch.zeros((300, 400), device=gpu)  # height % 96 == 12: the reference's tile fill panics
    out = torch.empty((300, 400, 3), device=gpu)
    rc = _call(im.lib().imops_demosaic_amaze_noalloc, m, out, torch.cuda.current_stream())
    assert rc == 3
    assert "tile" in im.last_error()
