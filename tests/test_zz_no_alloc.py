"""imops_film_baseline_noalloc: the baseline film preset for callers that
cannot allocate device memory -- a host application that gives the GPU a
fixed budget through its own allocator, or a real-time preview loop that
cannot take the synchronisation cudaMalloc may cause.  Its working planes
live in one fixed device array shared by every call, so the test checks two
calls in a row (different images and presets: the second runs over the
first one's leftovers) against imops_film_process, within the film tests'
1e-4, and that images above the array's limit are refused before any GPU
work.

This file is named so pytest collects it last; it also passes when run
alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from imops_b200 import synthetic

pytestmark = pytest.mark.gpu

TOL = 1e-4  # the film parity tolerance of tests/test_gpu_film.py


def _noalloc(lib, rgb, preset, stream):
    H, W = rgb.shape[:2]
    import imops_b200 as im
    f = lib.imops_film_baseline_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(im.BaselineFilm),
                  ctypes.c_void_p]
    return f(ctypes.c_void_p(rgb.data_ptr()), W, H, im.CS_ACESCG, ctypes.byref(preset),
             ctypes.c_void_p(stream.cuda_stream))


def _frame(H, W, seed):
    # demosaiced scene-linear ACEScg with highlights above the halation threshold
    rng = np.random.default_rng(seed)
    return (synthetic.scene(H, W, seed=seed) * 1.3 + 0.02 * rng.random((H, W, 3))).astype(np.float32)


def test_noalloc_matches_film_process_twice(gpu):
    import torch

    import imops_b200 as im

    lib = im.lib()
    stream = torch.cuda.current_stream()
    cases = [(512, 768, im.baseline_film_defaults(seed=7)),
             (300, 410, im.baseline_film_defaults(seed=8, hal_strength=0.3, grain_sigma=0.03))]
    for H, W, preset in cases:
        x = torch.from_numpy(_frame(H, W, seed=H)).to(gpu)
        ref = x.clone()
        im.film_process(ref, stock=im.STOCK_BASELINE81, baseline=preset, stream=stream)
        got = x.clone()
        assert _noalloc(lib, got, preset, stream) == 0, im.last_error()
        torch.cuda.synchronize()
        err = float((got - ref).abs().max())
        assert err <= TOL, f"{W}x{H}: max |no-alloc - film_process| = {err}"
        assert torch.isfinite(got).all()


def test_noalloc_rejects_images_above_its_array(gpu):
    import torch

    import imops_b200 as im

    lib = im.lib()
    lib.imops_film_noalloc_max_pixels.restype = ctypes.c_size_t
    cap = lib.imops_film_noalloc_max_pixels()
    assert cap == 1 << 21
    big = torch.zeros((1082, 1940, 3), device=gpu)  # 2,099,080 px: just above the limit
    assert big.shape[0] * big.shape[1] > cap
    rc = _noalloc(lib, big, im.baseline_film_defaults(seed=1), torch.cuda.current_stream())
    assert rc == 3  # IMOPS_ERR_UNSUPPORTED_SIZE
    assert "imops_film_process" in im.last_error()
    assert float(big.abs().max()) == 0.0  # nothing ran
