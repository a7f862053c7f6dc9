"""Failure paths without a GPU fault: host-side fault injection.

IMOPS_FAULT_INJECT=alloc / launch makes the library's C++ layer fail its
allocation / launch sites before any device work there.  Each test checks
that the call returns the status and message a host would see, and that the
next call on the same CUDA context succeeds with the right output.  Nothing
here faults, traps or hangs a GPU.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rgb(gpu, H=96, W=128, seed=5):
    import torch
    rng = np.random.default_rng(seed)
    return torch.from_numpy(rng.uniform(0.02, 0.9, (H, W, 3)).astype(np.float32)).to(gpu)


def test_injected_workspace_failure_reports_and_recovers(gpu, monkeypatch):
    import torch

    import imops_b200 as im
    x = _rgb(gpu)
    ref = im.film_process(x.clone(), stock=im.STOCK_BASELINE81)
    monkeypatch.setenv("IMOPS_FAULT_INJECT", "alloc")
    with pytest.raises(im.ImopsError) as e:
        im.film_process(x.clone(), stock=im.STOCK_BASELINE81)
    assert e.value.code == 5 and "injected allocation failure" in e.value.message
    monkeypatch.delenv("IMOPS_FAULT_INJECT")
    got = im.film_process(x.clone(), stock=im.STOCK_BASELINE81)
    torch.cuda.synchronize()
    assert torch.equal(got, ref)


def test_injected_launch_failure_reports_and_recovers(gpu, monkeypatch):
    import torch

    import imops_b200 as im
    from imops_b200 import synthetic
    m = torch.from_numpy(synthetic.mosaic_f32(192, 256, seed=9)).to(gpu)
    ref = im.demosaic_amaze(m)
    monkeypatch.setenv("IMOPS_FAULT_INJECT", "launch")
    with pytest.raises(im.ImopsError) as e:
        im.demosaic_amaze(m)
    assert e.value.code == 4 and "injected launch failure" in e.value.message
    monkeypatch.delenv("IMOPS_FAULT_INJECT")
    got = im.demosaic_amaze(m)
    torch.cuda.synchronize()
    assert torch.equal(got, ref)


def test_pipeline_c_abi_returns_null_and_last_error(gpu, monkeypatch):
    """run_pixel_pipeline_c's convention (extern_pipeline.rs:343-359): NULL
    and a message from get_last_error_c; the pipeline keeps working after."""
    import imops_b200 as im
    from imops_b200 import synthetic
    from imops_b200.pipeline import Image, get_last_error, make_meta, parse_config, run_pixel_pipeline
    raw = synthetic.mosaic_u16(192, 256, seed=3)
    meta = make_meta(cfa="RGGB", wb=synthetic.WB, calibration=synthetic.CALIB_D65, black=synthetic.BLACK,
                     white=synthetic.WHITE)
    cfg = parse_config('[[pipeline_modules]]\nname = "Demosaic"\nalgorithm = "amaze"\n'
                       '[[pipeline_modules]]\nname = "CST"\ntarget_color_space = "AcesCg"\n')
    ref = run_pixel_pipeline(Image.from_u16(raw, meta), cfg).rgb_f32()
    img = Image.from_u16(raw, meta)
    monkeypatch.setenv("IMOPS_FAULT_INJECT", "alloc,launch")
    L = im.lib()
    L.run_pixel_pipeline_c.restype = ctypes.c_void_p
    L.run_pixel_pipeline_c.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    assert not L.run_pixel_pipeline_c(img._h, cfg._h)
    assert "injected" in get_last_error()
    monkeypatch.delenv("IMOPS_FAULT_INJECT")
    got = run_pixel_pipeline(Image.from_u16(raw, meta), cfg).rgb_f32()
    assert np.array_equal(got, ref)


def test_injected_failures_in_xtrans_and_display(gpu, monkeypatch):
    """The 3-pass X-Trans demosaic and the display chain fail with a status
    at their launch sites and recover the same way; the X-Trans demosaic
    allocates nothing, so an allocation fault leaves it unaffected."""
    import torch

    import imops_b200 as im
    from imops_b200 import synthetic
    m = torch.from_numpy(synthetic.mosaic_f32(96, 120, seed=4, pattern=synthetic.XTRANS)).to(gpu)
    ref = im.demosaic_markesteijn3(m, synthetic.XTRANS)
    monkeypatch.setenv("IMOPS_FAULT_INJECT", "alloc")
    assert torch.equal(im.demosaic_markesteijn3(m, synthetic.XTRANS), ref)
    monkeypatch.setenv("IMOPS_FAULT_INJECT", "launch")
    with pytest.raises(im.ImopsError) as e:
        im.demosaic_markesteijn3(m, synthetic.XTRANS)
    assert e.value.code == 4 and "injected launch failure" in e.value.message
    x = _rgb(gpu)
    with pytest.raises(im.ImopsError) as e:
        im.sigmoid_tone_map(x.clone())
    assert e.value.code == 4 and "injected launch failure" in e.value.message
    monkeypatch.delenv("IMOPS_FAULT_INJECT")
    got = im.demosaic_markesteijn3(m, synthetic.XTRANS)
    torch.cuda.synchronize()
    assert torch.equal(got, ref)
    a = im.sigmoid_tone_map(x.clone())
    b = im.sigmoid_tone_map(x.clone())
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_release_working_sets_then_reuse(gpu):
    """Freeing the cached working sets between calls changes no result."""
    import torch

    import imops_b200 as im
    from imops_b200 import synthetic
    x = _rgb(gpu)
    a = im.film_process(x.clone(), stock=im.STOCK_BASELINE81)
    m = torch.from_numpy(synthetic.mosaic_f32(96, 120, seed=4, pattern=synthetic.XTRANS)).to(gpu)
    xa = im.demosaic_markesteijn3(m, synthetic.XTRANS)
    torch.cuda.synchronize()
    im.release_working_sets()
    b = im.film_process(x.clone(), stock=im.STOCK_BASELINE81)
    xb = im.demosaic_markesteijn3(m, synthetic.XTRANS)
    torch.cuda.synchronize()
    assert torch.equal(a, b) and torch.equal(xa, xb)
    im.release_working_sets()
