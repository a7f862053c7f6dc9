"""GPU parity of the per-pixel colour stages against the CPU oracle."""
import numpy as np
import pytest

from imops_b200 import synthetic

pytestmark = pytest.mark.gpu


def _rgb(seed, n=4099):
    rng = np.random.default_rng(seed)
    return (rng.random((n, 3), dtype=np.float32) * 1.2).astype(np.float32)


def test_scale_u16_crop_and_levels(oracle_lib, gpu):
    import torch
    import imops_b200 as im
    raw = synthetic.mosaic_u16(70, 90, seed=2)
    black = [600.0, 610.0, 590.0, 605.0]
    white = [16383.0, 16000.0, 16383.0, 15000.0]
    crop = (3, 5, 80, 61)
    ref = oracle_lib.scale_u16(raw, crop, black, white)
    t = torch.from_numpy(raw.view(np.int16)).to(gpu)
    out = im.scale_u16(t, crop, black, white).cpu().numpy()
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("period", [(6, 6), (1, 1), (2, 2)])
def test_scale_u16_period_levels_several_blocks(oracle_lib, gpu, period):
    """Per-site levels over a 6x6 (X-Trans), 1x1 and 2x2 period, a crop at an
    odd origin, rows and columns spanning several blocks and a partial last
    row group."""
    import torch
    import imops_b200 as im
    raw = synthetic.mosaic_u16(157, 611, seed=4, pattern=synthetic.XTRANS)
    n = period[0] * period[1]
    rng = np.random.default_rng(n)
    black = [float(v) for v in rng.uniform(580.0, 620.0, n).astype(np.float32)]
    white = [float(v) for v in rng.uniform(15000.0, 16383.0, n).astype(np.float32)]
    crop = (5, 7, 600, 141)
    ref = oracle_lib.scale_u16(raw, crop, black, white, cfa_period=period)
    t = torch.from_numpy(raw.view(np.int16)).to(gpu)
    out = im.scale_u16(t, crop, black, white, period=period).cpu().numpy()
    assert np.array_equal(out, ref)


def test_cfa_coeffs(oracle_lib, gpu):
    import torch
    import imops_b200 as im
    x = _rgb(1)
    ref = oracle_lib.wb(x, synthetic.WB)
    t = torch.from_numpy(x).to(gpu)
    im.cfa_coeffs(t, synthetic.WB)
    assert np.array_equal(t.cpu().numpy(), ref)


@pytest.mark.parametrize("ev", [0.0, 0.37, -1.25, 3.0])
def test_exp(oracle_lib, gpu, ev):
    import torch
    import imops_b200 as im
    x = _rgb(2)
    ref = oracle_lib.exposure(x, ev)
    t = torch.from_numpy(x).to(gpu)
    im.exp(t, ev)
    assert np.array_equal(t.cpu().numpy(), ref)


def test_baseline_exposure(oracle_lib, gpu):
    import torch
    import imops_b200 as im
    x = _rgb(3)
    ref, applied_ref = oracle_lib.baseline_exposure(x, 0.5, 1 / 200, 8.0, 200.0)
    t = torch.from_numpy(x).to(gpu)
    applied = im.baseline_exposure(t, 0.5, 1 / 200, 8.0, 200.0)
    assert applied and applied_ref
    assert np.array_equal(t.cpu().numpy(), ref)
    # missing EXIF: only the baseline EV is applied
    t = torch.from_numpy(x).to(gpu)
    assert not im.baseline_exposure(t, 0.0, 0.0, 8.0, 200.0)
    assert np.array_equal(t.cpu().numpy(), x)


def test_camera_forward_matrix_matches_oracle(oracle_lib):
    import imops_b200 as im
    ref = oracle_lib.camera_forward_matrix(synthetic.CALIB_D65).reshape(9)
    got = np.asarray(im.camera_forward_matrix(synthetic.CALIB_D65), dtype=np.float32)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("target", [0, 1, 3])
def test_camera_cst_linear_targets(oracle_lib, gpu, target):
    import torch
    import imops_b200 as im
    x = _rgb(4)
    ref = oracle_lib.camera_cst(x, synthetic.CALIB_D65, target)
    t = torch.from_numpy(x).to(gpu)
    im.camera_cst(t, synthetic.CALIB_D65, target)
    assert np.array_equal(t.cpu().numpy(), ref)


def test_camera_cst_srgb(oracle_lib, gpu):
    import torch
    import imops_b200 as im
    x = _rgb(5)
    ref = oracle_lib.camera_cst(x, synthetic.CALIB_D65, 2)
    t = torch.from_numpy(x).to(gpu)
    im.camera_cst(t, synthetic.CALIB_D65, 2)
    # the transfer uses CUDA powf (<= 2 ulp) against glibc powf
    np.testing.assert_allclose(t.cpu().numpy(), ref, rtol=1e-6, atol=1e-7)
