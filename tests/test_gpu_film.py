"""GPU film simulation against the CPU oracle.

Reference stocks: the oracle restates film::process in the reference's
precision mix (f64 spectral work, f32 planes); the GPU runs everything in
f32 with the spectral exposure collapsed to a 3xE matrix.  Tolerance: 1e-4
absolute in linear [0, 1] (the path's stated bar), with grain off and on
(the SplitMix64 noise is generated bit-identically on the GPU).
Baseline preset: GPU (f32, rank-3 exposure) against the FP64 oracle that
integrates all 81 bins per pixel.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _abs_scene(H, W, seed, box_iso=200.0):
    import oracle  # noqa: F401
    rng = np.random.default_rng(seed)
    rel = (rng.random((H, W, 3)) ** 2 * 1.2).astype(np.float32)
    rel[: H // 4] = 0.0  # unexposed band
    g = np.float32(12.5 * 64.0)  # relative -> absolute at sunny-16, t*S = 1
    return (rel * g).astype(np.float32)


def _run(gpu, x, **kw):
    import torch
    import imops_b200 as im
    t = torch.from_numpy(x).to(gpu)
    im.film_process(t, **kw)
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("grain", [False, True])
@pytest.mark.parametrize("output", [0, 1])
def test_colorneg200_strip_matches_oracle(oracle_lib, gpu, grain, output):
    # a 6048-wide strip: 35 mm pitch 5.95 um, so every blur has its real radius
    x = _abs_scene(64, 6048, seed=3)
    ref = oracle_lib.film_process(x, stock=1, seed=7, output=output, grain=grain, precision="f32")
    out = _run(gpu, x, stock=1, seed=7, output=output, grain=grain)
    err = np.abs(out - ref)
    assert np.isfinite(out).all()
    assert err.max() < TOL, f"max {err.max():.3g} rms {np.sqrt((err**2).mean()):.3g}"


def test_colorneg200_small_frame(oracle_lib, gpu):
    x = _abs_scene(48, 64, seed=4)
    ref = oracle_lib.film_process(x, stock=1, seed=1, grain=True, precision="f32")
    out = _run(gpu, x, stock=1, seed=1, grain=True)
    assert np.abs(out - ref).max() < TOL


def test_bwstub_matches_oracle(oracle_lib, gpu):
    x = _abs_scene(40, 2048, seed=5, box_iso=100.0)
    ref = oracle_lib.film_process(x, stock=0, seed=2, grain=True, precision="f32")
    out = _run(gpu, x, stock=0, seed=2, grain=True)
    assert np.abs(out - ref).max() < TOL


def test_unexposed_scans_to_dmin(gpu):
    # film/mod.rs:257-273: unexposed -> peak ~1; stock_dmin_drives_invert:
    # normalised Dmin peak is 1 with R > G > B (orange mask)
    x = np.zeros((16, 16, 3), np.float32)
    out = _run(gpu, x, stock=1, grain=False)
    peak = out.max(axis=2)
    assert np.abs(peak - 1.0).max() < 1e-5
    m = out.reshape(-1, 3).mean(0)
    assert m[0] > m[1] > m[2]


def test_wrong_color_space_and_dimensions(gpu):
    import torch
    import imops_b200 as im
    t = torch.zeros((8, 8, 3), device=gpu)
    with pytest.raises(im.ImopsError) as e:
        im.film_process(t, color_space=im.CS_SRGB)
    assert e.value.code == 6
    with pytest.raises(im.ImopsError) as e:
        im.film_process(torch.zeros((0, 8, 3), device=gpu))
    assert e.value.code == 7


@pytest.mark.parametrize("scan", [0, 1], ids=["fp32", "bf16_tc"])
@pytest.mark.parametrize("grain_on", [0, 1])
def test_baseline_preset_against_fp64_oracle(oracle_lib, gpu, grain_on, scan):
    """The 81-bin preset with the scan's contractions on the CUDA cores
    (FP32) and on the tensor cores (BF16 hi/lo, FP32 accumulation)."""
    import imops_b200 as im
    rng = np.random.default_rng(11)
    x = (rng.random((96, 160, 3)) * 1.1).astype(np.float32)  # relative ACEScg incl. highlights > 0.8
    x[20:40, 30:60] = 1.05
    p_or = oracle_lib.baseline_params(grain_on=grain_on, seed=5)
    ref = oracle_lib.film_baseline(x, p_or, precision="f64")
    p = im.baseline_film_defaults(grain_on=grain_on, seed=5, scan=scan)
    out = _run(gpu, x, stock=im.STOCK_BASELINE81, baseline=p)
    err = np.abs(out - ref)
    assert err.max() < TOL, f"max {err.max():.3g} rms {np.sqrt((err**2).mean()):.3g}"


@pytest.mark.parametrize("H,W", [(128, 32), (1, 1), (37, 45), (300, 1000), (257, 129)])
def test_tensor_core_scan_shapes(oracle_lib, gpu, H, W):
    """The tensor-core scan on frames that fill its 128-pixel MMA tiles
    partly (columns past the width and rows past the height are computed as
    zeros and not stored): within 1e-4 of the FP64 oracle, and no MMA
    completion lost."""
    import ctypes

    import imops_b200 as im
    x = (synthetic_scene(H, W, seed=H * 7 + W) * 1.2).astype(np.float32)
    p_or = oracle_lib.baseline_params(grain_on=1, seed=9)
    ref = oracle_lib.film_baseline(x, p_or, precision="f64")
    p = im.baseline_film_defaults(grain_on=1, seed=9, scan=im.SCAN_BF16_TC)
    out = _run(gpu, x, stock=im.STOCK_BASELINE81, baseline=p)
    assert np.abs(out - ref).max() < TOL
    n = ctypes.c_uint()
    im.check(im.lib().imops_tensor_timeouts(ctypes.byref(n)))
    assert n.value == 0


def synthetic_scene(H, W, seed):
    from imops_b200 import synthetic
    return synthetic.scene(H, W, seed=seed)


def test_scan_arm_rejects_unknown(gpu):
    import torch
    import imops_b200 as im
    t = torch.zeros((8, 8, 3), device=gpu)
    with pytest.raises(im.ImopsError) as e:
        im.film_process(t, stock=im.STOCK_BASELINE81, baseline=im.baseline_film_defaults(scan=7))
    assert e.value.code == 1


# Portra400, Ektar100, FujiPro400H (7 emulsions), EktachromeE100 (reversal),
# TriX400 (two silver layers)
OTHER_STOCKS = [2, 3, 4, 5, 6]


@pytest.mark.parametrize("stock", OTHER_STOCKS)
@pytest.mark.parametrize("grain,output", [(False, 0), (True, 0), (True, 1)])
def test_other_stocks_strip_match_oracle(oracle_lib, gpu, stock, grain, output):
    x = _abs_scene(32, 6048, seed=10 + stock)
    ref = oracle_lib.film_process(x, stock=stock, seed=5, output=output, grain=grain, precision="f32")
    out = _run(gpu, x, stock=stock, seed=5, output=output, grain=grain)
    err = np.abs(out - ref)
    assert np.isfinite(out).all()
    assert err.max() < TOL, f"max {err.max():.3g} rms {np.sqrt((err**2).mean()):.3g}"


@pytest.mark.parametrize("stock", OTHER_STOCKS)
def test_other_stocks_small_frame(oracle_lib, gpu, stock):
    x = _abs_scene(48, 64, seed=20 + stock)
    ref = oracle_lib.film_process(x, stock=stock, seed=3, grain=True, precision="f32")
    out = _run(gpu, x, stock=stock, seed=3, grain=True)
    assert np.abs(out - ref).max() < TOL


@pytest.mark.parametrize("stock", [0, 1, 2, 5, 6])
@pytest.mark.parametrize("output", [0, 1])
def test_film_sub_stages_chain_to_film_process(gpu, stock, output):
    """expose -> halation -> develop -> grain -> scan -> invert as separate
    C-ABI calls equals film_process bit for bit (film/mod.rs:77-129)."""
    import torch
    import imops_b200 as im
    x = torch.from_numpy(_abs_scene(96, 160, seed=30 + stock)).to(gpu)
    ref = im.film_process(x.clone(), stock=stock, seed=9, output=output, grain=True)
    st = im.FilmStages(stock=stock, seed=9, output=output, grain=True)
    assert st.layers >= 1
    got = st.run(x.clone())
    torch.cuda.synchronize()
    assert torch.equal(got, ref)


def test_film_sub_stages_shapes_and_errors(gpu):
    import torch
    import imops_b200 as im
    st = im.FilmStages(stock=im.STOCK_PORTRA400)
    x = torch.from_numpy(_abs_scene(32, 48, seed=3)).to(gpu)
    planes = st.expose(x)
    assert planes.shape == (st.layers, 32, 48) and st.layers == 6
    with pytest.raises(im.ImopsError) as e:
        im.FilmStages(stock=im.STOCK_BASELINE81)
    assert e.value.code == 8
