"""GPU parity of the 3-pass directional X-Trans demosaic
(imops_demosaic_markesteijn3) with its CPU specification (oracle/xtrans.c):
bit for bit on whole frames, under every CFA phase, and at full size through
crops (a pixel depends on inputs within radius 9, so the oracle run on a crop
equals the full-frame result inside the crop)."""
import numpy as np
import pytest

from imops_b200 import synthetic

pytestmark = pytest.mark.gpu


def _gpu(gpu, x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(gpu)


@pytest.mark.parametrize("H,W", [(64, 72), (97, 131), (200, 257), (20, 30), (21, 21), (22, 53), (53, 22), (75, 107),
                                 (142, 84)])
def test_matches_oracle_bit_exact(oracle_lib, gpu, H, W):
    import imops_b200 as im
    m = synthetic.mosaic_f32(H, W, seed=H + W, pattern=synthetic.XTRANS)
    ref = oracle_lib.markesteijn3(m, synthetic.XTRANS)
    out = im.demosaic_markesteijn3(_gpu(gpu, m), synthetic.XTRANS).cpu().numpy()
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("sx", range(6))
@pytest.mark.parametrize("sy", range(6))
def test_all_phases(oracle_lib, gpu, sx, sy):
    import imops_b200 as im
    m = synthetic.mosaic_f32(48, 54, seed=7 * sx + sy, pattern=synthetic.XTRANS)
    ref = oracle_lib.markesteijn3(m, synthetic.XTRANS, shift=(sx, sy))
    out = im.demosaic_markesteijn3(_gpu(gpu, m), synthetic.XTRANS, shift=(sx, sy)).cpu().numpy()
    assert np.array_equal(out, ref)


def test_full_size_crops(oracle_lib, gpu):
    """6032x4032 X-Trans (the 24 MP X-Trans workload): crops of the oracle."""
    import imops_b200 as im
    H, W = 4032, 6032
    m = synthetic.mosaic_f32(H, W, seed=1001, pattern=synthetic.XTRANS)
    out = im.demosaic_markesteijn3(_gpu(gpu, m), synthetic.XTRANS).cpu().numpy()
    assert np.isfinite(out).all()
    cols = synthetic.cfa_colors(synthetic.XTRANS, H, W)
    own = np.take_along_axis(out, cols[..., None].astype(np.int64), axis=2)[..., 0]
    assert np.array_equal(own, m)  # every CFA sample kept
    for (y, x) in [(0, 0), (0, W - 160), (H - 160, 0), (H - 160, W - 160), (2011, 3017), (1234, 77)]:
        crop = m[y:y + 160, x:x + 160]
        ref = oracle_lib.markesteijn3(crop, synthetic.XTRANS, shift=(x, y))
        # inside the crop away from its cut edges (the image's own edges count)
        y0 = 0 if y == 0 else 10
        x0 = 0 if x == 0 else 10
        y1 = 160 if y + 160 == H else 150
        x1 = 160 if x + 160 == W else 150
        assert np.array_equal(out[y + y0:y + y1, x + x0:x + x1], ref[y0:y1, x0:x1]), (y, x)


def test_edge_band_is_the_reference_mean(gpu):
    import imops_b200 as im
    m = synthetic.mosaic_f32(120, 150, seed=3, pattern=synthetic.XTRANS)
    t = _gpu(gpu, m)
    out = im.demosaic_markesteijn3(t, synthetic.XTRANS).cpu().numpy()
    mean = im.demosaic_markesteijn(t, synthetic.XTRANS).cpu().numpy()
    band = np.ones((120, 150), bool)
    band[10:-10, 10:-10] = False
    assert np.array_equal(out[band], mean[band])


def test_better_than_the_mean_on_a_scene(gpu):
    import imops_b200 as im
    H, W = 480, 640
    sc = synthetic.scene(H, W, seed=12)
    cols = synthetic.cfa_colors(synthetic.XTRANS, H, W)
    m = np.take_along_axis(sc, cols[..., None].astype(np.int64), axis=2)[..., 0].astype(np.float32)
    t = _gpu(gpu, m)
    d3 = im.demosaic_markesteijn3(t, synthetic.XTRANS).cpu().numpy()
    mean = im.demosaic_markesteijn(t, synthetic.XTRANS).cpu().numpy()
    psnr = lambda x: 10 * np.log10(1.0 / np.mean((x[12:-12, 12:-12] - sc[12:-12, 12:-12]) ** 2))
    assert psnr(d3) > psnr(mean) + 5.0


def test_rejects_bayer(gpu):
    import imops_b200 as im
    m = synthetic.mosaic_f32(32, 32, seed=1)
    with pytest.raises(im.ImopsError) as e:
        im.demosaic_markesteijn3(_gpu(gpu, m), "RGGB")
    assert e.value.code == 2


def test_other_6x6_cfa_generic_tiles(oracle_lib, gpu):
    """A 6x6 CFA that is not a shift of the X-Trans period (here a Bayer period
    tiled to 6x6) takes the generic tile kernel: bit for bit the same method."""
    import imops_b200 as im
    pattern = "RGRGRGGBGBGB" * 3
    m = synthetic.mosaic_f32(90, 118, seed=5, pattern=pattern)
    ref = oracle_lib.markesteijn3(m, pattern, shift=(1, 2))
    out = im.demosaic_markesteijn3(_gpu(gpu, m), pattern, shift=(1, 2)).cpu().numpy()
    assert np.array_equal(out, ref)


def test_other_6x6_cfa_window_masks(oracle_lib, gpu):
    """A 6x6 CFA with more than four red sites in some 3x3 window (up to eight
    around the green sites of row 1) is beyond the per-phase site lists, so the
    red / blue step tests the window masks instead: bit for bit the same
    method."""
    import imops_b200 as im
    pattern = "RRRRRR" "RGRBRG" "RRRRRR" "GBGBGB" "RRRRRR" "BGBGBG"
    m = synthetic.mosaic_f32(90, 118, seed=6, pattern=pattern)
    ref = oracle_lib.markesteijn3(m, pattern, shift=(2, 1))
    out = im.demosaic_markesteijn3(_gpu(gpu, m), pattern, shift=(2, 1)).cpu().numpy()
    assert np.array_equal(out, ref)
