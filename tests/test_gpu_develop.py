"""The fused forward (imops_develop_*) equals the stage entry points run in
the reference's module order, and the oracle chain."""
import numpy as np
import pytest

from imops_b200 import synthetic

pytestmark = pytest.mark.gpu


def _params(im, film, demosaic=0, target=3, cfa=b"RGGB", ev=()):
    p = im.DevelopParams()
    p.demosaic = demosaic
    p.cfa = cfa
    p.clip_pt = 1.0
    for i in range(4):
        p.wb[i] = synthetic.WB[i]
    p.n_gain = len(ev)
    for i, v in enumerate(ev):
        p.ev[i] = v
    p.target = target
    for i in range(9):
        p.calib_d65[i] = synthetic.CALIB_D65[i]
    p.film = int(film)
    p.film_params = im.FilmParams(im.STOCK_BASELINE81, 0, 1, 0, -1.0, 1)
    p.baseline = im.baseline_film_defaults(seed=3)
    return p


def _staged(im, gpu, raw, crop, p, film):
    import torch
    x, y, w, h = crop
    m = im.scale_u16(raw, crop, synthetic.BLACK, synthetic.WHITE)
    out = im.demosaic_amaze(m, "RGGB", shift=(x, y)) if p.demosaic == 0 else \
        im.demosaic_markesteijn(m, p.cfa.decode(), shift=(x, y))
    im.cfa_coeffs(out, synthetic.WB)
    for i in range(p.n_gain):
        im.exp(out, p.ev[i])
    if p.target != im.CS_CAMERA:
        im.camera_cst(out, synthetic.CALIB_D65, p.target)
    if film:
        im.film_process(out, stock=im.STOCK_BASELINE81, baseline=p.baseline)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("film", [False, True])
@pytest.mark.parametrize("crop", [(0, 0, 400, 320), (1, 3, 400, 320)])
def test_develop_u16_equals_staged(gpu, film, crop):
    import torch
    import imops_b200 as im
    raw = torch.from_numpy(synthetic.mosaic_u16(330, 410, seed=21).view(np.int16)).to(gpu)
    p = _params(im, film, ev=(0.3,))
    fused = im.develop_u16(raw, crop, synthetic.BLACK, synthetic.WHITE, p)
    staged = _staged(im, gpu, raw, crop, p, film)
    assert torch.equal(fused, staged)


def test_develop_markesteijn_xtrans(gpu):
    import torch
    import imops_b200 as im
    raw = torch.from_numpy(synthetic.mosaic_u16(120, 150, seed=22, pattern=synthetic.XTRANS).view(np.int16)).to(gpu)
    p = _params(im, False, demosaic=1, target=1, cfa=synthetic.XTRANS.encode())
    crop = (2, 1, 144, 114)
    fused = im.develop_u16(raw, crop, synthetic.BLACK, synthetic.WHITE, p)
    staged = _staged(im, gpu, raw, crop, p, False)
    assert torch.equal(fused, staged)


def test_develop_matches_oracle_chain(oracle_lib, gpu):
    import torch
    import imops_b200 as im
    raw_np = synthetic.mosaic_u16(256, 320, seed=23)
    raw = torch.from_numpy(raw_np.view(np.int16)).to(gpu)
    p = _params(im, True)
    out = im.develop_u16(raw, (0, 0, 320, 256), synthetic.BLACK, synthetic.WHITE, p).cpu().numpy()
    m = oracle_lib.scale_u16(raw_np, (0, 0, 320, 256), synthetic.BLACK, synthetic.WHITE)
    rgb = oracle_lib.amaze(m, "RGGB")
    rgb = oracle_lib.wb(rgb, synthetic.WB)
    rgb = oracle_lib.camera_cst(rgb, synthetic.CALIB_D65, oracle_lib.CS_ACESCG)
    ref = oracle_lib.film_baseline(rgb, oracle_lib.baseline_params(seed=3), precision="f64")
    assert np.abs(out - ref).max() < 1e-4


def test_develop_film_requires_acescg(gpu):
    import torch
    import imops_b200 as im
    raw = torch.zeros((64, 64), dtype=torch.int16, device=gpu)
    p = _params(im, True, target=1)
    with pytest.raises(im.ImopsError) as e:
        im.develop_u16(raw, (0, 0, 64, 64), synthetic.BLACK, synthetic.WHITE, p)
    assert e.value.code == 6


def test_develop_largest_frame_45mp(gpu):
    """The fused forward (AMaZE + colour + 81-bin film, grain on) on an
    8256x5504 frame: runs within the working sets and stays finite."""
    import torch
    import imops_b200 as im
    from imops_b200 import synthetic
    H, W = 5504, 8256
    raw = torch.from_numpy(synthetic.mosaic_u16(H, W, seed=46).view(np.int16)).to(gpu)
    p = im.DevelopParams()
    p.demosaic, p.cfa, p.clip_pt = im.DEMOSAIC_AMAZE, b"RGGB", 1.0
    for i in range(4):
        p.wb[i] = synthetic.WB[i]
    p.target = im.CS_ACESCG
    for i in range(9):
        p.calib_d65[i] = synthetic.CALIB_D65[i]
    p.film = 1
    p.film_params = im.FilmParams(im.STOCK_BASELINE81, 0, 1, 0, -1.0, 1)
    p.baseline = im.baseline_film_defaults()
    out = im.develop_u16(raw, (0, 0, W, H), synthetic.BLACK, synthetic.WHITE, p)
    torch.cuda.synchronize()
    assert out.shape == (H, W, 3)
    assert bool(torch.isfinite(out).all())
