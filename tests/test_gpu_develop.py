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


@pytest.mark.parametrize("crop", [(0, 0, 600, 141), (5, 4, 590, 137)])
@pytest.mark.parametrize("cfa", [synthetic.XTRANS, "RGGB", "RGBG"])
def test_develop_mean_route_equals_staged(gpu, crop, cfa):
    """The 3x3-mean route of develop_u16 (scaling, then the mean with the
    colour epilogue applied before its store; "RGBG", no shift of RGGB,
    through the per-pixel mean) equals the separate calls, with gains and an
    ACEScg target, rows of several warps."""
    import torch
    import imops_b200 as im
    raw = torch.from_numpy(synthetic.mosaic_u16(150, 610, seed=24, pattern=cfa).view(np.int16)).to(gpu)
    p = _params(im, False, demosaic=1, target=im.CS_ACESCG, cfa=cfa.encode(), ev=(0.4, -0.2))
    period = (6, 6) if len(cfa) == 36 else (2, 2)
    fused = im.develop_u16(raw, crop, synthetic.BLACK, synthetic.WHITE, p, period=period)
    staged = _staged(im, gpu, raw, crop, p, False)
    assert torch.equal(fused, staged)


@pytest.mark.parametrize("cfa,period", [(synthetic.XTRANS, (6, 6)), (synthetic.XTRANS, (1, 1)), ("RGGB", (2, 2))])
def test_develop_mean_route_site_levels(gpu, cfa, period):
    """Per-site black and white levels over the level period: the develop
    route equals imops_scale_u16 then the mean."""
    import torch
    import imops_b200 as im
    raw = torch.from_numpy(synthetic.mosaic_u16(203, 433, seed=26, pattern=cfa).view(np.int16)).to(gpu)
    n = period[0] * period[1]
    rng = np.random.default_rng(7 + n)
    black = [float(v) for v in rng.uniform(580.0, 620.0, n).astype(np.float32)]
    white = [float(v) for v in rng.uniform(15000.0, 16383.0, n).astype(np.float32)]
    p = _params(im, False, demosaic=1, target=im.CS_CAMERA, cfa=cfa.encode())
    for i in range(4):
        p.wb[i] = 1.0
    crop = (7, 3, 420, 197)
    fused = im.develop_u16(raw, crop, black, white, p, period=period)
    m = im.scale_u16(raw, crop, black, white, period=period)
    staged = im.demosaic_markesteijn(m, cfa, shift=crop[:2])
    assert torch.equal(fused, staged)


def test_develop_f32_mean_route_equals_staged(gpu):
    import torch
    import imops_b200 as im
    m = torch.from_numpy(synthetic.mosaic_f32(97, 420, seed=25, pattern=synthetic.XTRANS)).to(gpu)
    p = _params(im, False, demosaic=1, target=im.CS_ACESCG, cfa=synthetic.XTRANS.encode(), ev=(0.25,))
    fused = im.develop_f32(m, p, shift=(2, 3))
    staged = im.demosaic_markesteijn(m, synthetic.XTRANS, shift=(2, 3))
    im.cfa_coeffs(staged, synthetic.WB)
    im.exp(staged, 0.25)
    im.camera_cst(staged, synthetic.CALIB_D65, im.CS_ACESCG)
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


LSB = 1.0 / 65535.0  # one 16-bit step of linear [0, 1]
FLIP_LSB = 8.0  # errors above this are AMaZE taking another branch in f32 than in f64


def test_forward_error_vs_fp64_in_lsb(oracle_lib, gpu):
    """Error of the forward against the FP64 oracle chain, in 16-bit LSB.  The
    colour forward (AMaZE + WB + camera matrix) equals the reference-order
    f32 chain bit for bit, so its error is the reference's own f32 error: a
    few pixels where a comparison in AMaZE resolves differently in f32 than in
    f64 (decision flips, counted separately), sub-LSB elsewhere.  The film
    forward (81-bin baseline, grain on) adds its f32 kernels' error."""
    import torch
    import imops_b200 as im
    H, W = 480, 768
    raw_np = synthetic.mosaic_u16(H, W, seed=31)
    raw = torch.from_numpy(raw_np.view(np.int16)).to(gpu)

    def chain(prec):
        m = oracle_lib.scale_u16(raw_np, (0, 0, W, H), synthetic.BLACK, synthetic.WHITE, precision=prec)
        rgb = oracle_lib.wb(oracle_lib.amaze(m, "RGGB", precision=prec), synthetic.WB, precision=prec)
        return oracle_lib.camera_cst(rgb, synthetic.CALIB_D65, oracle_lib.CS_ACESCG, precision=prec)

    c32, c64 = chain("f32"), chain("f64")
    colour = im.develop_u16(raw, (0, 0, W, H), synthetic.BLACK, synthetic.WHITE, _params(im, False)).cpu().numpy()
    assert np.array_equal(colour, c32)
    e = np.abs(colour.astype(np.float64) - c64) / LSB
    flip = e.max(axis=2) > FLIP_LSB
    ok = ~flip
    film = im.develop_u16(raw, (0, 0, W, H), synthetic.BLACK, synthetic.WHITE, _params(im, True)).cpu().numpy()
    f64 = oracle_lib.film_baseline(c64, oracle_lib.baseline_params(seed=3), precision="f64")
    ef = np.abs(film.astype(np.float64) - f64) / LSB
    figures = {
        "pixels": H * W, "colour_flips": int(flip.sum()), "colour_max_lsb": float(e[ok].max()),
        "colour_rms_lsb": float(np.sqrt((e[ok] ** 2).mean())), "film_max_lsb": float(ef[ok].max()),
        "film_rms_lsb": float(np.sqrt((ef[ok] ** 2).mean())), "film_max_lsb_all": float(ef.max()),
    }
    print("forward vs FP64:", figures)
    assert flip.sum() <= 5e-4 * H * W
    assert figures["colour_rms_lsb"] < 0.1
    # measured 1.23 LSB max, 0.003 RMS
    assert figures["film_max_lsb"] < 2.0 and figures["film_rms_lsb"] < 0.05


def test_forward_error_vs_fp64_24mp(oracle_lib, gpu):
    """The 24 MP forward of the benchmark (6048x4024 RGGB, seed 1002: AMaZE,
    WB, camera matrix to ACEScg, 81-bin film with halation and grain) against
    FP64 over the whole frame, max and RMS absolute error in linear [0, 1]
    and in 16-bit LSB, for both forms of the film's scan:
      colour  the colour forward against the FP64 colour chain; it equals the
              reference-order f32 chain bit for bit, so this is the
              reference's own f32 error.  AMaZE decision flips (more than
              8 LSB from FP64: a comparison resolved differently in f32) are
              counted apart;
      film    the film stage alone: its output against the FP64 film of the
              same f32 colour input;
      chain   the output against the FP64 chain end to end (flips apart): the
              film's density curves amplify the colour stage's own error."""
    import torch
    import imops_b200 as im
    H, W = 4024, 6048
    raw_np = synthetic.mosaic_u16(H, W, seed=1002)
    raw = torch.from_numpy(raw_np.view(np.int16)).to(gpu)
    colour = im.develop_u16(raw, (0, 0, W, H), synthetic.BLACK, synthetic.WHITE, _params(im, False)).cpu().numpy()
    p = _params(im, True)
    films = {}
    for name, scan in (("fp32", im.SCAN_FP32), ("bf16_tc", im.SCAN_BF16_TC)):
        p.baseline = im.baseline_film_defaults(seed=1002, scan=scan)
        films[name] = im.develop_u16(raw, (0, 0, W, H), synthetic.BLACK, synthetic.WHITE, p).cpu().numpy()
    c32 = oracle_lib.colour_chain(raw_np, synthetic.BLACK, synthetic.WHITE, synthetic.WB, synthetic.CALIB_D65, "f32")
    assert np.array_equal(colour, c32)
    del c32
    bp = oracle_lib.baseline_params(seed=1002)
    stage64 = oracle_lib.film_baseline(colour, bp, precision="f64")
    stage = {k: oracle_lib.error_figures(v, stage64) for k, v in films.items()}
    del stage64
    c64 = oracle_lib.colour_chain(raw_np, synthetic.BLACK, synthetic.WHITE, synthetic.WB, synthetic.CALIB_D65)
    flips = oracle_lib.decision_flips(colour, c64)
    ec = oracle_lib.error_figures(colour, c64, skip=flips)
    chain64 = oracle_lib.film_baseline(c64, bp, precision="f64")
    chain = {k: oracle_lib.error_figures(v, chain64, skip=flips) for k, v in films.items()}
    print(f"24 MP vs FP64: flips {int(flips.sum())} of {H * W}; colour {ec}; film stage {stage}; chain {chain}")
    assert flips.sum() <= 5e-4 * H * W
    assert ec["rms_lsb"] < 0.1
    for k in films:
        assert stage[k]["max_lsb"] < 2.0 and stage[k]["rms_lsb"] < 0.05, k
        assert chain[k]["rms_lsb"] < 0.05 and chain[k]["max_lsb"] < 100.0, k


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
