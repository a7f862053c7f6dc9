"""run_pixel_pipeline_c (the reference-facing C-ABI) on the GPU."""
import numpy as np
import pytest

from imops_b200 import synthetic

pytestmark = pytest.mark.gpu

CFG_FILM = """
[[pipeline_modules]]
name = "Demosaic"
algorithm = "amaze"
[[pipeline_modules]]
name = "CFACoeffs"
[[pipeline_modules]]
name = "CST"
target_color_space = "AcesCg"
[[pipeline_modules]]
name = "Film"
stock = "Baseline81"
film_format = "Film35mm"
seed = 3
output = "NegativeLinear"
"""


def _meta(**kw):
    from imops_b200.pipeline import make_meta
    d = dict(cfa="RGGB", crop=(0, 0, 0, 0), wb=synthetic.WB, calibration=synthetic.CALIB_D65,
             black=synthetic.BLACK, white=synthetic.WHITE)
    d.update(kw)
    return make_meta(**d)


def test_pipeline_u16_film_equals_develop(gpu):
    import torch
    import imops_b200 as im
    from imops_b200.pipeline import Image, parse_config, run_pixel_pipeline
    raw = synthetic.mosaic_u16(330, 410, seed=31)
    crop = (1, 3, 400, 320)
    img = Image.from_u16(raw, _meta(crop=crop))
    run_pixel_pipeline(img, parse_config(CFG_FILM))
    w, h, cs = img.info()
    assert (w, h, cs) == (400, 320, im.CS_ACESCG)
    got = img.rgb_f32()
    p = im.DevelopParams()
    p.demosaic, p.cfa, p.clip_pt = 0, b"RGGB", 1.0
    for i in range(4):
        p.wb[i] = synthetic.WB[i]
    p.target = im.CS_ACESCG
    for i in range(9):
        p.calib_d65[i] = synthetic.CALIB_D65[i]
    p.film = 1
    p.film_params = im.FilmParams(im.STOCK_BASELINE81, 0, 3, 0, -1.0, 1)
    p.baseline = im.baseline_film_defaults(seed=3)
    ref = im.develop_u16(torch.from_numpy(raw.view(np.int16)).to(gpu), crop, synthetic.BLACK, synthetic.WHITE,
                         p).cpu().numpy()
    assert np.array_equal(got, ref)


def test_pipeline_markesteijn_exp_linear_srgb(gpu, oracle_lib):
    from imops_b200.pipeline import Image, parse_config, run_pixel_pipeline
    m = synthetic.mosaic_f32(96, 120, seed=32, pattern=synthetic.XTRANS)
    cfg = ('[[pipeline_modules]]\nname = "Demosaic"\nalgorithm = "markesteijn"\n'
           '[[pipeline_modules]]\nname = "Exp"\nev = 0.5\n'
           '[[pipeline_modules]]\nname = "CFACoeffs"\n'
           '[[pipeline_modules]]\nname = "CST"\ntarget_color_space = "LinearSrgb"\n')
    img = Image.from_mosaic(m, _meta(cfa=synthetic.XTRANS, crop=(2, 1, 0, 0)))
    run_pixel_pipeline(img, parse_config(cfg))
    got = img.rgb_f32()
    ref = oracle_lib.mean3x3(m, synthetic.XTRANS, shift=(2, 1))
    ref = oracle_lib.exposure(ref, 0.5)
    ref = oracle_lib.wb(ref, synthetic.WB)
    ref = oracle_lib.camera_cst(ref, synthetic.CALIB_D65, oracle_lib.CS_LINEAR_SRGB)
    assert np.array_equal(got, ref)


def test_pipeline_markesteijn_fused_chain_u16(gpu, oracle_lib):
    """A u16 X-Trans frame through Demosaic(markesteijn) with CFACoeffs, Exp and
    CST fused into the 3x3 mean's store: equal to the oracle chain."""
    from imops_b200.pipeline import Image, parse_config, run_pixel_pipeline
    raw = synthetic.mosaic_u16(90, 126, seed=34, pattern=synthetic.XTRANS)
    cfg = ('[[pipeline_modules]]\nname = "Demosaic"\nalgorithm = "markesteijn"\n'
           '[[pipeline_modules]]\nname = "CFACoeffs"\n'
           '[[pipeline_modules]]\nname = "Exp"\nev = 0.4\n'
           '[[pipeline_modules]]\nname = "CST"\ntarget_color_space = "AcesCg"\n')
    img = Image.from_u16(raw, _meta(cfa=synthetic.XTRANS, crop=(3, 2, 114, 80)))
    run_pixel_pipeline(img, parse_config(cfg))
    got = img.rgb_f32()
    m = oracle_lib.scale_u16(raw, (3, 2, 114, 80), synthetic.BLACK, synthetic.WHITE, cfa_period=(1, 1))
    ref = oracle_lib.mean3x3(m, synthetic.XTRANS, shift=(3, 2))
    ref = oracle_lib.wb(ref, synthetic.WB)
    ref = oracle_lib.exposure(ref, 0.4)
    ref = oracle_lib.camera_cst(ref, synthetic.CALIB_D65, oracle_lib.CS_ACESCG)
    assert np.array_equal(got, ref)


def test_pipeline_amaze_fused_chain_equals_oracle(gpu, oracle_lib):
    from imops_b200.pipeline import Image, parse_config, run_pixel_pipeline
    m = synthetic.mosaic_f32(256, 320, seed=33)
    chain = ('[[pipeline_modules]]\nname = "Demosaic"\nalgorithm = "amaze"\n'
             '[[pipeline_modules]]\nname = "CFACoeffs"\n'
             '[[pipeline_modules]]\nname = "Exp"\nev = -0.25\n'
             '[[pipeline_modules]]\nname = "BaselineExposureCompensation"\n'
             '[[pipeline_modules]]\nname = "CST"\ntarget_color_space = "AcesCg"\n')
    meta = dict(baseline_exposure=0.3, shutter=1 / 250, f_number=5.6, iso=400.0)
    img = Image.from_mosaic(m, _meta(**meta))
    run_pixel_pipeline(img, parse_config(chain))
    got = img.rgb_f32()
    ref = oracle_lib.amaze(m, "RGGB")
    ref = oracle_lib.wb(ref, synthetic.WB)
    ref = oracle_lib.exposure(ref, -0.25)
    ref, _ = oracle_lib.baseline_exposure(ref, 0.3, 1 / 250, 5.6, 400.0)
    ref = oracle_lib.camera_cst(ref, synthetic.CALIB_D65, oracle_lib.CS_ACESCG)
    assert np.array_equal(got, ref)  # the modules fused into AMaZE's output stage are bit-exact
    # then AcesCg -> Srgb (colour space to colour space; the `color` crate step is unpinned)
    img = Image.from_mosaic(m, _meta(**meta))
    run_pixel_pipeline(img, parse_config(chain + '[[pipeline_modules]]\nname = "CST"\ntarget_color_space = "Srgb"\n'))
    got = img.rgb_f32()
    M = np.array([[0.6624541811, 0.1340042065, 0.1561876870], [0.2722287168, 0.6740817658, 0.0536895174],
                  [-0.0055746495, 0.0040607335, 1.0103391003]])
    X2S = np.array([[12831 / 3959, -329 / 214, -1974 / 3959], [-851781 / 878810, 1648619 / 878810, 36519 / 878810],
                    [705 / 12673, -2585 / 12673, 705 / 667]])
    lin = ref.astype(np.float64) @ (X2S @ M).T
    a = np.abs(lin)
    enc = np.where(a <= 0.0031308, 12.92 * a, 1.055 * a ** (1 / 2.4) - 0.055) * np.sign(lin)
    # two f32 mat-vecs with cancellation on values ~10: relative to the pixel's scale
    scale = np.abs(ref).max(axis=2, keepdims=True) + 1e-3
    assert (np.abs(got - enc) / scale).max() < 2e-5


def test_pipeline_colorneg_film_matches_oracle(gpu, oracle_lib):
    from imops_b200.pipeline import Image, parse_config, run_pixel_pipeline
    rng = np.random.default_rng(34)
    rel = (rng.random((48, 2048, 3)) ** 2).astype(np.float32)
    cfg = ('[[pipeline_modules]]\nname = "BaselineExposureCompensation"\n'
           '[[pipeline_modules]]\nname = "Film"\nstock = "ColorNeg200"\nfilm_format = "Film35mm"\nseed = 5\n'
           'output = "PositiveLinear"\n')
    img = Image.from_rgb(rel, 3, _meta(shutter=1 / 200, f_number=8.0, iso=200.0))
    run_pixel_pipeline(img, parse_config(cfg))
    got = img.rgb_f32()
    x, _ = oracle_lib.baseline_exposure(rel, 0.0, 1 / 200, 8.0, 200.0)
    ref = oracle_lib.film_process(x, stock=1, seed=5, output=1, shutter=1 / 200)
    assert np.abs(got - ref).max() < 1e-4


@pytest.mark.parametrize("name,sid", [("Portra400", 2), ("Ektar100", 3), ("FujiPro400H", 4),
                                      ("EktachromeE100", 5), ("TriX400", 6)])
def test_pipeline_stock_names(gpu, oracle_lib, name, sid):
    """modules.rs:846-853: the config's stock string selects the StockId."""
    from imops_b200.pipeline import Image, parse_config, run_pixel_pipeline
    rng = np.random.default_rng(40 + sid)
    rel = (rng.random((32, 512, 3)) ** 2).astype(np.float32)
    cfg = ('[[pipeline_modules]]\nname = "BaselineExposureCompensation"\n'
           f'[[pipeline_modules]]\nname = "Film"\nstock = "{name}"\nfilm_format = "Film35mm"\nseed = 7\n'
           'output = "PositiveLinear"\n')
    img = Image.from_rgb(rel, 3, _meta(shutter=1 / 125, f_number=5.6, iso=400.0))
    run_pixel_pipeline(img, parse_config(cfg))
    got = img.rgb_f32()
    x, _ = oracle_lib.baseline_exposure(rel, 0.0, 1 / 125, 5.6, 400.0)
    ref = oracle_lib.film_process(x, stock=sid, seed=7, output=1, shutter=1 / 125)
    assert np.abs(got - ref).max() < 1e-4


def test_pipeline_u8_export(gpu):
    from imops_b200.pipeline import Image
    x = np.array([[[-0.5, 0.0, 0.25], [0.5, 0.999, 1.7]]], np.float32)
    img = Image.from_rgb(x, 1)
    u8 = img.rgb_u8()
    ref = (np.clip(x, 0, 1) * np.float32(255)).astype(np.uint8)
    assert np.array_equal(u8, ref)
    meta = img.metadata()
    assert meta["width"] == 2 and meta["color_space"] == "LinearSrgb"


def test_pipeline_errors(gpu):
    import imops_b200 as im
    from imops_b200.pipeline import Image, get_last_error, parse_config, run_pixel_pipeline
    rgb = np.zeros((8, 8, 3), np.float32)
    film = parse_config('[[pipeline_modules]]\nname = "Film"\nstock = "ColorNeg200"\nfilm_format = "Film35mm"\n'
                        'seed = 1\noutput = "NegativeLinear"\n')
    with pytest.raises(im.ImopsError) as e:
        run_pixel_pipeline(Image.from_rgb(rgb, 2), film)
    assert "WrongColorSpace" in e.value.message and "Srgb" in e.value.message
    assert "WrongColorSpace" in get_last_error()
    with pytest.raises(im.ImopsError) as e:
        run_pixel_pipeline(Image.from_rgb(rgb, 3), parse_config('[[pipeline_modules]]\nname = "BM3D"\nintensity = 1\n'))
    assert e.value.code == 10
    from imops_b200.pipeline import make_meta
    with pytest.raises(im.ImopsError) as e:
        run_pixel_pipeline(Image.from_rgb(rgb, -1, make_meta()), parse_config('[[pipeline_modules]]\nname = "CFACoeffs"\n'))
    assert "wb_coeffs" in e.value.message


@pytest.mark.parametrize("pattern", ["RGGB", "XTRANS"])
@pytest.mark.parametrize("raw_kind", ["u16", "f32"])
@pytest.mark.parametrize("target", ["AcesCg", "Srgb"])
def test_pipeline_markesteijn_fused_chain_variants(gpu, oracle_lib, pattern, raw_kind, target):
    """Demosaic(markesteijn) + CFACoeffs + BaselineExposureCompensation + CST
    fused into the 3x3 mean's store, on Bayer (the aligned RGGB kernel) and
    X-Trans, from a u16 frame and from an f32 mosaic, frames wider than one
    192-pixel warp run (the interior aligned path and the float4 stores):
    bit-exact to the oracle chain for linear targets, sRGB within 1e-6 of
    scale (its transfer function is the f32 pow)."""
    from imops_b200.pipeline import Image, parse_config, run_pixel_pipeline
    cfa = synthetic.XTRANS if pattern == "XTRANS" else "RGGB"
    H, W, crop = 70, 430, (3, 2, 418, 60)
    cfg = ('[[pipeline_modules]]\nname = "Demosaic"\nalgorithm = "markesteijn"\n'
           '[[pipeline_modules]]\nname = "CFACoeffs"\n'
           '[[pipeline_modules]]\nname = "BaselineExposureCompensation"\n'
           f'[[pipeline_modules]]\nname = "CST"\ntarget_color_space = "{target}"\n')
    meta = dict(cfa=cfa, baseline_exposure=0.3, shutter=1 / 250, f_number=5.6, iso=400.0)
    if raw_kind == "u16":
        raw = synthetic.mosaic_u16(H, W, seed=35, pattern=cfa)
        img = Image.from_u16(raw, _meta(crop=crop, **meta))
        m = oracle_lib.scale_u16(raw, crop, synthetic.BLACK, synthetic.WHITE, cfa_period=(1, 1))
    else:
        full = synthetic.mosaic_f32(H, W, seed=35, pattern=cfa)
        m = np.ascontiguousarray(full[crop[1]:crop[1] + crop[3], crop[0]:crop[0] + crop[2]])
        img = Image.from_mosaic(m, _meta(crop=(crop[0], crop[1], 0, 0), **meta))
    run_pixel_pipeline(img, parse_config(cfg))
    got = img.rgb_f32()
    ref = oracle_lib.mean3x3(m, cfa, shift=crop[:2])
    ref = oracle_lib.wb(ref, synthetic.WB)
    ref, applied = oracle_lib.baseline_exposure(ref, 0.3, 1 / 250, 5.6, 400.0)
    assert applied
    cs = oracle_lib.CS_SRGB if target == "Srgb" else oracle_lib.CS_ACESCG
    ref = oracle_lib.camera_cst(ref, synthetic.CALIB_D65, cs)
    assert got.shape == (crop[3], crop[2], 3)
    if target == "Srgb":
        scale = np.abs(ref).max(axis=2, keepdims=True) + 1e-3
        assert (np.abs(got - ref) / scale).max() < 1e-6
    else:
        assert np.array_equal(got, ref)


def test_pipeline_markesteijn_nothing_fused(gpu, oracle_lib):
    """A 3x3-mean Demosaic followed by no foldable module keeps its plain
    output stage: equal to the mean itself, then Contrast as its own pass."""
    from imops_b200.pipeline import Image, parse_config, run_pixel_pipeline
    m = synthetic.mosaic_f32(64, 400, seed=36, pattern=synthetic.XTRANS)
    cfg = ('[[pipeline_modules]]\nname = "Demosaic"\nalgorithm = "markesteijn"\n'
           '[[pipeline_modules]]\nname = "Contrast"\nc = 1.2\n')
    img = Image.from_mosaic(m, _meta(cfa=synthetic.XTRANS))
    run_pixel_pipeline(img, parse_config(cfg))
    got = img.rgb_f32()
    ref = oracle_lib.contrast(oracle_lib.mean3x3(m, synthetic.XTRANS), 1.2)
    nan = np.isnan(ref)  # negative means (sensor noise below black) to a fractional power
    assert np.array_equal(np.isnan(got), nan)
    assert np.abs(got[~nan] - ref[~nan]).max() <= 2e-5 * max(1.0, float(np.abs(ref[~nan]).max()))
    assert img.info()[2] == -1  # camera RGB: no colour space set
