"""GPU parity of the display stages (highlight reconstruction, contrast,
gamma, LCH, sigmoid tone map) and of the colour-space conversions to and from
Oklch against the CPU oracle, through the C-ABI and through the pipeline
C-ABI (where a run of per-pixel modules is one launch)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# f32 kernels against the f32 restatement: only the math library differs
# (CUDA's cbrtf / atan2f / sinf / cosf / powf against glibc's, <= 2 ulp each)
TOL = 2e-5


def _rgb(seed, n=65537, lo=-0.3, hi=3.0):
    rng = np.random.default_rng(seed)
    x = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    x[:64] = rng.uniform(0.0, 1.0, (64, 1)).astype(np.float32)  # grays
    x[64:72] = 0.0
    return x


def _close(got, ref, tol=TOL, ref64=None):
    """got within tol (relative to max(1, |ref|)) of the f32 oracle.  With
    ref64: got's worst error against the FP64 oracle is at most twice the f32
    oracle's worst error over the same inputs (or tol): the kernel is in the
    accuracy class of the reference's own f32 arithmetic.  Per value the two
    f32 results may differ by more than tol where the conversion is
    ill-conditioned: a 1-ulp cbrtf difference, cubed and mixed by Oklab's
    inverse matrix (coefficients ~4), then scaled by the sRGB encode's slope
    of 12.92 near zero, moves an output by ~5e-5."""
    assert got.shape == ref.shape
    nan = np.isnan(ref)
    assert np.array_equal(np.isnan(got), nan), "NaN positions differ"
    g, r = got[~nan].astype(np.float64), ref[~nan].astype(np.float64)
    scale = np.maximum(1.0, np.abs(r))
    if ref64 is None:
        err = np.abs(g - r) / scale
        assert err.max() < tol, f"max rel err {err.max():.3g}"
        return
    r64 = ref64[~nan]
    err_gpu = (np.abs(g - r64) / scale).max()
    err_cpu = (np.abs(r - r64) / scale).max()
    assert err_gpu <= max(tol, 2.0 * err_cpu), f"GPU err {err_gpu:.3g}, f32 oracle err {err_cpu:.3g}"


def _gpu(gpu, x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(gpu)


def test_highlight_reconstruction(oracle_lib, gpu):
    import imops_b200 as im
    x = _rgb(1)
    wb = [2.0, 0.9, 1.5, 0.0]
    t = _gpu(gpu, x)
    im.highlight_reconstruction(t, wb)
    got = t.cpu().numpy()
    ref = oracle_lib.highlight(x, wb)
    assert np.array_equal(got, ref)  # no math-library call: bit-exact
    k = _gpu(gpu, np.array([[0.6, 0.4, 0.8]], np.float32))
    im.highlight_reconstruction(k, [1, 1, 1, 1])
    assert abs(float(k[0, 1]) - 0.52) < 1e-6


@pytest.mark.parametrize("c", [1.0, 1.35, 0.7])
def test_contrast(oracle_lib, gpu, c):
    import imops_b200 as im
    x = _rgb(2)
    t = _gpu(gpu, x)
    im.contrast(t, c)
    _close(t.cpu().numpy(), oracle_lib.contrast(x, c), ref64=oracle_lib.contrast(x, c, "f64"))


@pytest.mark.parametrize("g", [2.2, 2.4, 1.0, 0.0])
def test_gamma(oracle_lib, gpu, g):
    import imops_b200 as im
    x = _rgb(3)
    t = _gpu(gpu, x)
    im.gamma(t, g)
    ref = oracle_lib.gamma(x, g)
    if g == 0.0:  # exponent 1e6: results are 0, 1 or overflow alike
        got = t.cpu().numpy()
        assert np.array_equal(np.isinf(got), np.isinf(ref))
        fin = np.isfinite(ref)
        assert np.abs(got[fin] - ref[fin]).max() < 1e-3
        return
    _close(t.cpu().numpy(), ref, ref64=oracle_lib.gamma(x, g, "f64"))


CS = [0, 1, 2, 3, 4]  # XyzD65, LinearSrgb, Srgb, AcesCg, Oklch


def _space_input(cs, seed):
    x = _rgb(seed, lo=-0.1, hi=1.5)
    if cs == 4:  # Oklch: L, C, hue in degrees
        rng = np.random.default_rng(seed)
        x[:, 0] = rng.uniform(0.0, 1.2, len(x))
        x[:, 1] = rng.uniform(0.0, 0.4, len(x))
        x[:, 2] = rng.uniform(0.0, 360.0, len(x))
    return x


@pytest.mark.parametrize("src", CS)
@pytest.mark.parametrize("dst", CS)
def test_cst_pairs(oracle_lib, gpu, src, dst):
    import imops_b200 as im
    x = _space_input(src, 10 + src)
    t = _gpu(gpu, x)
    im.cst(t, src, dst)
    got = t.cpu().numpy()
    ref = oracle_lib.cst_space(x, src, dst)
    ref64 = oracle_lib.cst_space(x, src, dst, "f64")
    if 4 not in (src, dst):
        assert np.array_equal(got, ref) or np.abs(got - ref).max() < 1e-6
    else:
        if dst == 4:  # hue is ill-conditioned at zero chroma: compare as Lab
            def lab(v):
                h = np.radians(v[:, 2].astype(np.float64))
                return np.stack([v[:, 0], v[:, 1] * np.cos(h), v[:, 1] * np.sin(h)], axis=1)
            got, ref, ref64 = lab(got), lab(ref), lab(ref64)
        _close(got, ref, ref64=ref64)


@pytest.mark.parametrize("cs", CS)
@pytest.mark.parametrize("coef", [(1.0, 1.0, 1.0), (1.1, 0.6, 0.93)])
def test_lch(oracle_lib, gpu, cs, coef):
    import imops_b200 as im
    x = _space_input(cs, 20 + cs)
    t = _gpu(gpu, x)
    im.lch(t, cs, *coef)
    ref = oracle_lib.lch(x, cs, *coef)
    ref64 = oracle_lib.lch(x, cs, *coef, precision="f64")
    got = t.cpu().numpy()
    if coef[2] != 1.0:
        # hue * hc is discontinuous where the hue wraps (h -> 0 / 360);
        # pixels within 1e-3 degrees of the wrap may differ
        lchv = oracle_lib.cst_space(x, cs, 4)
        ok = (lchv[:, 2] > 1e-3) & (lchv[:, 2] < 360 - 1e-3) & (lchv[:, 1] > 1e-4)
        got, ref, ref64 = got[ok], ref[ok], ref64[ok]
    _close(got, ref, TOL, ref64)


def test_lch_identity_known_answer(gpu):
    # lch.rs:24-36
    import imops_b200 as im
    t = _gpu(gpu, np.array([[0.4, 0.7, 0.2]], np.float32))
    im.lch(t, im.CS_SRGB, 1.0, 1.0, 1.0)
    assert np.abs(t.cpu().numpy() - [0.4, 0.7, 0.2]).max() < 1e-4


def test_lch_rejects_camera_space(gpu):
    import imops_b200 as im
    t = _gpu(gpu, np.zeros((4, 3), np.float32))
    with pytest.raises(im.ImopsError):
        im.lch(t, im.CS_CAMERA, 1.0, 1.0, 1.0)


def test_sigmoid_tone_map(oracle_lib, gpu):
    import imops_b200 as im
    x = _rgb(5, lo=-0.5, hi=8.0)
    t = _gpu(gpu, x)
    im.sigmoid_tone_map(t)
    _close(t.cpu().numpy(), oracle_lib.sigmoid(x), TOL, oracle_lib.sigmoid(x, "f64"))
    g = _gpu(gpu, np.full((1, 3), 0.18, np.float32))
    im.sigmoid_tone_map(g)
    assert np.abs(g.cpu().numpy() - 0.18).max() < 1e-4


def test_sigmoid_against_fp64(oracle_lib, gpu):
    """Error of the f32 kernel against the FP64 oracle, in 16-bit LSB."""
    import imops_b200 as im
    x = _rgb(6, lo=0.0, hi=4.0)
    t = _gpu(gpu, x)
    im.sigmoid_tone_map(t)
    ref = oracle_lib.sigmoid(x.astype(np.float64), "f64")
    err = np.abs(t.cpu().numpy() - ref)
    assert err.max() * 65535 < 1.0


def _meta(**kw):
    from imops_b200.pipeline import make_meta
    return make_meta(wb=[2.0, 0.9, 1.5, 0.0], **kw)


def test_pipeline_display_chain_is_one_pass(oracle_lib, gpu):
    """HighlightReconstruction -> Contrast -> LCH -> SigmoidToneMap -> CST Srgb
    -> Gamma on an ACEScg image: one launch, equal to the stages one by one."""
    import imops_b200 as im
    from imops_b200.pipeline import Image, parse_config, run_pixel_pipeline
    rng = np.random.default_rng(7)
    x = rng.uniform(0.0, 2.0, (64, 1024, 3)).astype(np.float32)
    cfg = parse_config('[[pipeline_modules]]\nname = "HighlightReconstruction"\n'
                       '[[pipeline_modules]]\nname = "Contrast"\nc = 1.2\n'
                       '[[pipeline_modules]]\nname = "LCH"\nlc = 1.05\ncc = 0.8\nhc = 1.0\n'
                       '[[pipeline_modules]]\nname = "SigmoidToneMap"\n'
                       '[[pipeline_modules]]\nname = "CST"\ntarget_color_space = "LinearSrgb"\n'
                       '[[pipeline_modules]]\nname = "Gamma"\ngamma = 2.4\n')
    img = Image.from_rgb(x, im.CS_ACESCG, _meta())
    n0 = im.launch_count()
    run_pixel_pipeline(img, cfg)
    got = img.rgb_f32()
    assert im.launch_count() - n0 == 1
    assert img.metadata()["color_space"] == "LinearSrgb"
    refs = []
    for prec in ("f32", "f64"):
        r = x.reshape(-1, 3)
        r = oracle_lib.highlight(r, [2.0, 0.9, 1.5, 0.0], prec)
        r = oracle_lib.contrast(r, 1.2, prec)
        r = oracle_lib.lch(r, oracle_lib.CS_ACESCG, 1.05, 0.8, 1.0, prec)
        r = oracle_lib.sigmoid(r, prec)
        r = oracle_lib.cst_space(r, oracle_lib.CS_ACESCG, oracle_lib.CS_LINEAR_SRGB, prec)
        refs.append(oracle_lib.gamma(r, 2.4, prec))
    _close(got.reshape(-1, 3), refs[0], TOL, refs[1])


def test_pipeline_cst_through_oklch(oracle_lib, gpu):
    import imops_b200 as im
    from imops_b200.pipeline import Image, parse_config, run_pixel_pipeline
    rng = np.random.default_rng(8)
    x = rng.uniform(0.0, 1.0, (32, 512, 3)).astype(np.float32)
    img = Image.from_rgb(x, im.CS_ACESCG, _meta())
    run_pixel_pipeline(img, parse_config('[[pipeline_modules]]\nname = "CST"\ntarget_color_space = "Oklch"\n'))
    assert img.metadata()["color_space"] == "Oklch"
    run_pixel_pipeline(img, parse_config('[[pipeline_modules]]\nname = "CST"\ntarget_color_space = "AcesCg"\n'))
    back = img.rgb_f32()
    assert np.abs(back - x).max() < 1e-5
    r = oracle_lib.cst_space(oracle_lib.cst_space(x.reshape(-1, 3), 3, 4), 4, 3)
    r64 = oracle_lib.cst_space(oracle_lib.cst_space(x.reshape(-1, 3), 3, 4, "f64"), 4, 3, "f64")
    _close(back.reshape(-1, 3), r, TOL, r64)


def test_pipeline_lch_needs_colour_space(gpu):
    import imops_b200 as im
    from imops_b200.pipeline import Image, get_last_error, parse_config, run_pixel_pipeline
    img = Image.from_rgb(np.zeros((8, 8, 3), np.float32), im.CS_CAMERA, _meta())
    with pytest.raises(im.ImopsError):
        run_pixel_pipeline(img, parse_config('[[pipeline_modules]]\nname = "Exp"\nev = 1\n'
                                             '[[pipeline_modules]]\nname = "LCH"\nlc = 1\ncc = 1\nhc = 1\n'))
    assert "unwrap" in get_last_error()


def test_pipeline_highlight_needs_wb(gpu):
    import imops_b200 as im
    from imops_b200.pipeline import Image, make_meta, parse_config, run_pixel_pipeline
    img = Image.from_rgb(np.zeros((8, 8, 3), np.float32), im.CS_ACESCG, make_meta())
    with pytest.raises(im.ImopsError) as e:
        run_pixel_pipeline(img, parse_config('[[pipeline_modules]]\nname = "HighlightReconstruction"\n'))
    assert "wb_coeffs" in e.value.message
