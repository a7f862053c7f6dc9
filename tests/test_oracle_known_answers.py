"""The CPU oracle against the reference's own known-answer and property
tests (the reference cannot be built here, so these pin the restatement).
Each test names the reference test it ports."""
import math

import numpy as np
import pytest


def test_cfa_color_at_and_shift(oracle_lib):
    # cfa.rs:54-62, 189-203, 343-360
    c = oracle_lib.parse_cfa("RGGB")
    assert [c.col[i] for i in range(4)] == [0, 1, 1, 2]
    s = oracle_lib.parse_cfa("RGGB", 1, 1)
    assert [s.col[i] for i in range(4)] == [2, 1, 1, 0]  # BGGR
    with pytest.raises(ValueError):
        oracle_lib.parse_cfa("RGB")


@pytest.mark.parametrize("n", [32, 160])
def test_amaze_flat_field(oracle_lib, n):
    # demosaic.rs:1410-1443
    out = oracle_lib.amaze(np.full((n, n), 0.5, np.float32), "RGGB")
    assert out.shape == (n, n, 3)
    assert np.abs(out - 0.5).max() < 0.2


def test_fast_flat_field(oracle_lib):
    # demosaic.rs:1388-1408
    out = oracle_lib.quad(np.full((16, 16), 0.5, np.float32), "RGGB", 2)
    assert out.shape == (8, 8, 3)
    assert np.abs(out - 0.5).max() < 1e-4


def test_blur_identity_mass_symmetry(oracle_lib):
    # blur.rs:95-143
    buf = np.arange(64, dtype=np.float32).reshape(8, 8)
    assert np.array_equal(oracle_lib.blur(buf, 0.0), buf)
    ones = np.ones((64, 64), np.float32)
    out = oracle_lib.blur(ones, 2.0)
    assert abs(out.astype(np.float64).sum() / ones.sum() - 1) < 1e-3
    imp = np.zeros((65, 65), np.float32)
    imp[32, 32] = 1
    b = oracle_lib.blur(imp, 3.0)
    for dx, dy in [(5, 0), (0, 5), (4, 3), (3, 4), (-5, 0), (0, -5)]:
        a = b[32 + dy, 32 + dx]
        assert abs(a - b[32 - dy, 32 - dx]) < 1e-5
        assert abs(a - b[32 + dx, 32 + dy]) < 1e-5


def test_capture_lut_properties(oracle_lib):
    # capture.rs:113-186 with the reference tests' distribution: ln s ~ N(ln 0.7, 0.35^2), k = 1
    mu, sg, k = math.log(0.7), 0.35, 1.0
    def lut(phi):
        return oracle_lib.lut_build_sample(mu, sg, k, phi)
    prev = -1.0
    for i in range(64):
        f = lut(10 ** (-4 + i * (12 / 63)))
        assert f + 1e-12 >= prev
        prev = f
    assert lut(1e-6) < 0.05
    assert lut(1e10) > 0.99
    n = 40
    fs = [lut(10 ** (-3 + i * (10 / (n - 1)))) for i in range(n)]
    slopes = [fs[i] - fs[i - 1] for i in range(1, n)]
    mi = 1 + int(np.argmax(slopes))
    ti = max(mi // 3, 2)
    si = max(min((mi + n) // 2, n - 1), mi + 2)
    assert (fs[ti] - fs[ti - 1]) - (fs[ti - 1] - fs[ti - 2]) > 0
    assert (fs[si] - fs[si - 1]) - (fs[si - 1] - fs[si - 2]) < 0
    assert lut(3.0) == lut(3.0)  # deterministic


def test_stock_lut_monotone(oracle_lib):
    # the same LUT machinery on ColorNeg200's three emulsions
    for layer in range(3):
        fs = [oracle_lib.lut_sample(1, layer, 10 ** (-4 + i * 12 / 63)) for i in range(64)]
        assert all(b + 1e-12 >= a for a, b in zip(fs, fs[1:]))


def test_upsample_roundtrip_gray_and_red(oracle_lib):
    # upsample.rs:187-224
    spec, back = oracle_lib.upsample_roundtrip([0.185, 0.185, 0.185])
    assert (spec >= 0).all()
    assert np.abs(back - 0.185).max() < 0.02
    spec, _ = oracle_lib.upsample_roundtrip([0.8, 0.05, 0.02])
    assert spec[12:16].sum() > spec[0:4].sum()


def test_invert_dmin_black_mid_gray(oracle_lib):
    # invert.rs:131-148
    dmin = [1.0, 0.45, 0.13]
    mid = [0.23, 0.15, 0.10]
    out = oracle_lib.invert(np.array([dmin, mid], np.float32), mid, dmin)
    assert np.abs(out[0]).max() < 1e-5
    assert np.abs(out[1] - 0.185).max() < 1e-3


def test_invert_pathological_blue_bounded(oracle_lib):
    # invert.rs:150-175
    dmin, mid = [1.0, 0.45, 0.127], [0.65, 0.315, 0.122]
    p = oracle_lib.invert(np.array([[0.16, 0.087, 0.058]], np.float32), mid, dmin)[0]
    y = 0.2722287168 * p[0] + 0.6740817658 * p[1] + 0.0536895174 * p[2]
    assert math.isfinite(y) and y > 0
    assert (p < 2.5).all()
    assert p.max() / max(p.min(), 1e-6) < 4.0


def test_baseline_exposure_ratios(oracle_lib):
    # radiance.rs:76-128: L = K v N^2 / (t S); doubling t halves L, N x2 -> x4, ISO x2 -> /2
    x = np.full((1, 3), 0.185, np.float32)
    def L(t, n, s):
        return float(oracle_lib.baseline_exposure(x, 0.0, t, n, s, precision="f64")[0][0, 0])
    l1 = L(1 / 200, 8.0, 200.0)
    assert abs(l1 - 12.5 * 0.185 * 64) < 1e-5 * l1
    assert abs(L(2 / 200, 8.0, 200.0) / l1 - 0.5) < 1e-10
    assert abs(L(1 / 200, 16.0, 200.0) / l1 - 4.0) < 1e-10
    assert abs(L(1 / 200, 8.0, 400.0) / l1 - 0.5) < 1e-10
    _, applied = oracle_lib.baseline_exposure(x, 0.0, 0.0, 8.0, 200.0)
    assert not applied


def test_film_bwstub_hd_monotone_and_dmin(oracle_lib):
    # film/mod.rs:234-273 (BwStub, box ISO 100)
    g = 12.5 * 64.0
    ys = []
    for y in [0.02, 0.05, 0.1, 0.185, 0.3, 0.5, 0.8, 1.2]:
        img = np.full((8, 8, 3), y * g, np.float32)
        out = oracle_lib.film_process(img, stock=0, seed=1)
        ys.append(float((0.2722287168 * out[..., 0] + 0.6740817658 * out[..., 1] +
                         0.0536895174 * out[..., 2]).mean()))
    assert all(b <= a + 1e-4 for a, b in zip(ys, ys[1:]))
    z = oracle_lib.film_process(np.zeros((8, 8, 3), np.float32), stock=0, seed=1)
    assert abs(z.max(axis=2).mean() - 1.0) < 0.05
    mg = oracle_lib.film_process(np.full((8, 8, 3), 0.185 * g, np.float32), stock=0, seed=1)
    assert np.isfinite(mg).all() and (mg > 0).all() and (mg < 1.5).all()


def test_film_determinism_and_dmin_norm(oracle_lib):
    # film/mod.rs:325-334 and 516-535
    img = np.tile(np.array([0.185, 0.1, 0.05], np.float32) * 1600, (8, 8, 1))
    a = oracle_lib.film_process(img, stock=1, seed=1)
    b = oracle_lib.film_process(img, stock=1, seed=1)
    assert np.array_equal(a, b)
    d = oracle_lib.normalized_dmin(1)
    assert abs(d.max() - 1.0) < 1e-5
    assert d[0] > d[1] > d[2]


def test_film_neutral_positive_near_neutral(oracle_lib):
    # film/mod.rs:285-300: mid gray through ColorNeg200 PositiveLinear has |a|,|b| < 5
    g = 0.185 * 12.5 * 64.0
    out = oracle_lib.film_process(np.full((16, 16, 3), g, np.float32), stock=1, seed=1, output=1)
    m = out.reshape(-1, 3).astype(np.float64).mean(0)
    M = np.array([[0.6624541811, 0.1340042065, 0.1561876870], [0.2722287168, 0.6740817658, 0.0536895174],
                  [-0.0055746495, 0.0040607335, 1.0103391003]])
    xyz = M @ m
    def f(t):
        return np.cbrt(t) if t > (6 / 29) ** 3 else t / (3 * (6 / 29) ** 2) + 4 / 29
    fx, fy, fz = f(xyz[0] / 0.95047), f(xyz[1] / 1.0), f(xyz[2] / 1.08883)
    a, b = 500 * (fx - fy), 200 * (fy - fz)
    assert abs(a) < 5 and abs(b) < 5


def test_grain_noise_counter_based(oracle_lib):
    # grain.rs:20-45: the noise of row y does not depend on other rows
    full = oracle_lib.grain_noise(17, 9, seed=123, layer=1)
    assert full.shape == (9, 17)
    assert abs(full.mean()) < 0.5
    again = oracle_lib.grain_noise(17, 9, seed=123, layer=1)
    assert np.array_equal(full, again)
    other = oracle_lib.grain_noise(17, 9, seed=124, layer=1)
    assert not np.array_equal(full, other)


def test_baseline_preset_oracle_sane(oracle_lib):
    # the library's own 81-bin preset: D=0 (zero exposure) scans to peak 1,
    # more exposure gives a denser (darker) negative
    p = oracle_lib.baseline_params(grain_on=0)
    out0 = oracle_lib.film_baseline(np.zeros((4, 4, 3), np.float32), p)
    assert out0.max() <= 1.0 + 1e-9
    lo = oracle_lib.film_baseline(np.full((4, 4, 3), 0.05, np.float32), p)
    hi = oracle_lib.film_baseline(np.full((4, 4, 3), 0.5, np.float32), p)
    assert (hi < lo).all()
    x, y, z = oracle_lib.cmf81()
    assert abs(y.max() - 1.0) < 0.02 and 550 <= 380 + 5 * int(np.argmax(y)) <= 560


# emulsion layers per StockId (film/stock/*: BwStub, ColorNeg200, Portra400,
# Ektar100, FujiPro400H, EktachromeE100, TriX400)
STOCK_EMULSIONS = {0: 1, 1: 3, 2: 6, 3: 6, 4: 7, 5: 3, 6: 2}


def test_all_stocks_load_and_validate(oracle_lib):
    # film/mod.rs:221-233: every stock loads; its emulsions have a finite
    # grain kappa and a monotone capture LUT (capture.rs:113-130), and the
    # normalised Dmin peaks at 1 (film/mod.rs:526-535)
    for sid, ne in STOCK_EMULSIONS.items():
        ks = [oracle_lib.layer_kappa(sid, e) for e in range(ne)]
        assert all(np.isfinite(k) and k > 0 for k in ks), (sid, ks)
        assert np.isnan(oracle_lib.layer_kappa(sid, ne))
        for e in range(ne):
            fs = [oracle_lib.lut_sample(sid, e, 10.0 ** lp) for lp in np.linspace(-4, 8, 25)]
            assert all(b >= a - 1e-12 for a, b in zip(fs, fs[1:])), (sid, e)
        d = oracle_lib.normalized_dmin(sid)
        assert np.isfinite(d).all() and abs(d.max() - 1.0) < 1e-5, (sid, d)


def test_colour_negatives_have_orange_dmin(oracle_lib):
    # the orange mask of the masked negatives: R > G > B on the film base
    for sid in (1, 2, 3, 4):
        d = oracle_lib.normalized_dmin(sid)
        assert d[0] > d[1] > d[2], (sid, d)


def test_reversal_ektachrome_positive_slide(oracle_lib):
    # film/mod.rs:509-521: the reversal stock on mid grey gives a finite
    # positive (the output mode is ignored for reversal stocks)
    g = 0.185 * 12.5 * 64.0
    a = oracle_lib.film_process(np.full((16, 16, 3), g, np.float32), stock=5, seed=1, output=1)
    b = oracle_lib.film_process(np.full((16, 16, 3), g, np.float32), stock=5, seed=1, output=0)
    assert np.isfinite(a.reshape(-1, 3).mean(0)).all()
    assert np.array_equal(a, b)


# ---- display stages -----------------------------------------------------------

def test_highlight_reconstruction_known_answer(oracle_lib):
    # highlight_reconstruction.rs:19-31
    out = oracle_lib.highlight(np.array([[0.6, 0.4, 0.8]], np.float32), [1.0, 1.0, 1.0, 1.0])
    assert abs(out[0, 0] - 0.6) < 1e-6 and abs(out[0, 1] - 0.52) < 1e-6 and abs(out[0, 2] - 0.8) < 1e-6


def test_square_sigmoid_gray_preservation(oracle_lib):
    # tone_map.rs:176-186
    assert abs(oracle_lib.square_sigmoid(0.18) - 0.18) < 1e-5


def test_gamma_22_roundtrip_mid(oracle_lib):
    # tone_map.rs:188-195
    e = oracle_lib.gamma(np.full((1, 3), 0.18, np.float32), 2.2)[0, 0]
    assert abs(np.float32(e) ** np.float32(2.2) - 0.18) < 1e-5


def test_lch_roundtrip_identity(oracle_lib):
    # lch.rs:24-36
    out = oracle_lib.lch(np.array([[0.4, 0.7, 0.2]], np.float32), oracle_lib.CS_SRGB, 1.0, 1.0, 1.0)
    assert np.abs(out - [0.4, 0.7, 0.2]).max() < 1e-4


def test_oklab_published_values(oracle_lib):
    # Ottosson (2020), "A perceptual color space for image processing": XYZ
    # (D65) -> Oklab table, three decimals
    xyz = np.array([[0.950, 1.000, 1.089], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float64)
    lab = np.array([[1.000, 0.000, 0.000], [0.450, 1.236, -0.019], [0.922, -0.671, 0.263],
                    [0.153, -1.415, -0.449]])
    lch = oracle_lib.cst_space(xyz, oracle_lib.CS_XYZD65, oracle_lib.CS_OKLCH, precision="f64")
    h = np.radians(lch[:, 2])
    got = np.stack([lch[:, 0], lch[:, 1] * np.cos(h), lch[:, 1] * np.sin(h)], axis=1)
    assert np.abs(got - lab).max() < 1.5e-3
    assert ((lch[:, 2] >= 0) & (lch[:, 2] < 360)).all()


def test_oklch_roundtrips(oracle_lib):
    rng = np.random.default_rng(3)
    x = rng.uniform(-0.2, 2.0, (2000, 3))
    for cs in (oracle_lib.CS_ACESCG, oracle_lib.CS_SRGB, oracle_lib.CS_LINEAR_SRGB, oracle_lib.CS_XYZD65):
        back = oracle_lib.cst_space(oracle_lib.cst_space(x, cs, oracle_lib.CS_OKLCH, "f64"),
                                    oracle_lib.CS_OKLCH, cs, "f64")
        # the Oklab matrices are the published 10-digit values, rounded to f32
        assert np.abs(back - x).max() < 1e-4, cs


def test_sigmoid_keeps_mid_gray_and_zero(oracle_lib):
    # tone_map.rs:6-33: grays are not gamut-compressed and at mid grey the
    # chroma factor 1 - Y^5 is ~1, so 18% grey maps to 18% grey (the square
    # sigmoid's fixed point, tone_map.rs:176-186); black stays black
    out = oracle_lib.sigmoid(np.array([[0.18, 0.18, 0.18], [0.0, 0.0, 0.0]], np.float32), "f64")
    assert np.abs(out[0] - 0.18).max() < 1e-5
    assert np.abs(out[1]).max() < 1e-12


# ---- 3-pass directional X-Trans demosaic (the library's own method) -----------

def _xtrans_scene(H, W, seed):
    from imops_b200 import synthetic
    sc = synthetic.scene(H, W, seed=seed)
    cols = synthetic.cfa_colors(synthetic.XTRANS, H, W)
    m = np.take_along_axis(sc, cols[..., None].astype(np.int64), axis=2)[..., 0].astype(np.float32)
    return sc, cols, m


def test_markesteijn3_properties(oracle_lib):
    from imops_b200 import synthetic
    sc, cols, m = _xtrans_scene(180, 210, 4)
    out = oracle_lib.markesteijn3(m, synthetic.XTRANS)
    own = np.take_along_axis(out, cols[..., None].astype(np.int64), axis=2)[..., 0]
    assert np.array_equal(own, m)  # CFA samples kept
    flat = oracle_lib.markesteijn3(np.full((60, 66), 0.3, np.float32), synthetic.XTRANS)
    assert np.abs(flat[10:-10, 10:-10] - 0.3).max() == 0.0
    mean = oracle_lib.mean3x3(m, synthetic.XTRANS)
    band = np.ones(m.shape, bool)
    band[10:-10, 10:-10] = False
    assert np.array_equal(out[band], mean[band])  # edge band = the reference's 3x3 mean
    psnr = lambda x: 10 * np.log10(1.0 / np.mean((x[12:-12, 12:-12] - sc[12:-12, 12:-12]) ** 2))
    assert psnr(out) > psnr(mean) + 5.0
    # f32 specification close to its FP64 instantiation
    f64 = oracle_lib.markesteijn3(m, synthetic.XTRANS, precision="f64")
    assert np.abs(out - f64)[10:-10, 10:-10].mean() < 1e-5


def test_xtrans_cube_root_over_every_binade(oracle_lib):
    """The Lab step's division-free cube root (the kernel uses the same f32
    steps): from the first guess 0x54AAAAAA - bits(t)/3, which is 0..8.17%
    high for every normal t, four Newton steps reach the exact cube root to
    5e-7 relative, from 2^-126 to 2^127 (the Lab step uses t > 216/24389)."""
    t = np.logspace(-37.9, 38.2, 400_001).astype(np.float32)
    t = t[np.isfinite(t) & (t >= np.finfo(np.float32).tiny)]
    guess = (np.uint32(0x54AAAAAA) - t.view(np.uint32) // np.uint32(3)).view(np.float32).astype(np.float64)
    e = guess * np.cbrt(t.astype(np.float64)) - 1.0  # guess / t^(-1/3) - 1
    assert e.min() >= -1e-7 and e.max() < 0.0817
    got = oracle_lib.xt_cbrt(t).astype(np.float64)
    rel = np.abs(got / np.cbrt(t.astype(np.float64)) - 1.0)
    assert rel.max() < 5e-7
    f64 = oracle_lib.xt_cbrt(t.astype(np.float64), precision="f64")
    assert np.abs(f64 / np.cbrt(t.astype(np.float64)) - 1.0).max() < 1e-15
