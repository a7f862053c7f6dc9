"""GPU parity of the demosaic stages against the CPU oracle.

AMaZE and the 3x3 mean are integer-free f32 pipelines restated in the
reference's operation order; the CUDA kernels must match the f32 oracle
bit for bit (including tile borders, the per-tile Nyquist box and the
in-place scan-order updates).
"""
import numpy as np
import pytest

from imops_b200 import synthetic

pytestmark = pytest.mark.gpu

BAYER_SHIFTS = [(0, 0), (1, 0), (0, 1), (1, 1)]  # RGGB, GRBG, GBRG, BGGR


def _amaze_pair(oracle_lib, gpu, mosaic, shift=(0, 0), clip=1.0):
    import torch
    import imops_b200 as im
    ref = oracle_lib.amaze(mosaic, "RGGB", shift=shift, clip_pt=clip, precision="f32")
    out = im.demosaic_amaze(torch.from_numpy(mosaic).to(gpu), "RGGB", shift=shift, clip_pt=clip)
    torch.cuda.synchronize()
    return ref, out.cpu().numpy()


@pytest.mark.parametrize("n", [32, 160])
def test_amaze_flat_field(oracle_lib, gpu, n):
    # demosaic.rs:1410-1443: flat 0.5 stays within 0.2 (it is exact here)
    m = np.full((n, n), 0.5, np.float32)
    ref, out = _amaze_pair(oracle_lib, gpu, m)
    assert out.shape == (n, n, 3)
    assert np.abs(out - 0.5).max() < 0.2
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("shape", [(320, 400), (50, 100), (81, 113), (20, 20), (177, 305)])
@pytest.mark.parametrize("shift", BAYER_SHIFTS)
def test_amaze_bit_exact_random(oracle_lib, gpu, shape, shift):
    rng = np.random.default_rng(shape[0] * 1000 + shape[1] + 17 * shift[0] + 31 * shift[1])
    m = rng.random(shape, dtype=np.float32)
    ref, out = _amaze_pair(oracle_lib, gpu, m, shift)
    diff = np.abs(out - ref)
    assert np.array_equal(out, ref), f"max diff {diff.max()} at {np.unravel_index(diff.argmax(), diff.shape)}"


def test_amaze_bit_exact_scene_highlights(oracle_lib, gpu):
    # a synthetic scene scaled past clip to exercise the clip branches
    m = synthetic.mosaic_f32(256, 320, seed=3) * np.float32(1.3)
    ref, out = _amaze_pair(oracle_lib, gpu, m)
    assert np.array_equal(out, ref)
    ref2, out2 = _amaze_pair(oracle_lib, gpu, m, clip=0.7)
    assert np.array_equal(out2, ref2)


def test_amaze_full_size_c1(oracle_lib, gpu):
    # 1536x1024 RGGB, the CPU-runnable workload
    m = synthetic.mosaic_f32(1024, 1536, seed=1000)
    ref, out = _amaze_pair(oracle_lib, gpu, m)
    assert np.array_equal(out, ref)


def test_amaze_full_size_24mp(oracle_lib, gpu):
    # 6048x4024 RGGB (the 24 MP Bayer workload), bit-exact against the oracle
    m = synthetic.mosaic_f32(4024, 6048, seed=1002)
    ref, out = _amaze_pair(oracle_lib, gpu, m)
    assert np.array_equal(out, ref)


def test_amaze_rejects_reference_panic_sizes(gpu):
    import torch
    import imops_b200 as im
    assert not im.amaze_size_supported(400, 300)  # 300 % 96 == 12
    m = torch.zeros((300, 400), device=gpu)
    with pytest.raises(im.ImopsError) as e:
        im.demosaic_amaze(m)
    assert e.value.code == 3


def test_amaze_rejects_xtrans(gpu):
    import torch
    import imops_b200 as im
    m = torch.zeros((96, 96), device=gpu)
    with pytest.raises(im.ImopsError) as e:
        im.demosaic_amaze(m, synthetic.XTRANS)
    assert e.value.code == 2


@pytest.mark.parametrize("sx", range(6))
@pytest.mark.parametrize("sy", range(6))
def test_markesteijn_xtrans_all_phases(oracle_lib, gpu, sx, sy):
    import torch
    import imops_b200 as im
    rng = np.random.default_rng(sx * 6 + sy)
    m = rng.random((37, 53), dtype=np.float32)
    ref = oracle_lib.mean3x3(m, synthetic.XTRANS, shift=(sx, sy))
    out = im.demosaic_markesteijn(torch.from_numpy(m).to(gpu), synthetic.XTRANS, shift=(sx, sy)).cpu().numpy()
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("shift", BAYER_SHIFTS)
def test_markesteijn_bayer(oracle_lib, gpu, shift):
    import torch
    import imops_b200 as im
    m = synthetic.mosaic_f32(65, 97, seed=5)
    ref = oracle_lib.mean3x3(m, "RGGB", shift=shift)
    out = im.demosaic_markesteijn(torch.from_numpy(m).to(gpu), "RGGB", shift=shift).cpu().numpy()
    assert np.array_equal(out, ref)


def test_markesteijn_full_size_xtrans(oracle_lib, gpu):
    import torch
    import imops_b200 as im
    m = synthetic.mosaic_f32(4032, 6032, seed=1001, pattern=synthetic.XTRANS)
    ref = oracle_lib.mean3x3(m, synthetic.XTRANS)
    out = im.demosaic_markesteijn(torch.from_numpy(m).to(gpu), synthetic.XTRANS).cpu().numpy()
    assert np.array_equal(out, ref)


def test_markesteijn_single_pixel_edges(oracle_lib, gpu):
    import torch
    import imops_b200 as im
    for shape in [(1, 1), (1, 7), (7, 1), (2, 2)]:
        m = np.arange(np.prod(shape), dtype=np.float32).reshape(shape) / 10
        ref = oracle_lib.mean3x3(m, "RGGB")
        out = im.demosaic_markesteijn(torch.from_numpy(m).to(gpu), "RGGB").cpu().numpy()
        assert np.array_equal(out, ref), shape


@pytest.mark.parametrize("sx", range(6))
@pytest.mark.parametrize("sy", range(6))
def test_markesteijn_xtrans_phases_several_warps(oracle_lib, gpu, sx, sy):
    """Rows wider than one warp's 192-pixel span and an odd height: every
    phase alignment of the warps' runs against the image edges."""
    import torch
    import imops_b200 as im
    rng = np.random.default_rng(100 + sx * 6 + sy)
    m = rng.random((29, 401), dtype=np.float32)
    ref = oracle_lib.mean3x3(m, synthetic.XTRANS, shift=(sx, sy))
    out = im.demosaic_markesteijn(torch.from_numpy(m).to(gpu), synthetic.XTRANS, shift=(sx, sy)).cpu().numpy()
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("shift", BAYER_SHIFTS)
def test_markesteijn_bayer_several_warps(oracle_lib, gpu, shift):
    import torch
    import imops_b200 as im
    m = synthetic.mosaic_f32(31, 579, seed=6)
    ref = oracle_lib.mean3x3(m, "RGGB", shift=shift)
    out = im.demosaic_markesteijn(torch.from_numpy(m).to(gpu), "RGGB", shift=shift).cpu().numpy()
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("pattern", ["RBGGRGBGGRGBGBRGGRRGBGGBGRBGGRGBGRGG", "RGBG", "RGEB",
                                     "GGRGGBGGBGGRBRGRBGGGBGGRGGRGGBRBGBEG"])
def test_markesteijn_other_cfas(oracle_lib, gpu, pattern):
    """CFAs that are no shift of RGGB or of the X-Trans period (a scrambled
    6x6, greens on one row, a fourth colour) take the per-pixel kernel."""
    import torch
    import imops_b200 as im
    rng = np.random.default_rng(len(pattern))
    m = rng.random((27, 230), dtype=np.float32)
    ref = oracle_lib.mean3x3(m, pattern)
    out = im.demosaic_markesteijn(torch.from_numpy(m).to(gpu), pattern).cpu().numpy()
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("pattern", [synthetic.XTRANS, "RGGB"])
def test_markesteijn_non_finite_samples(oracle_lib, gpu, pattern):
    """NaN and infinite samples reach only the sums of their own colour, as in
    the reference's per-colour loops."""
    import torch
    import imops_b200 as im
    rng = np.random.default_rng(3)
    m = rng.random((40, 300), dtype=np.float32)
    idx = rng.choice(m.size, 60, replace=False)
    m.flat[idx[:20]] = np.nan
    m.flat[idx[20:40]] = np.inf
    m.flat[idx[40:]] = -np.inf
    ref = oracle_lib.mean3x3(m, pattern)
    out = im.demosaic_markesteijn(torch.from_numpy(m).to(gpu), pattern).cpu().numpy()
    np.testing.assert_array_equal(out, ref)


@pytest.mark.parametrize("factor", [2, 4, 8])
def test_quad_previews(oracle_lib, gpu, factor):
    import torch
    import imops_b200 as im
    m = synthetic.mosaic_f32(64, 96, seed=9)
    for shift in BAYER_SHIFTS:
        ref = oracle_lib.quad(m, "RGGB", factor, shift=shift)
        out = im.demosaic_quad(torch.from_numpy(m).to(gpu), "RGGB", factor, shift=shift).cpu().numpy()
        assert np.array_equal(out, ref)
    # demosaic.rs:1388-1408: flat 0.5 stays 0.5
    flat = torch.full((16, 16), 0.5, device=gpu)
    assert torch.all((im.demosaic_quad(flat, "RGGB", 2) - 0.5).abs() < 1e-4)


def test_amaze_largest_frame_45mp(oracle_lib, gpu):
    """8256x5504 (45 MP, the largest frame of the uneven-size batch): the
    oracle on tile-aligned corner crops.  A tile's output depends only on its
    own window, so a crop whose origin is a multiple of 96 holds the same
    tiles; their cores match where the window lies inside the crop or at an
    edge the crop shares with the frame."""
    import torch
    import imops_b200 as im
    H, W = 5504, 8256
    m = synthetic.mosaic_f32(H, W, seed=45)
    out = im.demosaic_amaze(torch.from_numpy(m).to(gpu)).cpu().numpy()
    assert np.isfinite(out).all()
    tl = oracle_lib.amaze(m[:384, :384])
    assert np.array_equal(out[:288, :288], tl[:288, :288])
    y, x = 96 * 53, 96 * 82
    br = oracle_lib.amaze(m[y:, x:], shift=(x, y))
    assert np.array_equal(out[y + 96:, x + 96:], br[96:, 96:])
