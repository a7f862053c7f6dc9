"""Seeded synthetic raw mosaics with the shapes and noise of the benchmark
workloads (no real raw file is available to the reference or to us).

Scene: smooth per-channel colour gradients plus random-orientation sinusoidal
edges (periods 2-40 px), values in [0, 0.9].  Mosaic: 14-bit sensor with
black 600 / white 16383; signal DN = scene * (white - black) at the site's
CFA colour, shot noise Poisson(0.5 e-/DN * DN) / 0.5, read noise N(0, 3 DN),
rounded and clamped to [0, 16383].
"""
from __future__ import annotations

import numpy as np

BLACK = 600.0
WHITE = 16383.0
XTRANS = "GGRGGBGGBGGRBRGRBGGGBGGRGGRGGBRBGBRG"


def cfa_colors(pattern: str, H: int, W: int) -> np.ndarray:
    sizes = {4: (2, 2), 36: (6, 6), 16: (2, 8), 144: (12, 12)}
    pw, ph = sizes[len(pattern)]
    lut = {"R": 0, "G": 1, "B": 2}
    per = np.array([lut[c] for c in pattern], dtype=np.int8).reshape(ph, pw)
    return np.tile(per, (H // ph + 1, W // pw + 1))[:H, :W]


def scene(H: int, W: int, seed: int, n_waves: int = 6) -> np.ndarray:
    rng = np.random.default_rng(seed)
    y = np.linspace(0.0, 1.0, H, dtype=np.float32)[:, None]
    x = np.linspace(0.0, 1.0, W, dtype=np.float32)[None, :]
    out = np.empty((H, W, 3), dtype=np.float32)
    yy = np.arange(H, dtype=np.float32)[:, None]
    xx = np.arange(W, dtype=np.float32)[None, :]
    waves = np.zeros((H, W), dtype=np.float32)
    for _ in range(n_waves):
        period = rng.uniform(2.0, 40.0)
        th = rng.uniform(0, np.pi)
        ph = rng.uniform(0, 2 * np.pi)
        amp = rng.uniform(0.03, 0.12)
        waves += (amp * np.sin(2 * np.pi * (xx * np.cos(th) + yy * np.sin(th)) / period + ph)).astype(np.float32)
    for c in range(3):
        a, bx, by = rng.uniform(0.15, 0.45), rng.uniform(-0.3, 0.4), rng.uniform(-0.3, 0.4)
        out[..., c] = a + bx * x + by * y + waves * rng.uniform(0.6, 1.0)
    return np.clip(out, 0.0, 0.9)


def mosaic_u16(H: int, W: int, seed: int, pattern: str = "RGGB") -> np.ndarray:
    sc = scene(H, W, seed)
    col = cfa_colors(pattern, H, W)
    sig = np.take_along_axis(sc, col[..., None].astype(np.int64), axis=2)[..., 0] * (WHITE - BLACK)
    rng = np.random.default_rng(seed + 7919)
    e = rng.poisson(np.maximum(sig, 0.0) * 0.5) / 0.5
    v = e + rng.normal(0.0, 3.0, size=sig.shape) + BLACK
    return np.clip(np.rint(v), 0, WHITE).astype(np.uint16)


def normalize(raw: np.ndarray) -> np.ndarray:
    """(v - black) / (white - black) in f32, the library's scaling formula."""
    return ((raw.astype(np.float32) - np.float32(BLACK)) / (np.float32(WHITE) - np.float32(BLACK))).astype(np.float32)


def mosaic_f32(H: int, W: int, seed: int, pattern: str = "RGGB") -> np.ndarray:
    return normalize(mosaic_u16(H, W, seed, pattern))


# A fixed camera calibration (XYZ->camera, D65) used by the workloads; any
# well-conditioned matrix works, this one resembles a typical Bayer sensor.
CALIB_D65 = (0.6722, -0.0635, -0.0963,
             -0.4287, 1.2460, 0.2028,
             -0.0908, 0.2162, 0.5668)
WB = (2.0, 1.0, 1.5, 0.0)

# XYZ (D65) -> ACES AP1, the matrix the film model uses for ACEScg.
XYZ2AP1 = np.array([[1.6410233797, -0.3248032942, -0.2364246952], [-0.6636628587, 1.6153315917, 0.0167563477],
                    [0.0117218943, -0.0082844165, 0.9883948585]])


def film_grad_base() -> np.ndarray:
    """The 24 parameters of the differentiable colour + film model at the
    workload's settings: WB, camera->ACEScg matrix (rows of the D65
    calibration scaled to map D65 white to 1, inverted, then XYZ->AP1),
    EV 0 and the baseline preset's curves and halation."""
    M = np.array(CALIB_D65, np.float64).reshape(3, 3)
    d65 = M @ np.array([0.95042, 1.0, 1.08890])
    C = XYZ2AP1 @ np.linalg.inv(M / d65[:, None])
    return np.array([*WB[:3], *C.reshape(9), 0.0, 2.0, 2.1, 2.2, 2.3, 2.5, 2.7, -0.70, -0.73, -0.76, 0.15, 20.0])


def film_grad_perturbed(seed: int = 0) -> np.ndarray:
    """film_grad_base() perturbed as the fitting workload does: +-5% WB,
    +-0.02 matrix, +-0.1 EV, +-5% curve parameters, +-10% halation."""
    rng = np.random.default_rng(seed)
    v = film_grad_base()
    v[0:3] *= 1 + rng.uniform(-0.05, 0.05, 3)
    v[3:12] += rng.uniform(-0.02, 0.02, 9)
    v[12] += rng.uniform(-0.1, 0.1)
    v[13:22] *= 1 + rng.uniform(-0.05, 0.05, 9)
    v[22:24] *= 1 + rng.uniform(-0.1, 0.1, 2)
    return v
