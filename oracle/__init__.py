"""CPU oracle of the raw-development path (TEST INFRASTRUCTURE).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
legs import this package; the CUDA library never calls it.  It wraps
``oracle/liboracle.so`` (built by ``oracle/Makefile`` from the C restatements
in this directory) with numpy-friendly functions.

Every function takes ``precision="f32"`` (the reference's f32 operation order:
the parity target) or ``"f64"`` (the same steps in double: the FP64 oracle for
error reporting).

Parity status: the reference (Rust) cannot be built or run here, so the
restatements are pinned by the reference's own known-answer tests (ported in
``tests/test_oracle_known_answers.py``); the black/white scaling formula
(rawler) and the colour-space conversions (``color`` crate: XYZ->target, and
Oklab / Oklch, the latter checked against Ottosson's published XYZ->Oklab
table) are restated from their published definitions and are "parity
unpinned".  ``markesteijn3`` (``xtrans.c``) is the specification of the
library's own X-Trans method, which has no counterpart in the reference.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

CS_XYZD65, CS_LINEAR_SRGB, CS_SRGB, CS_ACESCG, CS_OKLCH = 0, 1, 2, 3, 4
STOCK_BWSTUB, STOCK_COLORNEG200 = 0, 1
ERR_NAMES = {0: "ok", 1: "invalid argument", 2: "unsupported CFA", 3: "unsupported size"}


class OracleCfa(ctypes.Structure):
    _fields_ = [("pw", ctypes.c_int), ("ph", ctypes.c_int), ("col", ctypes.c_uint8 * 144)]


class OracleBaseline(ctypes.Structure):
    """Parameters of the baseline (81-bin) film preset; mirrors OBaseline."""

    _fields_ = [
        ("dmax", ctypes.c_float * 3),
        ("k", ctypes.c_float * 3),
        ("x0", ctypes.c_float * 3),
        ("hal_strength", ctypes.c_float),
        ("hal_sigma", ctypes.c_float),
        ("hal_radius", ctypes.c_int),
        ("hal_threshold", ctypes.c_float),
        ("grain_sigma", ctypes.c_float),
        ("grain_blur", ctypes.c_float),
        ("grain_on", ctypes.c_int),
        ("seed", ctypes.c_uint64),
    ]


def build() -> str:
    """Compile liboracle.so (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
    return _lib


def _f(name: str, precision: str):
    if precision not in ("f32", "f64"):
        raise ValueError("precision must be 'f32' or 'f64'")
    return getattr(lib(), f"{name}_{precision}")


def _dt(precision: str):
    return np.float32 if precision == "f32" else np.float64


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def parse_cfa(pattern: str, shift_x: int = 0, shift_y: int = 0) -> OracleCfa:
    """CFA::new + CFA::shift (pichromatic/src/cfa.rs:98-129, 204-233)."""
    sizes = {4: (2, 2), 36: (6, 6), 16: (2, 8), 144: (12, 12)}
    if len(pattern) not in sizes:
        raise ValueError(f"Unknown CFA size \"{pattern}\"")
    pw, ph = sizes[len(pattern)]
    lut = {"R": 0, "G": 1, "B": 2, "E": 3, "C": 3, "M": 4, "Y": 5}
    base = [lut[ch] for ch in pattern]
    c = OracleCfa()
    c.pw, c.ph = pw, ph
    for r in range(ph):
        for q in range(pw):
            c.col[r * pw + q] = base[((r + shift_y) % ph) * pw + (q + shift_x) % pw]
    return c


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"oracle {what}: {ERR_NAMES.get(rc, rc)}")


def amaze(mosaic: np.ndarray, cfa: str = "RGGB", shift=(0, 0), clip_pt: float = 1.0,
          precision: str = "f32", threads: int = 0) -> np.ndarray:
    dt = _dt(precision)
    m = np.ascontiguousarray(mosaic, dtype=dt)
    H, W = m.shape
    out = np.zeros((H, W, 3), dtype=dt)
    c = parse_cfa(cfa, *shift)
    fn = _f("oracle_amaze", precision)
    real = ctypes.c_float if precision == "f32" else ctypes.c_double
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OracleCfa), real,
                   ctypes.c_void_p, ctypes.c_int]
    _check(fn(_ptr(m), W, H, ctypes.byref(c), clip_pt, _ptr(out), threads or os.cpu_count()), "amaze")
    return out


def amaze_size_ok(W: int, H: int) -> bool:
    fn = lib().oracle_amaze_size_ok_f32
    fn.argtypes = [ctypes.c_int, ctypes.c_int]
    return bool(fn(W, H))


def mean3x3(mosaic: np.ndarray, cfa: str, shift=(0, 0), precision: str = "f32", threads: int = 0):
    dt = _dt(precision)
    m = np.ascontiguousarray(mosaic, dtype=dt)
    H, W = m.shape
    out = np.zeros((H, W, 3), dtype=dt)
    c = parse_cfa(cfa, *shift)
    fn = _f("oracle_mean3x3", precision)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OracleCfa), ctypes.c_void_p,
                   ctypes.c_int]
    _check(fn(_ptr(m), W, H, ctypes.byref(c), _ptr(out), threads or os.cpu_count()), "mean3x3")
    return out


def markesteijn3(mosaic: np.ndarray, cfa: str, shift=(0, 0), precision: str = "f32"):
    """The library's 3-pass directional X-Trans demosaic (oracle/xtrans.c)."""
    dt = _dt(precision)
    m = np.ascontiguousarray(mosaic, dtype=dt)
    H, W = m.shape
    out = np.zeros((H, W, 3), dtype=dt)
    c = parse_cfa(cfa, *shift)
    fn = _f("oracle_markesteijn3", precision)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OracleCfa), ctypes.c_void_p]
    _check(fn(_ptr(m), W, H, ctypes.byref(c), _ptr(out)), "markesteijn3")
    return out


def xt_cbrt(t: np.ndarray, precision: str = "f32") -> np.ndarray:
    """The division-free cube root of the 3-pass X-Trans Lab step
    (oracle/xtrans.c ``xt_cbrt``, the same arithmetic as the kernel's)."""
    dt = _dt(precision)
    a = np.ascontiguousarray(t, dtype=dt)
    out = np.empty_like(a)
    fn = _f("oracle_xt_cbrt", precision)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p]
    fn.restype = None
    fn(_ptr(a), a.size, _ptr(out))
    return out


def quad(mosaic: np.ndarray, cfa: str, factor: int, shift=(0, 0), precision: str = "f32"):
    dt = _dt(precision)
    m = np.ascontiguousarray(mosaic, dtype=dt)
    H, W = m.shape
    out = np.zeros((H // factor, W // factor, 3), dtype=dt)
    c = parse_cfa(cfa, *shift)
    fn = _f("oracle_quad", precision)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OracleCfa), ctypes.c_int,
                   ctypes.c_void_p]
    _check(fn(_ptr(m), W, H, ctypes.byref(c), factor, _ptr(out)), "quad")
    return out


def scale_u16(raw: np.ndarray, crop, black, white, cfa_period=(2, 2), precision: str = "f32"):
    """crop = (x, y, w, h); black/white: per CFA cell (ph*pw values)."""
    dt = _dt(precision)
    r = np.ascontiguousarray(raw, dtype=np.uint16)
    rh, rw = r.shape
    x, y, w, h = crop
    pw, ph = cfa_period
    b = np.ascontiguousarray(np.broadcast_to(np.asarray(black, dtype=dt), (ph * pw,)))
    wt = np.ascontiguousarray(np.broadcast_to(np.asarray(white, dtype=dt), (ph * pw,)))
    out = np.zeros((h, w), dtype=dt)
    fn = _f("oracle_scale_u16", precision)
    fn.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 6 + [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                            ctypes.c_int, ctypes.c_void_p]
    _check(fn(_ptr(r), rw, rh, x, y, w, h, _ptr(b), _ptr(wt), pw, ph, _ptr(out)), "scale")
    return out


def wb(rgb: np.ndarray, coeffs, precision: str = "f32"):
    dt = _dt(precision)
    out = np.ascontiguousarray(rgb, dtype=dt).copy()
    c = np.asarray(list(coeffs) + [0.0] * (4 - len(coeffs)), dtype=dt)
    fn = _f("oracle_wb", precision)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    fn(_ptr(out), out.size // 3, _ptr(c))
    return out


def exposure(rgb: np.ndarray, ev: float, precision: str = "f32"):
    dt = _dt(precision)
    out = np.ascontiguousarray(rgb, dtype=dt).copy()
    fn = _f("oracle_exp", precision)
    real = ctypes.c_float if precision == "f32" else ctypes.c_double
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, real]
    fn(_ptr(out), out.size // 3, ev)
    return out


def baseline_exposure(rgb, baseline_ev, shutter, f_number, iso, precision: str = "f32"):
    dt = _dt(precision)
    out = np.ascontiguousarray(rgb, dtype=dt).copy()
    fn = _f("oracle_baseline_exposure", precision)
    real = ctypes.c_float if precision == "f32" else ctypes.c_double
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, real, real, real, real]
    applied = fn(_ptr(out), out.size // 3, baseline_ev, shutter, f_number, iso)
    return out, bool(applied)


def camera_forward_matrix(calib, precision: str = "f32"):
    dt = _dt(precision)
    c = np.ascontiguousarray(calib, dtype=dt).reshape(9)
    out = np.zeros(9, dtype=dt)
    fn = _f("oracle_camera_forward_matrix", precision)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    fn(_ptr(c), _ptr(out))
    return out.reshape(3, 3)


def camera_cst(rgb: np.ndarray, calib, target: int, precision: str = "f32"):
    dt = _dt(precision)
    out = np.ascontiguousarray(rgb, dtype=dt).copy()
    c = np.ascontiguousarray(calib, dtype=dt).reshape(9)
    fn = _f("oracle_camera_cst", precision)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_int]
    _check(fn(_ptr(out), out.size // 3, _ptr(c), target), "camera_cst")
    return out


def _rgb_op(name, rgb, precision, argtypes, *args, check=False):
    dt = _dt(precision)
    out = np.ascontiguousarray(rgb, dtype=dt).copy()
    fn = _f(name, precision)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t] + argtypes
    rc = fn(_ptr(out), out.size // 3, *args)
    if check:
        _check(rc, name)
    return out


def _real(precision):
    return ctypes.c_float if precision == "f32" else ctypes.c_double


def cst_space(rgb: np.ndarray, src: int, dst: int, precision: str = "f32"):
    """cst (cst.rs:6-10) between XyzD65, LinearSrgb, Srgb, AcesCg and Oklch."""
    return _rgb_op("oracle_cst_space", rgb, precision, [ctypes.c_int, ctypes.c_int], src, dst, check=True)


def highlight(rgb: np.ndarray, wb, precision: str = "f32"):
    """highlight_reconstruction (highlight_reconstruction.rs:5-13); clip_g = wb[1]."""
    return _rgb_op("oracle_highlight", rgb, precision, [_real(precision)], float(wb[1]))


def contrast(rgb: np.ndarray, c: float, precision: str = "f32"):
    return _rgb_op("oracle_contrast", rgb, precision, [_real(precision)], c)


def gamma(rgb: np.ndarray, g: float, precision: str = "f32"):
    return _rgb_op("oracle_gamma", rgb, precision, [_real(precision)], g)


def lch(rgb: np.ndarray, cs: int, lc: float, cc: float, hc: float, precision: str = "f32"):
    r = _real(precision)
    return _rgb_op("oracle_lch", rgb, precision, [ctypes.c_int, r, r, r], cs, lc, cc, hc, check=True)


def sigmoid(rgb: np.ndarray, precision: str = "f32"):
    return _rgb_op("oracle_sigmoid", rgb, precision, [])


def square_sigmoid(x: float, precision: str = "f32") -> float:
    fn = _f("oracle_square_sigmoid", precision)
    fn.argtypes = [_real(precision)]
    fn.restype = _real(precision)
    return fn(x)


def blur(plane: np.ndarray, sigma: float, precision: str = "f32"):
    dt = _dt(precision)
    out = np.ascontiguousarray(plane, dtype=dt).copy()
    H, W = out.shape
    fn = _f("oracle_blur", precision)
    real = ctypes.c_float if precision == "f32" else ctypes.c_double
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, real]
    fn(_ptr(out), W, H, sigma)
    return out


def grain_noise(W: int, H: int, seed: int, layer: int, precision: str = "f32"):
    dt = _dt(precision)
    out = np.zeros((H, W), dtype=dt)
    fn = _f("oracle_grain_noise", precision)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int]
    fn(_ptr(out), W, H, seed, layer)
    return out


def film_process(rgb: np.ndarray, stock: int = STOCK_COLORNEG200, film_format: int = 0, seed: int = 1,
                 output: int = 0, shutter: float = -1.0, grain: bool = True, precision: str = "f32"):
    dt = _dt(precision)
    out = np.ascontiguousarray(rgb, dtype=dt).copy()
    H, W = out.shape[:2]
    fn = _f("oracle_film_process", precision)
    real = ctypes.c_float if precision == "f32" else ctypes.c_double
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                   ctypes.c_int, real, ctypes.c_int]
    _check(fn(_ptr(out), W, H, stock, film_format, seed, output, shutter, int(grain)), "film_process")
    return out


def invert(buf: np.ndarray, mid, dmin, precision: str = "f32"):
    dt = _dt(precision)
    out = np.ascontiguousarray(buf, dtype=dt).copy()
    m = np.asarray(mid, dtype=dt)
    d = np.asarray(dmin, dtype=dt)
    fn = _f("oracle_invert", precision)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    fn(_ptr(out), out.size // 3, _ptr(m), _ptr(d))
    return out


def lut_sample(stock: int, layer: int, phi: float) -> float:
    fn = lib().oracle_lut_sample_f32
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
    fn.restype = ctypes.c_double
    return fn(stock, layer, phi)


def lut_build_sample(mu_ln: float, sigma_ln: float, k: float, phi: float) -> float:
    fn = lib().oracle_lut_build_sample_f64
    fn.argtypes = [ctypes.c_double] * 4
    fn.restype = ctypes.c_double
    return fn(mu_ln, sigma_ln, k, phi)


def layer_kappa(stock: int, layer: int) -> float:
    fn = lib().oracle_layer_kappa_f32
    fn.argtypes = [ctypes.c_int, ctypes.c_int]
    fn.restype = ctypes.c_float
    return fn(stock, layer)


def normalized_dmin(stock: int):
    out = np.zeros(3, dtype=np.float32)
    fn = lib().oracle_normalized_dmin_f32
    fn.argtypes = [ctypes.c_int, ctypes.c_void_p]
    fn(stock, _ptr(out))
    return out


def upsample_roundtrip(rgb):
    v = np.asarray(rgb, dtype=np.float64)
    spec = np.zeros(16)
    back = np.zeros(3)
    fn = lib().oracle_upsample_roundtrip_f64
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn(_ptr(v), _ptr(spec), _ptr(back))
    return spec, back


def cmf81():
    x, y, z = np.zeros(81), np.zeros(81), np.zeros(81)
    fn = lib().oracle_cmf81_f64
    fn.argtypes = [ctypes.c_void_p] * 3
    fn(_ptr(x), _ptr(y), _ptr(z))
    return x, y, z


def baseline_params(**kw) -> OracleBaseline:
    """The baseline preset's defaults (the 24 MP film workload), overridable."""
    p = OracleBaseline()
    d = dict(dmax=(2.0, 2.1, 2.2), k=(2.3, 2.5, 2.7), x0=(-0.70, -0.73, -0.76), hal_strength=0.15,
             hal_sigma=20.0, hal_radius=64, hal_threshold=0.8, grain_sigma=0.02, grain_blur=1.0, grain_on=1,
             seed=1)
    d.update(kw)
    for name in ("dmax", "k", "x0"):
        for i in range(3):
            getattr(p, name)[i] = d[name][i]
    for name in ("hal_strength", "hal_sigma", "hal_radius", "hal_threshold", "grain_sigma", "grain_blur",
                 "grain_on", "seed"):
        setattr(p, name, d[name])
    return p


def film_baseline(rgb: np.ndarray, params: OracleBaseline | None = None, precision: str = "f64",
                  threads: int = 0):
    """Baseline (81-bin) film preset; the FP64 build is the oracle of record."""
    dt = _dt(precision)
    out = np.ascontiguousarray(rgb, dtype=dt).copy()
    H, W = out.shape[:2]
    p = params if params is not None else baseline_params()
    fn = _f("oracle_film_baseline", precision)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OracleBaseline), ctypes.c_int]
    _check(fn(_ptr(out), W, H, ctypes.byref(p), threads or os.cpu_count()), "film_baseline")
    return out


class OracleGrad(ctypes.Structure):
    """Parameters of the differentiable colour + film model (mirrors OGrad /
    ImopsFilmGradParams): wb3, matrix9, ev, dmax3, k3, x03, hal_strength, hal_sigma."""

    _fields_ = [("wb", ctypes.c_float * 3), ("matrix", ctypes.c_float * 9), ("ev", ctypes.c_float),
                ("dmax", ctypes.c_float * 3), ("k", ctypes.c_float * 3), ("x0", ctypes.c_float * 3),
                ("hal_strength", ctypes.c_float), ("hal_sigma", ctypes.c_float)]

    def to_vector(self) -> np.ndarray:
        return np.array(list(self.wb) + list(self.matrix) + [self.ev] + list(self.dmax) + list(self.k) +
                        list(self.x0) + [self.hal_strength, self.hal_sigma], dtype=np.float64)

    @classmethod
    def from_vector(cls, v) -> "OracleGrad":
        g = cls()
        v = list(map(float, v))
        for i in range(3):
            g.wb[i] = v[i]
        for i in range(9):
            g.matrix[i] = v[3 + i]
        g.ev = v[12]
        for i in range(3):
            g.dmax[i], g.k[i], g.x0[i] = v[13 + i], v[16 + i], v[19 + i]
        g.hal_strength, g.hal_sigma = v[22], v[23]
        return g


def param_forward(x: np.ndarray, params: OracleGrad, fixed: OracleBaseline | None = None) -> np.ndarray:
    """FP64 forward of the differentiable model from camera RGB (H, W, 3)."""
    xx = np.ascontiguousarray(x, dtype=np.float64)
    H, W = xx.shape[:2]
    out = np.zeros_like(xx)
    f = fixed if fixed is not None else baseline_params(grain_on=0)
    fn = lib().oracle_param_forward_f64
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OracleGrad),
                   ctypes.POINTER(OracleBaseline), ctypes.c_void_p]
    _check(fn(_ptr(xx), W, H, ctypes.byref(params), ctypes.byref(f), _ptr(out)), "param_forward")
    return out


def param_grad(x: np.ndarray, target: np.ndarray, params: OracleGrad, scale: float,
               fixed: OracleBaseline | None = None) -> np.ndarray:
    """Analytic FP64 gradient of scale * sum((out - target)^2); returns 25
    values (24 parameter gradients, then the loss)."""
    xx = np.ascontiguousarray(x, dtype=np.float64)
    tt = np.ascontiguousarray(target, dtype=np.float64)
    H, W = xx.shape[:2]
    g = np.zeros(25)
    f = fixed if fixed is not None else baseline_params(grain_on=0)
    fn = lib().oracle_param_grad_f64
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OracleGrad),
                   ctypes.POINTER(OracleBaseline), ctypes.c_double, ctypes.c_void_p]
    _check(fn(_ptr(xx), _ptr(tt), W, H, ctypes.byref(params), ctypes.byref(f), scale, _ptr(g)), "param_grad")
    return g


LSB16 = 1.0 / 65535.0  # one 16-bit step of linear [0, 1]
FLIP_LSB = 8.0  # colour errors above this are AMaZE taking another branch in f32 than in f64


def error_figures(got: np.ndarray, ref64: np.ndarray, skip: np.ndarray | None = None) -> dict:
    """Max and RMS absolute error of `got` against the FP64 oracle `ref64`,
    in linear [0, 1] and in 16-bit LSB, over the pixels not in `skip` (an
    (H, W) mask, e.g. AMaZE decision flips, counted apart)."""
    e = np.abs(got.astype(np.float64) - ref64)
    if skip is not None:
        e = e[~skip]
    mx, rms = float(e.max()), float(np.sqrt(np.mean(e * e)))
    return {"max_abs": mx, "rms_abs": rms, "max_lsb": mx / LSB16, "rms_lsb": rms / LSB16}


def decision_flips(colour_f32: np.ndarray, colour_f64: np.ndarray) -> np.ndarray:
    """Pixels whose f32 colour forward is more than FLIP_LSB from the FP64
    chain: AMaZE resolved a comparison differently in f32 than in f64."""
    return (np.abs(colour_f32.astype(np.float64) - colour_f64) / LSB16).max(axis=2) > FLIP_LSB


def colour_chain(raw: np.ndarray, black: float, white: float, wb_coeffs, calib, precision: str = "f64",
                 threads: int = 0) -> np.ndarray:
    """u16 frame -> black/white scaling -> AMaZE -> WB -> camera matrix to
    ACEScg: the colour half of the 24 MP forward (f32: the reference's
    operation order; f64: the FP64 oracle)."""
    H, W = raw.shape
    m = scale_u16(raw, (0, 0, W, H), black, white, precision=precision)
    rgb = wb(amaze(m, "RGGB", precision=precision, threads=threads), wb_coeffs, precision=precision)
    return camera_cst(rgb, calib, CS_ACESCG, precision=precision)
