"""imops_b200 -- B200 (sm_100a) raw-development path of DavRack/imops.

The product is the C-ABI shared library ``libimops_b200.so`` built from
``imops_b200/csrc`` (see ``include/imops_b200.h``).  This module loads it
with ctypes and offers thin torch wrappers over the device entry points.
There is no CPU fallback: without the library every call raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libimops_b200.so")
_lib = None

OK = 0
ERRORS = {
    1: "invalid argument", 2: "unsupported CFA", 3: "unsupported size", 4: "CUDA error", 5: "out of memory",
    6: "wrong color space", 7: "invalid dimensions", 8: "invalid stock", 9: "config error", 10: "not implemented",
    11: "timeout",
}
CS_CAMERA, CS_XYZD65, CS_LINEAR_SRGB, CS_SRGB, CS_ACESCG, CS_OKLCH = -1, 0, 1, 2, 3, 4
DEMOSAIC_AMAZE, DEMOSAIC_MARKESTEIJN, DEMOSAIC_FAST, DEMOSAIC_SUPERFAST, DEMOSAIC_SUPERSUPERFAST = range(5)


class ImopsError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"imops_b200 error {code} ({ERRORS.get(code, '?')}): {message}")
        self.code = code
        self.message = message


def lib() -> ctypes.CDLL:
    """The loaded C-ABI library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python imops_b200/build.py` (or __graft_entry__.build())")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.imops_last_error.restype = ctypes.c_char_p
        _lib.imops_version.restype = ctypes.c_char_p
    return _lib


def last_error() -> str:
    return (lib().imops_last_error() or b"").decode()


def check(rc: int) -> None:
    if rc != OK:
        raise ImopsError(rc, last_error())


def version() -> str:
    return lib().imops_version().decode()


def _stream(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _require_cuda_f32(t, name: str):
    import torch
    if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor")


def _cfa(pattern: str) -> bytes:
    return pattern.encode()


def demosaic_amaze(mosaic, cfa: str = "RGGB", shift=(0, 0), clip_pt: float = 1.0, out=None, stream=None):
    """AMaZE (demosaic.rs:358-1379) on a (H, W) float32 CUDA mosaic -> (H, W, 3)."""
    import torch
    _require_cuda_f32(mosaic, "mosaic")
    H, W = mosaic.shape
    out = out if out is not None else torch.empty((H, W, 3), device=mosaic.device, dtype=torch.float32)
    f = lib().imops_demosaic_amaze
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                  ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]
    check(f(_ptr(mosaic), W, H, _cfa(cfa), shift[0], shift[1], clip_pt, _ptr(out), _stream(stream)))
    return out


def amaze_size_supported(W: int, H: int) -> bool:
    f = lib().imops_amaze_size_supported
    f.argtypes = [ctypes.c_int, ctypes.c_int]
    return bool(f(W, H))


def demosaic_markesteijn(mosaic, cfa: str, shift=(0, 0), out=None, stream=None):
    import torch
    _require_cuda_f32(mosaic, "mosaic")
    H, W = mosaic.shape
    out = out if out is not None else torch.empty((H, W, 3), device=mosaic.device, dtype=torch.float32)
    f = lib().imops_demosaic_markesteijn
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p]
    check(f(_ptr(mosaic), W, H, _cfa(cfa), shift[0], shift[1], _ptr(out), _stream(stream)))
    return out


def demosaic_markesteijn3(mosaic, cfa: str, shift=(0, 0), out=None, stream=None):
    """3-pass directional X-Trans demosaic (imops_demosaic_markesteijn3); (H, W, 3)."""
    import torch
    _require_cuda_f32(mosaic, "mosaic")
    H, W = mosaic.shape
    out = out if out is not None else torch.empty((H, W, 3), device=mosaic.device, dtype=torch.float32)
    f = lib().imops_demosaic_markesteijn3
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p]
    check(f(_ptr(mosaic), W, H, _cfa(cfa), shift[0], shift[1], _ptr(out), _stream(stream)))
    return out


def demosaic_quad(mosaic, cfa: str, factor: int, shift=(0, 0), stream=None):
    import torch
    _require_cuda_f32(mosaic, "mosaic")
    H, W = mosaic.shape
    out = torch.empty((H // factor, W // factor, 3), device=mosaic.device, dtype=torch.float32)
    f = lib().imops_demosaic_quad
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                  ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    check(f(_ptr(mosaic), W, H, _cfa(cfa), shift[0], shift[1], factor, _ptr(out), _stream(stream)))
    return out


def scale_u16(raw, crop, black, white, period=(2, 2), out=None, stream=None):
    """raw: (Hr, Wr) uint16 CUDA tensor (stored as int16/uint16); crop = (x, y, w, h)."""
    import torch
    x, y, w, h = crop
    pw, ph = period
    n = pw * ph
    bl = (ctypes.c_float * n)(*([float(b) for b in black] if hasattr(black, "__len__") else [float(black)] * n))
    wh = (ctypes.c_float * n)(*([float(v) for v in white] if hasattr(white, "__len__") else [float(white)] * n))
    out = out if out is not None else torch.empty((h, w), device=raw.device, dtype=torch.float32)
    f = lib().imops_scale_u16
    f.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 6 + [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                           ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    check(f(_ptr(raw), raw.shape[1], raw.shape[0], x, y, w, h, bl, wh, pw, ph, _ptr(out), _stream(stream)))
    return out


def cfa_coeffs(rgb, wb, stream=None):
    _require_cuda_f32(rgb, "rgb")
    c = (ctypes.c_float * 4)(*(list(wb) + [0.0] * (4 - len(wb))))
    f = lib().imops_cfa_coeffs
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    check(f(_ptr(rgb), rgb.numel() // 3, c, _stream(stream)))
    return rgb


def exp(rgb, ev: float, stream=None):
    _require_cuda_f32(rgb, "rgb")
    f = lib().imops_exp
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_float, ctypes.c_void_p]
    check(f(_ptr(rgb), rgb.numel() // 3, ev, _stream(stream)))
    return rgb


def baseline_exposure(rgb, baseline_ev: float, shutter: float, f_number: float, iso: float, stream=None) -> bool:
    _require_cuda_f32(rgb, "rgb")
    applied = ctypes.c_int(0)
    f = lib().imops_baseline_exposure
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                  ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
    check(f(_ptr(rgb), rgb.numel() // 3, baseline_ev, shutter, f_number, iso, ctypes.byref(applied),
            _stream(stream)))
    return bool(applied.value)


def camera_forward_matrix(calib):
    c = (ctypes.c_float * 9)(*[float(v) for v in calib])
    out = (ctypes.c_float * 9)()
    f = lib().imops_camera_forward_matrix
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    check(f(c, out))
    return [out[i] for i in range(9)]


def camera_cst(rgb, calib, target: int, stream=None):
    _require_cuda_f32(rgb, "rgb")
    c = (ctypes.c_float * 9)(*[float(v) for v in calib])
    f = lib().imops_camera_cst
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    check(f(_ptr(rgb), rgb.numel() // 3, c, target, _stream(stream)))
    return rgb


# ---- display stages (one launch each; the pipeline fuses consecutive ones) ---

def _pixel_call(name, rgb, argtypes, *args, stream=None):
    _require_cuda_f32(rgb, "rgb")
    f = getattr(lib(), name)
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t] + argtypes + [ctypes.c_void_p]
    check(f(_ptr(rgb), rgb.numel() // 3, *args, _stream(stream)))
    return rgb


def cst(rgb, source: int, target: int, stream=None):
    """cst (cst.rs:6-10) between CS_XYZD65, CS_LINEAR_SRGB, CS_SRGB, CS_ACESCG and CS_OKLCH."""
    return _pixel_call("imops_cst", rgb, [ctypes.c_int, ctypes.c_int], source, target, stream=stream)


def highlight_reconstruction(rgb, wb, stream=None):
    c = (ctypes.c_float * 4)(*(list(wb) + [0.0] * (4 - len(wb))))
    return _pixel_call("imops_highlight_reconstruction", rgb, [ctypes.c_void_p], c, stream=stream)


def contrast(rgb, value: float, stream=None):
    return _pixel_call("imops_contrast", rgb, [ctypes.c_float], value, stream=stream)


def gamma(rgb, g: float, stream=None):
    return _pixel_call("imops_gamma", rgb, [ctypes.c_float], g, stream=stream)


def lch(rgb, color_space: int, lc: float, cc: float, hc: float, stream=None):
    return _pixel_call("imops_lch", rgb, [ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float],
                       color_space, lc, cc, hc, stream=stream)


def sigmoid_tone_map(rgb, stream=None):
    return _pixel_call("imops_sigmoid_tone_map", rgb, [], stream=stream)


# ---- film -------------------------------------------------------------------

STOCK_BWSTUB, STOCK_COLORNEG200, STOCK_PORTRA400, STOCK_EKTAR100, STOCK_FUJIPRO400H = 0, 1, 2, 3, 4
STOCK_EKTACHROMEE100, STOCK_TRIX400, STOCK_BASELINE81 = 5, 6, 100
SCAN_FP32, SCAN_BF16_TC = 0, 1
FORMAT_35MM, FORMAT_6X6, FORMAT_4X5 = 0, 1, 2
FILM_NEGATIVE_LINEAR, FILM_POSITIVE_LINEAR = 0, 1


class FilmParams(ctypes.Structure):
    """ImopsFilmParams (include/imops_b200.h)."""

    _fields_ = [("stock", ctypes.c_int), ("film_format", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("output", ctypes.c_int), ("shutter_seconds", ctypes.c_float), ("grain", ctypes.c_int)]


class BaselineFilm(ctypes.Structure):
    """ImopsBaselineFilm (include/imops_b200.h)."""

    _fields_ = [("dmax", ctypes.c_float * 3), ("k", ctypes.c_float * 3), ("x0", ctypes.c_float * 3),
                ("hal_strength", ctypes.c_float), ("hal_sigma", ctypes.c_float), ("hal_radius", ctypes.c_int),
                ("hal_threshold", ctypes.c_float), ("grain_sigma", ctypes.c_float), ("grain_blur", ctypes.c_float),
                ("grain_on", ctypes.c_int), ("seed", ctypes.c_uint64), ("scan", ctypes.c_int)]


def baseline_film_defaults(**overrides) -> BaselineFilm:
    p = BaselineFilm()
    f = lib().imops_baseline_film_defaults
    f.argtypes = [ctypes.POINTER(BaselineFilm)]
    f(ctypes.byref(p))
    for k, v in overrides.items():
        if k in ("dmax", "k", "x0"):
            for i in range(3):
                getattr(p, k)[i] = v[i]
        else:
            setattr(p, k, v)
    return p


def film_process(rgb, stock: int = STOCK_COLORNEG200, film_format: int = FORMAT_35MM, seed: int = 1,
                 output: int = FILM_NEGATIVE_LINEAR, shutter: float = -1.0, grain: bool = True,
                 baseline: BaselineFilm | None = None, color_space: int = CS_ACESCG, stream=None):
    """film::process (film/mod.rs:77-129) in place on an (H, W, 3) float32 CUDA image."""
    _require_cuda_f32(rgb, "rgb")
    H, W = rgb.shape[:2]
    p = FilmParams(stock, film_format, seed, output, shutter, int(grain))
    f = lib().imops_film_process
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(FilmParams),
                  ctypes.c_void_p, ctypes.c_void_p]
    bptr = ctypes.byref(baseline) if baseline is not None else None
    check(f(_ptr(rgb), W, H, color_space, ctypes.byref(p), bptr, _stream(stream)))
    return rgb


class FilmStages:
    """The reference model's film sub-stages (imops_film_expose .. _invert),
    one call each, on an (H, W, 3) float32 ACEScg CUDA image.  Chained in
    order they give film_process's result; the planes are (E, H, W)."""

    def __init__(self, stock: int = STOCK_COLORNEG200, film_format: int = FORMAT_35MM, seed: int = 1,
                 output: int = FILM_NEGATIVE_LINEAR, shutter: float = -1.0, grain: bool = True):
        self.p = FilmParams(stock, film_format, seed, output, shutter, int(grain))
        n = ctypes.c_int(0)
        f = lib().imops_film_layers
        f.argtypes = [ctypes.POINTER(FilmParams), ctypes.POINTER(ctypes.c_int)]
        check(f(ctypes.byref(self.p), ctypes.byref(n)))
        self.layers = n.value

    def _call(self, name, argtypes, *args, stream=None):
        f = getattr(lib(), name)
        f.argtypes = argtypes + [ctypes.c_void_p]
        check(f(*args, _stream(stream)))

    def expose(self, rgb, stream=None):
        import torch
        _require_cuda_f32(rgb, "rgb")
        H, W = rgb.shape[:2]
        planes = torch.empty((self.layers, H, W), device=rgb.device, dtype=torch.float32)
        self._call("imops_film_expose", [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(FilmParams),
                                         ctypes.c_void_p], _ptr(rgb), W, H, ctypes.byref(self.p), _ptr(planes),
                   stream=stream)
        return planes

    def halation(self, planes, stream=None):
        _, H, W = planes.shape
        self._call("imops_film_halation", [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(FilmParams)],
                   _ptr(planes), W, H, ctypes.byref(self.p), stream=stream)
        return planes

    def develop(self, planes, stream=None):
        import torch
        _, H, W = planes.shape
        mask = torch.empty_like(planes)
        self._call("imops_film_develop", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(FilmParams)],
                   _ptr(planes), _ptr(mask), W, H, ctypes.byref(self.p), stream=stream)
        return planes, mask

    def grain(self, planes, stream=None):
        _, H, W = planes.shape
        self._call("imops_film_grain", [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(FilmParams)],
                   _ptr(planes), W, H, ctypes.byref(self.p), stream=stream)
        return planes

    def scan(self, planes, mask, stream=None):
        import torch
        _, H, W = planes.shape
        rgb = torch.empty((H, W, 3), device=planes.device, dtype=torch.float32)
        self._call("imops_film_scan", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(FilmParams), ctypes.c_void_p],
                   _ptr(planes), _ptr(mask), W, H, ctypes.byref(self.p), _ptr(rgb), stream=stream)
        return rgb

    def invert(self, rgb, stream=None):
        H, W = rgb.shape[:2]
        self._call("imops_film_invert", [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(FilmParams)],
                   _ptr(rgb), W, H, ctypes.byref(self.p), stream=stream)
        return rgb

    def run(self, rgb, stream=None):
        """All stages in film::process's order; returns the film RGB."""
        planes = self.halation(self.expose(rgb, stream), stream)
        planes, mask = self.develop(planes, stream)
        return self.invert(self.scan(self.grain(planes, stream), mask, stream), stream)


class DevelopParams(ctypes.Structure):
    """ImopsDevelopParams (include/imops_b200.h)."""

    _fields_ = [("demosaic", ctypes.c_int), ("cfa", ctypes.c_char_p), ("clip_pt", ctypes.c_float),
                ("wb", ctypes.c_float * 4), ("n_gain", ctypes.c_int), ("ev", ctypes.c_float * 2),
                ("target", ctypes.c_int), ("calib_d65", ctypes.c_float * 9), ("film", ctypes.c_int),
                ("film_params", FilmParams), ("baseline", BaselineFilm)]


def develop_u16(raw, crop, black, white, params: DevelopParams, period=(2, 2), out=None, stream=None):
    """Fused forward from a u16 frame (imops_develop_u16); returns (h, w, 3)."""
    import torch
    x, y, w, h = crop
    pw, ph = period
    n = pw * ph
    bl = (ctypes.c_float * n)(*([float(b) for b in black] if hasattr(black, "__len__") else [float(black)] * n))
    wh = (ctypes.c_float * n)(*([float(v) for v in white] if hasattr(white, "__len__") else [float(white)] * n))
    out = out if out is not None else torch.empty((h, w, 3), device=raw.device, dtype=torch.float32)
    f = lib().imops_develop_u16
    f.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 6 + [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                           ctypes.c_int, ctypes.POINTER(DevelopParams),
                                                           ctypes.c_void_p, ctypes.c_void_p]
    check(f(_ptr(raw), raw.shape[1], raw.shape[0], x, y, w, h, bl, wh, pw, ph, ctypes.byref(params), _ptr(out),
            _stream(stream)))
    return out


def develop_f32(mosaic, params: DevelopParams, shift=(0, 0), out=None, stream=None):
    import torch
    _require_cuda_f32(mosaic, "mosaic")
    h, w = mosaic.shape
    out = out if out is not None else torch.empty((h, w, 3), device=mosaic.device, dtype=torch.float32)
    f = lib().imops_develop_f32
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.POINTER(DevelopParams), ctypes.c_void_p, ctypes.c_void_p]
    check(f(_ptr(mosaic), w, h, shift[0], shift[1], ctypes.byref(params), _ptr(out), _stream(stream)))
    return out


def release_working_sets():
    """Frees the cached per-(device, stream) working sets on the current device."""
    f = lib().imops_release_working_sets
    f.argtypes = []
    check(f())


def launch_count() -> int:
    f = lib().imops_launch_count
    f.restype = ctypes.c_uint64
    return int(f())


class FilmGradParams(ctypes.Structure):
    """ImopsFilmGradParams: the 24 parameters of the differentiable model."""

    _fields_ = [("wb", ctypes.c_float * 3), ("matrix", ctypes.c_float * 9), ("ev", ctypes.c_float),
                ("dmax", ctypes.c_float * 3), ("k", ctypes.c_float * 3), ("x0", ctypes.c_float * 3),
                ("hal_strength", ctypes.c_float), ("hal_sigma", ctypes.c_float)]

    NAMES = (["wb_r", "wb_g", "wb_b"] + [f"m{i}{j}" for i in range(3) for j in range(3)] + ["ev"] +
             [f"dmax{l}" for l in range(3)] + [f"k{l}" for l in range(3)] + [f"x0_{l}" for l in range(3)] +
             ["hal_strength", "hal_sigma"])

    def to_vector(self):
        return [*self.wb, *self.matrix, self.ev, *self.dmax, *self.k, *self.x0, self.hal_strength, self.hal_sigma]

    @classmethod
    def from_vector(cls, v):
        g = cls()
        v = [float(a) for a in v]
        for i in range(3):
            g.wb[i] = v[i]
        for i in range(9):
            g.matrix[i] = v[3 + i]
        g.ev = v[12]
        for i in range(3):
            g.dmax[i], g.k[i], g.x0[i] = v[13 + i], v[16 + i], v[19 + i]
        g.hal_strength, g.hal_sigma = v[22], v[23]
        return g


def param_forward(cam_rgb, params: FilmGradParams, fixed: BaselineFilm | None = None, out=None, stream=None):
    import torch
    _require_cuda_f32(cam_rgb, "cam_rgb")
    H, W = cam_rgb.shape[:2]
    out = out if out is not None else torch.empty_like(cam_rgb)
    f = lib().imops_param_forward
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(FilmGradParams), ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    check(f(_ptr(cam_rgb), W, H, ctypes.byref(params), ctypes.byref(fixed) if fixed is not None else None,
            _ptr(out), _stream(stream)))
    return out


def param_backward(cam_rgb, params: FilmGradParams, grad, g_out=None, target=None, loss_scale: float = 1.0,
                   fixed: BaselineFilm | None = None, stream=None):
    """Adds d(loss)/d(params) into `grad` (a (25,) float64 CUDA tensor; [24] is the loss)."""
    _require_cuda_f32(cam_rgb, "cam_rgb")
    H, W = cam_rgb.shape[:2]
    f = lib().imops_param_backward
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                  ctypes.POINTER(FilmGradParams), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    check(f(_ptr(cam_rgb), _ptr(g_out) if g_out is not None else None, _ptr(target) if target is not None else None,
            loss_scale, W, H, ctypes.byref(params), ctypes.byref(fixed) if fixed is not None else None, _ptr(grad),
            _stream(stream)))
    return grad
