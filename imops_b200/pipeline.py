"""Python mirror of the reference's pipeline API over the C-ABI.

Names follow pichromatic-pipeline: ``parse_config`` (config.rs:13-34),
``run_pixel_pipeline`` (pipeline.rs:4-13), ``get_pipeline_schema``
(modules.rs:917-923) and the Image accessors of extern_pipeline.rs.  The work
runs in libimops_b200.so (get_pixel_pipeline_c, run_pixel_pipeline_c, ...);
images stay on the GPU between modules.
"""
from __future__ import annotations

import ctypes
import json

import numpy as np

from . import CS_ACESCG, CS_CAMERA, CS_LINEAR_SRGB, CS_OKLCH, CS_SRGB, CS_XYZD65, ImopsError, last_error, lib

CS_NAMES = {CS_XYZD65: "XyzD65", CS_LINEAR_SRGB: "LinearSrgb", CS_SRGB: "Srgb", CS_ACESCG: "AcesCg",
            CS_OKLCH: "Oklch", CS_CAMERA: None}


class ImageMeta(ctypes.Structure):
    """ImopsImageMeta: the ImageMetadata fields the path reads (image.rs:7-50)."""

    _fields_ = [("cfa", ctypes.c_char_p), ("crop_x", ctypes.c_int), ("crop_y", ctypes.c_int),
                ("crop_w", ctypes.c_int), ("crop_h", ctypes.c_int), ("has_wb", ctypes.c_int),
                ("wb_coeffs", ctypes.c_float * 4), ("has_calibration", ctypes.c_int),
                ("calibration_matrix_d65", ctypes.c_float * 9), ("black_level", ctypes.c_float),
                ("white_level", ctypes.c_float), ("has_baseline_exposure", ctypes.c_int),
                ("baseline_exposure", ctypes.c_float), ("has_shutter", ctypes.c_int),
                ("shutter_seconds", ctypes.c_float), ("has_f_number", ctypes.c_int), ("f_number", ctypes.c_float),
                ("has_iso", ctypes.c_int), ("iso", ctypes.c_float)]


def make_meta(cfa: str | None = None, crop=(0, 0, 0, 0), wb=None, calibration=None, black=0.0, white=1.0,
              baseline_exposure=None, shutter=None, f_number=None, iso=None) -> ImageMeta:
    m = ImageMeta()
    m._cfa = cfa.encode() if cfa else None  # keep the bytes alive with the struct
    m.cfa = m._cfa
    m.crop_x, m.crop_y, m.crop_w, m.crop_h = crop
    if wb is not None:
        m.has_wb = 1
        for i, v in enumerate(list(wb) + [0.0] * (4 - len(wb))):
            m.wb_coeffs[i] = v
    if calibration is not None:
        m.has_calibration = 1
        for i, v in enumerate(calibration):
            m.calibration_matrix_d65[i] = v
    m.black_level, m.white_level = black, white
    for name, val in (("baseline_exposure", baseline_exposure), ("shutter_seconds", shutter),
                      ("f_number", f_number), ("iso", iso)):
        if val is not None:
            flag = {"baseline_exposure": "has_baseline_exposure", "shutter_seconds": "has_shutter",
                    "f_number": "has_f_number", "iso": "has_iso"}[name]
            setattr(m, flag, 1)
            setattr(m, name, val)
    return m


def _setup():
    L = lib()
    L.new_raw_image_u16_c.restype = ctypes.c_void_p
    L.new_raw_image_u16_c.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.POINTER(ImageMeta)]
    L.new_raw_image_f32_c.restype = ctypes.c_void_p
    L.new_raw_image_f32_c.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.POINTER(ImageMeta)]
    L.new_rgb_image_c.restype = ctypes.c_void_p
    L.new_rgb_image_c.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int,
                                  ctypes.POINTER(ImageMeta)]
    L.get_pixel_pipeline_c.restype = ctypes.c_void_p
    L.get_pixel_pipeline_c.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.run_pixel_pipeline_c.restype = ctypes.c_void_p
    L.run_pixel_pipeline_c.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.get_image_rgb_data_c.restype = ctypes.POINTER(ctypes.c_uint8)
    L.get_image_rgb_data_c.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                       ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
    L.get_image_rgb_f32_c.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
    L.get_image_info_c.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                   ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int)]
    L.get_image_metadata_c.restype = ctypes.c_void_p
    L.get_image_metadata_c.argtypes = [ctypes.c_void_p]
    L.get_pipeline_schema_c.restype = ctypes.c_void_p
    L.get_last_error_c.restype = ctypes.c_void_p
    L.free_image_c.argtypes = [ctypes.c_void_p]
    L.free_pipeline_c.argtypes = [ctypes.c_void_p]
    L.free_rgb_buffer_c.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
    L.free_string_c.argtypes = [ctypes.c_void_p]
    return L


def _take_string(L, ptr) -> str | None:
    if not ptr:
        return None
    s = ctypes.string_at(ptr).decode()
    L.free_string_c(ptr)
    return s


def get_last_error() -> str | None:
    L = _setup()
    return _take_string(L, L.get_last_error_c())


class Pipeline:
    """PipelineConfig: the parsed module list."""

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        if getattr(self, "_h", None):
            _setup().free_pipeline_c(self._h)
            self._h = None


def parse_config(text: str) -> Pipeline:
    L = _setup()
    b = text.encode()
    h = L.get_pixel_pipeline_c(b, len(b))
    if not h:
        raise ImopsError(9, last_error())
    return Pipeline(h)


def get_pipeline_schema() -> list:
    L = _setup()
    return json.loads(_take_string(L, L.get_pipeline_schema_c()))


class Image:
    """Device-resident Image (pixel.rs:23-27)."""

    def __init__(self, handle):
        self._h = handle

    @staticmethod
    def _check(h):
        if not h:
            raise ImopsError(1, last_error())
        return Image(h)

    @classmethod
    def from_u16(cls, raw: np.ndarray, meta: ImageMeta) -> "Image":
        r = np.ascontiguousarray(raw, dtype=np.uint16)
        L = _setup()
        img = cls._check(L.new_raw_image_u16_c(r.ctypes.data_as(ctypes.c_void_p), r.shape[1], r.shape[0],
                                               ctypes.byref(meta)))
        img._meta = meta
        return img

    @classmethod
    def from_mosaic(cls, raw_data: np.ndarray, meta: ImageMeta) -> "Image":
        r = np.ascontiguousarray(raw_data, dtype=np.float32)
        L = _setup()
        img = cls._check(L.new_raw_image_f32_c(r.ctypes.data_as(ctypes.c_void_p), r.shape[1], r.shape[0],
                                               ctypes.byref(meta)))
        img._meta = meta
        return img

    @classmethod
    def from_rgb(cls, rgb: np.ndarray, color_space: int, meta: ImageMeta | None = None) -> "Image":
        r = np.ascontiguousarray(rgb, dtype=np.float32)
        L = _setup()
        meta = meta if meta is not None else make_meta()
        img = cls._check(L.new_rgb_image_c(r.ctypes.data_as(ctypes.c_void_p), r.shape[1], r.shape[0], color_space,
                                           ctypes.byref(meta)))
        img._meta = meta
        return img

    def info(self):
        L = _setup()
        w, h, cs = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_int()
        if L.get_image_info_c(self._h, ctypes.byref(w), ctypes.byref(h), ctypes.byref(cs)):
            raise ImopsError(1, last_error())
        return w.value, h.value, cs.value

    def rgb_f32(self) -> np.ndarray:
        w, h, _ = self.info()
        out = np.empty((h, w, 3), np.float32)
        L = _setup()
        rc = L.get_image_rgb_f32_c(self._h, out.ctypes.data_as(ctypes.c_void_p), out.size)
        if rc:
            raise ImopsError(rc, last_error())
        return out

    def rgb_u8(self) -> np.ndarray:
        L = _setup()
        w, h, n = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
        p = L.get_image_rgb_data_c(self._h, ctypes.byref(w), ctypes.byref(h), ctypes.byref(n))
        if not p:
            raise ImopsError(1, last_error())
        out = np.ctypeslib.as_array(p, shape=(n.value,)).copy().reshape(h.value, w.value, 3)
        L.free_rgb_buffer_c(p, n.value)
        return out

    def metadata(self) -> dict:
        L = _setup()
        return json.loads(_take_string(L, L.get_image_metadata_c(self._h)))

    def __del__(self):
        if getattr(self, "_h", None):
            _setup().free_image_c(self._h)
            self._h = None


def run_pixel_pipeline(image: Image, pipeline: Pipeline) -> Image:
    L = _setup()
    r = L.run_pixel_pipeline_c(image._h, pipeline._h)
    if not r:
        err = last_error()
        code = 10 if "not part of the GPU path" in err or "not ported" in err or "not on the GPU path" in err else 1
        raise ImopsError(code, err)
    return image
