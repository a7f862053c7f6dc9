"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares (no compute call is made here)."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "for", "while", "return", "sizeof"):
                names.add(name)
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "imops_demosaic_amaze" in names
    assert "imops_last_error" in names


def test_library_exports_every_declared_symbol():
    import imops_b200
    lib = imops_b200.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_last_error_and_version_without_gpu():
    import imops_b200
    assert "sm_100a" in imops_b200.version()
    assert isinstance(imops_b200.last_error(), str)


def test_amaze_size_rule_matches_oracle():
    import imops_b200
    import oracle
    for W in (20, 32, 96, 97, 100, 111, 112, 113, 160, 207, 1536, 6048, 6032, 2048):
        for H in (20, 50, 96, 97, 300, 320, 1024, 1365, 4024, 4032):
            assert imops_b200.amaze_size_supported(W, H) == oracle.amaze_size_ok(W, H), (W, H)


def test_host_forward_matrix_matches_oracle():
    import numpy as np
    import imops_b200
    import oracle
    from imops_b200 import synthetic
    ref = oracle.camera_forward_matrix(synthetic.CALIB_D65).reshape(9)
    got = np.asarray(imops_b200.camera_forward_matrix(synthetic.CALIB_D65), dtype=np.float32)
    assert np.array_equal(got, ref)


def test_invalid_cfa_is_reported_without_gpu():
    import imops_b200
    lib = imops_b200.lib()
    f = lib.imops_demosaic_markesteijn
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p]
    rc = f(None, 4, 4, b"RGB", 0, 0, None, None)
    assert rc == 2
    assert "CFA" in imops_b200.last_error()
