"""CPU-side checks of the CUDA library: it loads, exports every symbol the
header declares, and its host-only helpers agree with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "mlp_b200.h")) as f:
        src = f.read()
    return sorted(set(re.findall(r"\b(mlp_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from ml_prec_b200 import _capi
    if not os.path.exists(_capi.LIB_PATH):
        pytest.skip("CUDA library not built")
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) == set(_capi.EXPORTS)


def test_generate_x0_matches_oracle():
    from ml_prec_b200 import _capi
    if not os.path.exists(_capi.LIB_PATH):
        pytest.skip("CUDA library not built")
    import ml_prec_b200 as M
    from oracle import oracle as O
    for n in (1, 7, 1000, 100003):
        assert np.array_equal(M.generate_x0(n), O.generate_x0(n))


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from ml_prec_b200 import _capi
    monkeypatch.setattr(_capi, "LIB_PATH", str(tmp_path / "nope.so"))
    monkeypatch.setattr(_capi, "_lib", None)
    with pytest.raises(ImportError):
        _capi.lib()


def test_argument_errors_need_no_device():
    """Invalid arguments are rejected with a status and a message before the
    library touches a device (the reference throws for the same inputs)."""
    from ml_prec_b200 import _capi
    if not os.path.exists(_capi.LIB_PATH):
        pytest.skip("CUDA library not built")
    import ctypes as C
    lib = _capi.lib()
    vp = C.c_void_p
    u32 = C.POINTER(C.c_uint32)
    f64 = C.POINTER(C.c_double)
    # a row whose diagonal is not first (SkylineMatrix layout, skyline.cc:30-58)
    ia = np.array([0, 2, 4], np.uint32)
    ja = np.array([1, 0, 1, 0], np.uint32)
    a = np.array([-1.0, 2.0, 2.0, -1.0])
    h = vp()
    rc = lib.mlp_matrix_create(2, ia.ctypes.data_as(u32), ja.ctypes.data_as(u32), a.ctypes.data_as(f64), C.byref(h))
    assert rc == 1 and b"diagonal must come first in row 0" in lib.mlp_last_error()
    # a row without entries
    ia = np.array([0, 1, 1], np.uint32)
    ja = np.array([0, 0, 0, 0], np.uint32)
    rc = lib.mlp_matrix_create(2, ia.ctypes.data_as(u32), ja.ctypes.data_as(u32), a.ctypes.data_as(f64), C.byref(h))
    assert rc == 1 and b"row 1" in lib.mlp_last_error()
    # a NaN matrix value is refused before anything reaches a device (MLP_ERR_NOT_FINITE)
    ia = np.array([0, 2, 4], np.uint32)
    ja = np.array([0, 1, 1, 0], np.uint32)
    a = np.array([2.0, -1.0, np.nan, -1.0])
    rc = lib.mlp_matrix_create(2, ia.ctypes.data_as(u32), ja.ctypes.data_as(u32), a.ctypes.data_as(f64), C.byref(h))
    assert rc == 5 and b"non-finite matrix value at entry 2" in lib.mlp_last_error()
    # null handles
    assert lib.mlp_prec_create(None, None, None) == 1
    assert lib.mlp_pcg(None, None, None, None, 1e-8, 0, 0, None) == 1
    assert lib.mlp_matrix_size(None, None, None) == 1
