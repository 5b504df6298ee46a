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
