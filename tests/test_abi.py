"""C ABI checks that need no GPU: the library loads, exports exactly the symbols
``include/imps_b200.h`` declares, and reports a missing device with IMPS_NO_DEVICE."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "imps_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(imps_[a-z0-9_]+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert len(syms) >= 40
    assert "imps_ac_apply" in syms and "imps_vumps_iter" in syms and "imps_envs_build" in syms


def test_library_exports_every_declared_symbol():
    from infinitempsalgorithms_b200 import _lib
    lib = _lib.load()
    for s in declared_symbols():
        assert hasattr(lib, s), f"{s} declared in imps_b200.h but not exported"
    # and the ctypes table covers the same set
    assert sorted(_lib.exported_symbols()) == declared_symbols()


def test_status_strings_and_no_device():
    from infinitempsalgorithms_b200 import _lib
    lib = _lib.load()
    assert lib.imps_status_string(_lib.IMPS_DIM_MISMATCH) == b"dimension mismatch"
    import torch
    if not torch.cuda.is_available():
        h = ctypes.c_void_p()
        assert lib.imps_ctx_create(0, ctypes.byref(h)) == _lib.IMPS_NO_DEVICE


def test_null_arguments_are_rejected():
    from infinitempsalgorithms_b200 import _lib
    lib = _lib.load()
    assert lib.imps_ctx_create(0, None) == _lib.IMPS_INVALID_ARG
    assert lib.imps_ctx_set_precision(None, 0, 5) == _lib.IMPS_INVALID_ARG
    assert lib.imps_ac_apply(None, None, 0, None, None) == _lib.IMPS_INVALID_ARG
    assert lib.imps_envs_build(None, None, None, 1e-10, 300, 30, 0, None) == _lib.IMPS_INVALID_ARG


def test_host_api_errors_without_touching_gpu():
    import infinitempsalgorithms_b200 as imps
    with pytest.raises(ValueError):
        imps.DynamicTol(dict(tol=1e-8, maxiter=10), 1.0, 0.1, 0.1)
    with pytest.raises(imps.DimensionMismatch):
        W = imps.mpohamiltonian(imps.sigma("z"), [(1.0, imps.sigma("x"), imps.sigma("x"))])
        W2 = imps.mpohamiltonian(imps.sigma("z"), [])
        imps.SparseIMPO([W, W2])
    assert imps.updatetol(imps.Defaults.alg_eigsolve(), 4, 1e-2)["tol"] == pytest.approx(5e-6)
