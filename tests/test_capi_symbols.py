"""The C-ABI library loads and exports every entry point include/incrmt.h
declares, and rejects invalid arguments before touching the GPU (CPU only)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "incrmt.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(incrmt_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from incrmt_b200 import capi
    L = capi.lib()
    names = _declared()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_bad_arguments_rejected_without_gpu():
    from incrmt_b200 import capi
    L = capi.lib()
    h = ctypes.c_void_p()
    assert L.incrmt_mg_create(7, 64, 64, -1.0, 1.0, -1.0, 1.0, 0, 0, 0, ctypes.byref(h)) == capi.ERR_BADARG
    assert b"unknown system" in L.incrmt_last_error()
    # A periodic direction needs an even number of unknowns (four-colour ordering).
    assert L.incrmt_mg_create(0, 63, 64, -1.0, 1.0, -1.0, 1.0, 1, 0, 0, ctypes.byref(h)) == capi.ERR_BADARG
    assert L.incrmt_mg_create(0, 1, 64, -1.0, 1.0, -1.0, 1.0, 0, 0, 0, ctypes.byref(h)) == capi.ERR_BADARG
    # The solver and simulation switches refuse a null handle before touching a device.
    assert L.incrmt_mg_set_krylov(None, 1) == capi.ERR_BADARG
    assert L.incrmt_mg_krylov_fallbacks(None) == 0
    assert L.incrmt_sim_set_krylov(None, 1) == capi.ERR_BADARG
    assert L.incrmt_mg_set_coarse_refresh(None, 4) == capi.ERR_BADARG
    assert L.incrmt_sim_set_guess(None, 1) == capi.ERR_BADARG


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from incrmt_b200 import capi
    monkeypatch.setattr(capi, "_lib", None)
    monkeypatch.setattr(capi, "_LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(ImportError):
        capi.lib()
