"""C-ABI library: loads without a GPU and exports every declared entry point."""
import ctypes
import os
import re

import pytest

from bfps_b200 import _lib


def declared_functions():
    txt = open(_lib.HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bfg_[a-z0-9_]+)\s*\(", txt)))


def test_library_built():
    assert os.path.exists(_lib.LIB_PATH), "run python -m bfps_b200.build"


def test_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_version():
    assert b"sm_100a" in _lib.lib().bfg_version()


@pytest.mark.parametrize("args,code", [
    ((33, 33, 33, 1.0, 1.0, 1.0, 8, 1, 0), _lib.BFG_EUNSUP),   # not a power of two
    ((32, 32, 64, 1.0, 1.0, 1.0, 8, 1, 0), _lib.BFG_EUNSUP),   # not cubic
    ((32, 32, 32, 1.0, 1.0, 1.0, 3, 1, 0), _lib.BFG_EINVAL),   # bad real size
    ((32, 32, 32, 1.0, 1.0, 1.0, 8, 7, 0), _lib.BFG_EINVAL),   # bad dealias type
    ((32, 32, 32, 0.0, 1.0, 1.0, 8, 1, 0), _lib.BFG_EINVAL),   # bad dk
    ((2048, 2048, 2048, 1.0, 1.0, 1.0, 4, 1, 0), _lib.BFG_EUNSUP),
])
def test_create_rejects_bad_arguments(args, code):
    # these return before any CUDA call
    h = ctypes.c_void_p()
    assert _lib.lib().bfg_ctx_create(ctypes.byref(h), *args) == code
    assert not h.value


def test_solver_has_no_cpu_fallback(monkeypatch):
    # the product path fails loudly when the CUDA library is absent
    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libbfps_b200.so")
    monkeypatch.setattr(_lib, "_LIB", None)
    with pytest.raises(RuntimeError, match="not built"):
        _lib.lib()
