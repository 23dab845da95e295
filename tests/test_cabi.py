"""The C-ABI library loads without a GPU and exports every function that
include/frost_b200.h declares, with the signatures frost_b200/_lib.py binds."""

import ctypes
import os
import re

from frost_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "frost_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(frost_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_without_gpu():
    L = _lib.lib()
    assert L.frost_version().decode().startswith("frost_b200")


def test_every_declared_symbol_is_exported_and_bound():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(L, name), f"{name} declared in frost_b200.h but not exported"
        assert name in _lib.SIGNATURES, f"{name} has no Python binding"


def test_errors_are_status_codes_not_crashes():
    import pytest
    from frost_b200.config import RfiConfig
    cfg = RfiConfig()
    cfg.narrow.threshold = -1.0
    c, keep = cfg.to_c()
    L = _lib.lib()
    rc = L.frost_rfi_config_validate(ctypes.byref(c))
    assert rc == -1
    assert "narrow.threshold" in L.frost_last_error().decode()
    with pytest.raises(ValueError):
        _lib.check(rc)
