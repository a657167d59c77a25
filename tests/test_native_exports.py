"""The C-ABI library loads and exports every symbol include/raspa_gpu.h
declares (no GPU needed: nothing is computed)."""
import ctypes as C
import os
import re

import pytest

from raspa2_b200 import build, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "raspa_gpu.h")) as fh:
        txt = fh.read()
    return sorted(set(re.findall(r"\b(rgpu_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = native.load()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert set(declared_symbols()) == set(native.EXPORTS)


def test_library_is_built_for_sm100a():
    # the in-tree build targets sm_100a only
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)
    assert os.path.exists(build.LIB)


def test_errors_are_codes_not_exits():
    L = native.load()
    h = C.c_void_p()
    rc = L.rgpu_system_create(C.byref(h), None)
    assert rc == -1
    assert b"null" in L.rgpu_error_string(rc)


def test_constants_match_header():
    """Precision, framework-model and error constants of native.py equal the
    header's #defines."""
    with open(os.path.join(ROOT, "include", "raspa_gpu.h")) as fh:
        defs = dict(re.findall(r"#define\s+(RGPU_[A-Z0-9_]+)\s+(-?\d+)\b", fh.read()))
    names = ["RGPU_FP64", "RGPU_MIXED", "RGPU_MIXED_CC64", "RGPU_E_INVALID", "RGPU_FRAMEWORK_FULL",
             "RGPU_FRAMEWORK_GRID"]
    for n in names:
        assert int(defs[n]) == getattr(native, n), n
