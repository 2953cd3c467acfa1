"""The C-ABI library builds for sm_100a, loads, and exports every entry point
include/profit_b200.h declares.  No compute call is made here (no GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

import profit_b200
from profit_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    hdr = open(os.path.join(ROOT, "include", "profit_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(pf_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(_capi.LIB_PATH), "build with python -m profit_b200.build"
    lib = ctypes.CDLL(_capi.LIB_PATH)
    declared = _declared()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) <= set(_capi.EXPORTED) | {"pf_last_error"}


def test_build_targets_sm100a_only():
    from profit_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "--fmad=false" in build.UNITS["render64.cu"]


def test_version_and_error_channel():
    L = _capi.lib()
    assert b"libprofit 1.9.3" in L.pf_version()
    # an invalid call reports through pf_last_error without touching a device
    st = L.pf_model_set_magzero(None, 1.0)
    assert st == _capi.PF_E_INVALID
    assert b"null" in L.pf_last_error()
