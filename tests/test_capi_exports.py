"""The C-ABI library loads and exports every entry point include/arctn_b200.h declares (no GPU needed)."""

import ctypes
import os
import re

from arctn_b200 import _capi as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "arctn_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(arctn_b200_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported():
    lib = ctypes.CDLL(C.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_bindings_cover_header():
    bound = {name for name, _, _ in C.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_abi_version_and_error_channel():
    L = C.lib()
    assert L.arctn_b200_abi_version() == 1
    net = C.NetworkArgs([[0, 1], [1, 2]], [0, 2], {0: 2, 1: 0, 2: 2})
    n, p = C.path_array([(0, 1)])
    h = C.vp()
    rc = L.arctn_b200_plan_compile(net.ptr, n, p.ctypes.data_as(C.u64p), ctypes.byref(h))
    assert rc == C.ERR_INVALID
    assert b"dimension 0" in L.arctn_b200_last_error()
