"""The C-ABI library loads and exports every symbol include/ocfd_b200.h
declares; no compute calls (runs without a GPU)."""
import ctypes
import os
import re

import pytest

from ocfd_b200 import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "ocfd_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text))
    return {n for n in names if n.startswith("ocfd_b200_") or n in
            ("du_comput", "OCFD_time_advance", "get_duvwT", "get_Amu", "OCFD_bc",
             "Set_Scheme_HybridAuto", "filtering")}


def test_header_and_binding_agree():
    assert _declared_symbols() == set(lib.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = lib.load()
    for name in _declared_symbols():
        assert hasattr(L, name), name


def test_abi_version_and_status_strings():
    L = lib.load()
    assert L.ocfd_b200_abi_version() == 1
    assert L.ocfd_b200_status_string(0) == b"ok"
    assert L.ocfd_b200_status_string(-2) == b"unsupported configuration"


def test_create_rejects_bad_arguments_without_a_gpu():
    # argument checks run before any device call
    L = lib.load()
    from ocfd_b200 import cases
    cfg = cases.taylor_green(16).cfg
    c = lib.make_config(cfg)
    c.nx = 4
    h = ctypes.c_void_p()
    assert L.ocfd_b200_create(ctypes.byref(c), ctypes.byref(h)) == -1
    c = lib.make_config(cfg)
    c.scheme_invis = 399
    assert L.ocfd_b200_create(ctypes.byref(c), ctypes.byref(h)) == -2
    c = lib.make_config(cfg)
    c.scheme_invis = 310
    c.hy_style = 1
    assert L.ocfd_b200_create(ctypes.byref(c), ctypes.byref(h)) == -2
    assert b"HY_STYLE" in L.ocfd_b200_last_error(None)
