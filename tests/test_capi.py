"""The C-ABI library loads and exports every entry point declared in include/hyteg_b200.h."""
import ctypes
import os
import re

import hyteg_b200 as hg
from hyteg_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "hyteg_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hg_[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_symbol_is_exported():
    syms = declared_symbols()
    assert len(syms) > 30
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_symbols()) == set(_capi.DECLARED)


def test_errors_are_reported_not_raised_in_c():
    # invalid arguments return a status and a message, without touching a GPU
    h = ctypes.c_void_p()
    lo = (ctypes.c_double * 3)(0, 0, 0)
    hi = (ctypes.c_double * 3)(1, 1, 1)
    rc = _capi.lib.hg_mesh_create_cuboid(lo, hi, 0, 1, 1, 2, ctypes.byref(h))
    assert rc == _capi.HG_ERR_ARG
    assert b"subdivisions" in _capi.lib.hg_last_error()
    rc = _capi.lib.hg_mesh_create_cuboid(lo, hi, 1, 1, 1, 11, ctypes.byref(h))
    assert rc == _capi.HG_ERR_ARG


def test_storage_without_gpu_fails_loudly():
    if hg.device_count() > 0:
        return
    try:
        hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), 1, 1, 1, 2)
    except hg.HygError as e:
        assert e.code == _capi.HG_ERR_CUDA
    else:
        raise AssertionError("storage creation must fail without a CUDA device")
