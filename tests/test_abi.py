"""The C ABI library loads and exports every symbol include/fmmcuda.h declares (no GPU
compute here)."""
import ctypes
import os
import re

import pytest

from bachelors_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fmmcuda.h")).read()
    return sorted(set(re.findall(r"\b(fmm_[A-Za-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_version_and_default_config():
    lib = _lib.load()
    assert b"sm_100a" in lib.fmm_version()
    cfg = _lib.FmmConfig()
    lib.fmm_default_config(ctypes.byref(cfg))
    assert cfg.order == 10 and cfg.leaf_capacity == 64 and cfg.precision == _lib.FMM_FP32


def test_bad_config_is_rejected_without_touching_the_gpu():
    lib = _lib.load()
    cfg = _lib.FmmConfig()
    lib.fmm_default_config(ctypes.byref(cfg))
    cfg.order = 40
    h = ctypes.c_void_p()
    assert lib.fmm_plan_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.FMM_E_INVALID
    assert b"order" in lib.fmm_last_error_string()
    assert lib.fmm_add_vectors(None, None, None, -1) == _lib.FMM_E_INVALID
