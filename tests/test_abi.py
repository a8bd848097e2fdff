"""The C ABI library loads and exports every symbol include/drnum_b200.h
declares (no compute call: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

from drnum_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "drnum_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*int\s+(dn_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_api():
    syms = declared_symbols()
    assert "dn_rk_step" in syms and "dn_ctx_create" in syms
    assert len(syms) >= 15


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for s in declared_symbols():
        assert hasattr(lib, s), s


def test_binding_covers_every_declared_symbol():
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_null_arguments_rejected_without_gpu():
    lib = _lib.load()
    assert lib.dn_ctx_create(0, 7, None) == _lib.DN_ERR_ARG
    assert lib.dn_ctx_destroy(None) == _lib.DN_OK
    assert lib.dn_rk_step(None, 1.0, None, 3) == _lib.DN_ERR_ARG
    assert lib.dn_sync(None) == _lib.DN_ERR_ARG
