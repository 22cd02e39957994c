"""The C-ABI library loads and exports every entry point that
include/pickle_b200.h declares (no device calls here)."""
import ctypes
import os
import re

import pytest

import pickle_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "pickle_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pk_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = pickle_b200.lib()
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(L, s), f"{s} not exported"


def test_version_and_error_string():
    L = pickle_b200.lib()
    assert L.pk_version() >= 100
    assert isinstance(L.pk_last_error(), bytes)


def test_bad_arguments_are_rejected_without_a_device():
    L = pickle_b200.lib()
    h = ctypes.c_void_p()
    # metric 7 is rejected before any device call
    assert L.pk_index_create(ctypes.byref(h), 7, 2, 16, 8, 32) == -1
    assert b"metric" in L.pk_last_error()
    assert L.pk_index_create(None, 1, 2, 16, 8, 32) == -1


def test_header_constants_match_reference_enums():
    src = open(os.path.join(ROOT, "include", "pickle_b200.h")).read()
    # DistFunc and DataType values of include/common.hpp:21-33
    assert "#define PK_METRIC_L2 1" in src and "#define PK_METRIC_IP 2" in src
    for name, v in [("U8", 0), ("I8", 1), ("F32", 2), ("F16", 3)]:
        assert f"#define PK_DTYPE_{name} {v}" in src


def test_no_device_gives_status_not_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    L = pickle_b200.lib()
    h = ctypes.c_void_p()
    assert L.pk_index_create(ctypes.byref(h), 1, 2, 16, 8, 32) == -9
