"""The C-ABI library loads on a machine without a GPU and exports every
entry point include/lmgpu.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

from lightmetrica_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "lmgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lmgpu_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("lmgpu_scene_create", "lmgpu_intersect", "lmgpu_render", "lmgpu_occluded"):
        assert s in syms


@pytest.mark.parametrize("path", [native.LIB_PATH, native.CHECK_LIB_PATH], ids=["product", "bounds_checked"])
def test_library_exports_every_declared_symbol(path):
    lib = ctypes.CDLL(path)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"missing exports: {missing}"


def test_python_binding_covers_header():
    assert set(declared_symbols()) <= set(native.SIGNATURES)
    assert native.lib().lmgpu_abi_version() == 1


def test_invalid_arguments_fail_without_gpu():
    L = native.lib()
    assert L.lmgpu_scene_create(None, None) == native.ERR_INVALID
    assert L.lmgpu_scene_info(None, None) == native.ERR_INVALID
    assert b"null" in L.lmgpu_last_error()
