"""The C-ABI library builds, loads and exports every symbol of include/ecs_mhd.h (no GPU calls)."""
import ctypes
import os
import re

from conftest import ROOT


def header_symbols():
    src = open(os.path.join(ROOT, "include", "ecs_mhd.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ecs_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header_symbols(built_lib):
    lib = ctypes.CDLL(built_lib)
    syms = header_symbols()
    assert len(syms) >= 10
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header(built_lib):
    from ecs_mhd_2d_b200 import _lib
    assert set(header_symbols()) <= set(_lib.SIGNATURES), set(header_symbols()) - set(_lib.SIGNATURES)


def test_version_string(built_lib):
    lib = ctypes.CDLL(built_lib)
    lib.ecs_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.ecs_version()


def test_invalid_arguments_rejected_without_gpu(built_lib):
    from ecs_mhd_2d_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    prm = _lib.EcsParams()
    assert lib.ecs_ctx_create(100, 0, ctypes.byref(prm), 1, ctypes.byref(h)) == 6   # unsupported n
    assert lib.ecs_ctx_create(64, 7, ctypes.byref(prm), 1, ctypes.byref(h)) == 6    # unsupported dtype
    assert lib.ecs_ctx_create(64, 0, ctypes.byref(prm), 0, ctypes.byref(h)) == 1    # bad batch
    assert lib.ecs_to_box(None, None, None, 1, None) == 1
