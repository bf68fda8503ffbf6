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


def test_status_codes_before_any_device_work(built_lib):
    """Each entry point refuses bad scalars with its documented status before it
    touches the device (so these run without a GPU)."""
    from ecs_mhd_2d_b200 import _lib
    lib = _lib.load()
    buf = (ctypes.c_double * 16)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    dp = ctypes.cast(buf, ctypes.POINTER(ctypes.c_double))
    INVALID, UNSUPPORTED, TOO_LARGE = 1, 6, 7
    # Arnoldi / Hessenberg: step index, lengths, re-orthogonalisation sweeps, m <= 128
    assert lib.ecs_arnoldi_mgs(dp, 8, -2, dp, dp, 8, None) == INVALID
    assert lib.ecs_arnoldi_mgs(dp, 4, 0, dp, dp, 8, None) == INVALID          # ld < len
    assert lib.ecs_arnoldi_mgs(dp, 8, 0, dp, dp, 0, None) == INVALID          # empty vectors
    assert lib.ecs_arnoldi_mgs_reorth(dp, 8, 0, dp, dp, 8, 5, None) == INVALID
    assert lib.ecs_arnoldi_mgs(None, 8, 0, dp, dp, 8, None) == INVALID
    assert lib.ecs_hessenberg_lstsq(dp, 130, 129, dp, dp, None) == INVALID
    assert lib.ecs_hessenberg_lstsq(dp, 4, 4, dp, dp, None) == INVALID       # ldh < m + 1
    assert lib.ecs_hessenberg_lstsq(dp, 2, 0, dp, dp, None) == INVALID
    # allocation-free state_vel: n and batch limits of its fixed scratch
    assert lib.ecs_state_vel_noalloc(256, 0.02, 0.02, 0.0, 0.1, dp, p, p, 1, 0, None) == TOO_LARGE
    assert lib.ecs_state_vel_noalloc(64, 0.02, 0.02, 0.0, 0.1, dp, p, p, 5, 0, None) == TOO_LARGE
    assert lib.ecs_state_vel_noalloc(64, 0.02, 0.02, 0.0, 0.1, dp, p, p, 0, 0, None) == INVALID
    assert lib.ecs_state_vel_noalloc(64, 0.02, 0.02, 0.0, 0.1, None, p, p, 1, 0, None) == INVALID
    # entry points given no context
    assert lib.ecs_objective(None, None, p, dp, dp, p, dp, dp, None, 1, None) == INVALID
    assert lib.ecs_jvp(None, p, dp, dp, p, dp, dp, 1, None) == INVALID
    assert lib.ecs_vjp(None, p, dp, dp, p, dp, dp, 1, None) == INVALID
    assert lib.ecs_ctx_create(256, 1, None, 1, None) == INVALID
    prm = _lib.EcsParams()
    h = ctypes.c_void_p()
    assert lib.ecs_ctx_create(512, 0, ctypes.byref(prm), 1, ctypes.byref(h)) == UNSUPPORTED
