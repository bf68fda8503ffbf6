"""ctypes binding of ``libecsmhd.so`` (declared in include/ecs_mhd.h).

The shared library is built in-tree by ``ecs_mhd_2d_b200.build``.  There is no
fallback: if the library is missing or CUDA is unavailable every compute call
raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libecsmhd.so")

ECS_F64, ECS_F32 = 0, 1
ECS_MODE_LAWSON_RK4, ECS_MODE_LAWSON_RK43, ECS_MODE_RK4, ECS_MODE_LAWSON_RK6, ECS_MODE_TDRK4 = 1, 2, 3, 4, 5

STATUS = {
    0: "ECS_OK", 1: "ECS_ERR_INVALID", 2: "ECS_ERR_CUDA", 3: "ECS_ERR_BAD_MODE",
    4: "ECS_ERR_NOT_COMPLETED", 5: "ECS_ERR_OOM", 6: "ECS_ERR_UNSUPPORTED", 7: "ECS_ERR_TOO_LARGE",
}


class EcsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class EcsParams(ctypes.Structure):
    _fields_ = [("nu", ctypes.c_double), ("eta", ctypes.c_double),
                ("b0x", ctypes.c_double), ("b0y", ctypes.c_double),
                ("forcing", ctypes.POINTER(ctypes.c_double)),
                ("kolmogorov_amp", ctypes.c_double), ("kolmogorov_k", ctypes.c_int)]


class EcsShootCfg(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("num_checkpoints", ctypes.c_int), ("ministeps", ctypes.c_int),
                ("shift_reflect_ny", ctypes.c_int), ("rot", ctypes.c_int), ("atol", ctypes.c_double),
                ("h0", ctypes.c_double), ("max_steps_per_checkpoint", ctypes.c_int),
                ("checkpoints", ctypes.c_int), ("ckpt_every", ctypes.c_int)]


class EcsInfo(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int), ("s", ctypes.c_double), ("accepted", ctypes.c_int),
                ("rejected", ctypes.c_int), ("fevals", ctypes.c_int)]


_VP = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double

# name -> (restype, argtypes); must match include/ecs_mhd.h
SIGNATURES = {
    "ecs_version": (ctypes.c_char_p, []),
    "ecs_ctx_create": (_I, [_I, _I, ctypes.POINTER(EcsParams), _I, ctypes.POINTER(_VP)]),
    "ecs_ctx_destroy": (_I, [_VP]),
    "ecs_last_error": (ctypes.c_char_p, [_VP]),
    "ecs_launch_count": (ctypes.c_longlong, [_VP]),
    "ecs_bench_kernel": (_I, [_VP, _I, _I, _I, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double), _VP]),
    "ecs_jvp_multi": (_I, [_VP, ctypes.POINTER(EcsShootCfg), _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _I,
                           _VP]),
    "ecs_loss_grad_multi": (_I, [_VP, ctypes.POINTER(EcsShootCfg), _VP, _VP, _VP, _VP, _VP, _VP, _VP, _I, _VP]),
    "ecs_kernel_timing": (_I, [_VP, _I, ctypes.POINTER(_D), ctypes.POINTER(_I), ctypes.POINTER(_D),
                               ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "ecs_box_dims": (_I, [_VP, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "ecs_to_box": (_I, [_VP, _VP, _VP, _I, _VP]),
    "ecs_from_box": (_I, [_VP, _VP, _VP, _I, _VP]),
    "ecs_dealias": (_I, [_VP, _VP, _VP, _I, _VP]),
    "ecs_state_vel": (_I, [_VP, _VP, _VP, _I, _I, _VP]),
    "ecs_lawson_rk4": (_I, [_VP, _VP, _D, _I, _I, _VP]),
    "ecs_objective": (_I, [_VP, ctypes.POINTER(EcsShootCfg), _VP, _VP, _VP, _VP, _VP, _VP,
                           ctypes.POINTER(EcsInfo), _I, _VP]),
    "ecs_loss": (_I, [_VP, ctypes.POINTER(EcsShootCfg), _VP, _VP, _VP, _VP,
                      ctypes.POINTER(EcsInfo), _I, _VP]),
    "ecs_linearize": (_I, [_VP, ctypes.POINTER(EcsShootCfg), _VP, _VP, _VP, _VP, ctypes.POINTER(EcsInfo), _VP]),
    "ecs_jvp": (_I, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _I, _VP]),
    "ecs_integrate": (_I, [_VP, _I, _VP, ctypes.c_double, _I, _I, _VP]),
    "ecs_recurrence": (_I, [_VP, _VP, _I, _VP, _VP]),
    "ecs_linearize_jvp": (_I, [_VP, ctypes.POINTER(EcsShootCfg), _VP, _VP, _VP, _VP, ctypes.POINTER(EcsInfo),
                               _VP, _VP, _VP, _VP, _VP, _VP, _I, _VP]),
    "ecs_vjp": (_I, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _I, _VP]),
    "ecs_arnoldi_mgs": (_I, [_VP, ctypes.c_long, _I, _VP, _VP, ctypes.c_long, _VP]),
    "ecs_arnoldi_mgs_reorth": (_I, [_VP, ctypes.c_long, _I, _VP, _VP, ctypes.c_long, _I, _VP]),
    "ecs_hessenberg_lstsq": (_I, [_VP, _I, _I, _VP, _VP, _VP]),
    "ecs_state_vel_noalloc": (_I, [_I, _D, _D, _D, _D, _VP, _VP, _VP, _I, _I, _VP]),
    "ecs_pool_reset": (_I, [_VP, _VP]),
    "ecs_pool_admit": (_I, [_VP, _I, ctypes.POINTER(EcsShootCfg), _VP, _D, _D, _VP]),
    "ecs_pool_advance": (_I, [_VP, _I, _VP]),
    "ecs_pool_poll": (_I, [_VP, ctypes.POINTER(_I), ctypes.POINTER(_I), _VP]),
    "ecs_pool_retire": (_I, [_VP, _I, _VP, _VP, _VP]),
}

_lib = None
_lock = threading.Lock()


def load(path: str = LIB_PATH):
    """Load the shared library and bind every declared symbol (raises if absent)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise EcsError(6, f"{path} not built; run ecs_mhd_2d_b200.build.build()")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(code, ctx=None):
    if code != 0:
        msg = ""
        if ctx is not None and _lib is not None:
            raw = _lib.ecs_last_error(ctx)
            msg = raw.decode() if raw else ""
        raise EcsError(code, msg)
