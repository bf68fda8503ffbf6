"""ecs_state_vel_noalloc: the allocation-free state_vel for callers that cannot
allocate device memory (e.g. inside a JAX/XLA process that owns the GPU's memory).

Called through the C ABI and checked against the regular entry point
ecs_state_vel (which allocates its workspace in a context) within the RHS
tolerance of the parity tests (1e-12 relative L2), on two calls in a row with
different sizes, so the second call also shows that contents left in the
shared scratch array by the first call do not leak into the result.  This file
sorts last so that a run stopping at the first failure has run everything else.
"""
import ctypes

import numpy as np
import pytest
import torch

import ecs_mhd_2d_b200 as E
from ecs_mhd_2d_b200 import _lib
from ecs_mhd_2d_b200.synthetic import initial_condition
from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL_RHS = 1e-12


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_state_vel_matches_state_vel_twice(cuda):
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    calls = [(128, 3, True, 0, 1 / 40, 1 / 45), (64, 4, False, 7, 1 / 50, 1 / 50)]
    for n, B, diss, seed, nu, eta in calls:
        pd = E.make_param_dict(n, nu, eta, b0=(0.0, 0.1), forcing="kolmogorov+")
        u = np.stack([initial_condition(seed + b, n) for b in range(B)])
        f = torch.as_tensor(np.fft.rfft2(u), device="cuda").contiguous()
        want = E.state_vel(f, pd, diss)
        forcing = pd["forcing"].to(device="cuda", dtype=torch.float64).contiguous()
        out = torch.full_like(f, float("nan"))
        rc = lib.ecs_state_vel_noalloc(n, nu, eta, 0.0, 0.1, _p(forcing), _p(f), _p(out), B, int(diss), stream)
        torch.cuda.synchronize()
        assert rc == 0, _lib.STATUS.get(rc, rc)
        assert rel_l2(out.cpu().numpy(), want.cpu().numpy()) < TOL_RHS


def test_noalloc_allocates_no_device_memory(cuda):
    """After a first call per size (the one-time set-up, and the lazy loading of
    the kernels), further calls leave the device's free memory unchanged: the
    entry point takes nothing from the device's allocator.  Every tensor is
    created before the first measurement."""
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    cases = []
    for n, B in ((128, 4), (64, 2)):
        pd = E.make_param_dict(n, 1 / 40, 1 / 40, b0=(0.0, 0.1), forcing="kolmogorov+")
        f = torch.as_tensor(np.fft.rfft2(np.stack([initial_condition(b, n) for b in range(B)])), device="cuda")
        forcing = pd["forcing"].to(device="cuda", dtype=torch.float64).contiguous()
        cases.append((n, B, f.contiguous(), forcing, torch.empty_like(f)))

    def call(i, diss):
        n, B, f, forcing, out = cases[i]
        return lib.ecs_state_vel_noalloc(n, 1 / 40, 1 / 40, 0.0, 0.1, _p(forcing), _p(f), _p(out), B, diss, stream)

    for i in range(2):
        for diss in (0, 1):
            assert call(i, diss) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for it in range(6):
        assert call(it % 2, (it // 2) % 2) == 0
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0, it


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    lib = _lib.load()
    f = torch.zeros((5, 2, 128, 65), dtype=torch.complex128, device="cuda")
    forcing = torch.zeros((128, 128), dtype=torch.float64, device="cuda")
    assert lib.ecs_state_vel_noalloc(128, 0.02, 0.02, 0.0, 0.1, _p(forcing), _p(f), _p(f), 5, 0, None) == 7
    assert lib.ecs_state_vel_noalloc(256, 0.02, 0.02, 0.0, 0.1, _p(forcing), _p(f), _p(f), 1, 0, None) == 7
