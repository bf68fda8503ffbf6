"""CPU oracle for the ecs_mhd_2d_b200 hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, on the CPU and in FP64, the reference algorithm of
mgolden30/ECS_MHD_2D for the pseudo-spectral 2D MHD right-hand side, the
steppers of every shooting mode (RK4, Lawson-RK4, Lawson-RK6, TDRK4 and the
adaptive Lawson-RK4(3)), the symmetry operations, the RPO
shooting objective/loss and their tangent (JVP) and adjoint (VJP).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it, and only as the checker (or as the timed CPU
baseline).  The product path (``ecs_mhd_2d_b200``) never imports it and has no
CPU fallback.

Parity status: pinned by closure of the reference's converged solutions
(``solutions/Re40/*.npz``, ``solutions/Re50/*.npz``, stored as fixtures in
``tests/golden/``) under the restated Lawson-RK4 integrator, and by the
reference's own self-check properties (RK4 order, JVP/VJP dot-product
adjointness, symmetry equivariance).  The reference's JAX code cannot be run in
this container (jax is not installed), so no value-level golden output of the
reference exists; FFT arithmetic is pocketfft (numpy/torch) instead of
XLA/DUCC/cuFFT.
"""

from .mhd_oracle import (  # noqa: F401
    NUMPY, TORCH, Backend,
    construct_domain, dissipation, state_vel, state_vel_jvp,
    rk4, lawson_rk4, lawson_rk6, tdrk4, lawson_rk43,
    shift_x, shift_reflect, rot180,
    mismatch_RPO, loss_RPO, phase_conditions, objective_RPO,
    make_param_dict, ravel_dict, unravel_dict, change_resolution,
    compute_observables, laminar_flow,
    gmres, line_search_unravel,
)
