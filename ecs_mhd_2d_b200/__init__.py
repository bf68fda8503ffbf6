"""B200-native (sm_100a) hot path of mgolden30/ECS_MHD_2D.

Pseudo-spectral 2D incompressible MHD right-hand side, Lawson-RK4 and adaptive
Lawson-RK4(3) steppers, RPO shooting objective/loss and their tangent and
adjoint, behind a C-ABI (include/ecs_mhd.h) with a Python dict API mirroring the
reference's jax_scripts/lib modules.
"""

from .mhd import construct_domain, dissipation, make_param_dict, state_vel  # noqa: F401
from .timestepping import lawson_rk4, lawson_rk6, rk4, tdrk4, integrate  # noqa: F401
from .loss_functions import objective_RPO, loss_RPO, dealias  # noqa: F401
from .synthetic import initial_condition, unit_tangents  # noqa: F401
from .autodiff import (Objective, compile_objective_and_Jacobian, vjp, loss_and_grad,  # noqa: F401
                       loss_rpo_autograd, jvp_multi, loss_grad_multi)

__version__ = "0.1.0"
