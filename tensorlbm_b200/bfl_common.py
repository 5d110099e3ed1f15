"""tensorlbm.bfl_common drop-ins (sphere links, BFL link update); see :mod:`tensorlbm_b200.bfl`."""

from .bfl import bfl_bounce_back_common, compute_q_sphere_common  # noqa: F401
