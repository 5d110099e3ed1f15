"""tensorlbm.interpolated_bc_common drop-in (D3Q27 sphere links); see :mod:`tensorlbm_b200.bfl`."""

from .bfl import compute_q_sphere_27  # noqa: F401
