"""tensorlbm.bfl_d3q19 drop-in (stationary-wall Bouzidi update with force); see :mod:`tensorlbm_b200.bfl`."""

from .bfl import bouzidi_bounce_back_d3q19  # noqa: F401
