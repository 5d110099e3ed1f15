"""Cumulant-family collisions (tensorlbm/cumulant.py)."""

from __future__ import annotations

import math

import torch

from . import _lib, _ops


def collide_cumulant_d3q27(f: torch.Tensor, tau: float, omega_b: float = 1.0, omega_odd: float = 1.0,
                           omega_even: float = 1.0, C_s: float = 0.0) -> torch.Tensor:
    """Legacy D3Q27 pseudo-cumulant collision on f_neq.  tensorlbm/cumulant.py:935.

    The domain-averaged Smagorinsky option (C_s > 0) needs a global mean of
    tau_eff before the collision; it is not built (NotImplementedError)."""
    if C_s > 0:
        raise NotImplementedError("collide_cumulant_d3q27: domain-averaged Smagorinsky (C_s > 0) is not built")
    return _ops.collide(27, f, _lib.COLL_CUMULANT, tau, omega_b=omega_b, omega_odd=omega_odd,
                        omega_even=omega_even)


def collide_cumulant_geier_d3q27(f: torch.Tensor, tau: float, omega_b: float = 1.0, omega_odd: float = 1.0,
                                 omega_even: float = 1.0, C_s: float = 0.0) -> torch.Tensor:
    """Geier-2015 D3Q27 cumulant collision.  tensorlbm/cumulant.py:1050."""
    if C_s > 0:
        raise NotImplementedError("collide_cumulant_geier_d3q27: domain-averaged Smagorinsky (C_s > 0) is not built")
    return _ops.collide(27, f, _lib.COLL_CUMULANT_GEIER, tau, omega_b=omega_b, omega_odd=omega_odd,
                        omega_even=omega_even)


def collide_cumulant_d3q19(f: torch.Tensor, tau: float, omega_b: float = 1.0, omega_odd: float = 1.0,
                           omega_even: float = 1.0, C_s: float = 0.0, C_w: float = 0.0, C_v: float = 0.0,
                           solid_mask: torch.Tensor | None = None,
                           wall_velocity: tuple[float, float, float] = (0.0, 0.0, 0.0)) -> torch.Tensor:
    """Hermite-regularised D3Q19 collision with local Smagorinsky.  tensorlbm/cumulant.py:1159.

    Argument checks follow the reference; the gradient closures (WALE C_w,
    Vreman C_v) are not built."""
    if min(C_s, C_w, C_v) < 0.0:
        raise ValueError("SGS coefficients must be non-negative")
    if sum(v > 0.0 for v in (C_s, C_w, C_v)) > 1:
        raise ValueError("only one SGS model may be active")
    if len(wall_velocity) != 3 or not all(math.isfinite(v) for v in wall_velocity):
        raise ValueError("wall_velocity must contain three finite values")
    if solid_mask is not None and (solid_mask.shape != f.shape[1:] or solid_mask.dtype is not torch.bool
                                   or solid_mask.device != f.device):
        raise ValueError("solid_mask must be bool with the population spatial shape")
    if C_w > 0.0 or C_v > 0.0:
        raise NotImplementedError("collide_cumulant_d3q19: WALE / Vreman closures are not built")
    return _ops.collide(19, f, _lib.COLL_CUMULANT_D3Q19, tau, omega_b=omega_b, omega_odd=omega_odd,
                        omega_even=omega_even, c_smag=C_s)


__all__ = ["collide_cumulant_d3q27", "collide_cumulant_geier_d3q27", "collide_cumulant_d3q19"]
