"""Cascaded central-moment collisions, drop-ins for
``tensorlbm.cascaded_collision`` (cascaded_collision.py:445-576).

The same operator as the reference: central moments of f - feq, second order
split into trace (s_bulk) and deviator (1/tau), orders 3-6 relaxed at their
own rates, back to populations.  The moment transforms run in the fused
form (factorised 1-D passes for D3Q27, straight-line basis sums for D3Q19)
instead of the reference's float32 matrix products, so results agree to
float32 rounding rather than bit for bit.
"""

from __future__ import annotations

import torch

from . import _lib, _ops


def _check(f: torch.Tensor, q: int, tau) -> float:
    if f.ndim != 4 or f.shape[0] != q:
        raise ValueError(f"D3Q{q} populations must have shape ({q}, nz, ny, nx), got {tuple(f.shape)}")
    if isinstance(tau, torch.Tensor):
        if tau.numel() != 1:
            raise NotImplementedError("a per-cell tau is not built for the cascaded collision")
        tau = float(tau.item())
    if tau <= 0.5:
        raise ValueError(f"tau must be > 0.5, got {tau}")
    return float(tau)


def collide_cascaded_d3q19(f: torch.Tensor, tau: float, s_bulk: float = 1.0, s_3: float = 1.0,
                           s_4: float = 1.0) -> torch.Tensor:
    """tensorlbm/cascaded_collision.py:445."""
    tau = _check(f, 19, tau)
    return _ops.collide(19, f, _lib.COLL_CASCADED, tau, omega_b=s_bulk, omega_odd=s_3, omega_even=s_4)


def collide_cascaded_d3q27(f: torch.Tensor, tau: float, s_bulk: float = 1.0, s_3: float = 1.0, s_4: float = 1.0,
                           s_5: float | None = None, s_6: float | None = None) -> torch.Tensor:
    """tensorlbm/cascaded_collision.py:512 (s_5, s_6 default to s_4)."""
    tau = _check(f, 27, tau)
    return _ops.collide(27, f, _lib.COLL_CASCADED, tau, omega_b=s_bulk, omega_odd=s_3, omega_even=s_4,
                        cm_s5=s_4 if s_5 is None else s_5, cm_s6=s_4 if s_6 is None else s_6)
