"""D2Q9 collisions and streaming (tensorlbm/solver.py)."""

from __future__ import annotations

import torch

from . import _lib, _ops


def collide_bgk(f: torch.Tensor, tau: float) -> torch.Tensor:
    """tensorlbm/solver.py:67."""
    return _ops.collide(9, f, _lib.COLL_BGK, tau)


# solver.py:74 is the same collision with fewer torch kernels
collide_bgk_fused = collide_bgk


def collide_mrt(f: torch.Tensor, tau: float, s_e: float = 1.64, s_eps: float = 1.54, s_q: float = 1.7,
                tau_field: torch.Tensor | None = None) -> torch.Tensor:
    """Lallemand-Luo MRT; tau_field gives a per-cell shear rate.  tensorlbm/solver.py:249."""
    if isinstance(tau, torch.Tensor):
        tau = float(tau.item())
    return _ops.collide(9, f, _lib.COLL_MRT, tau, s_e=s_e, s_eps=s_eps, s_q=s_q, tau_field=tau_field)


def collide_trt(f: torch.Tensor, tau_plus: float, lambda_trt: float = 3.0 / 16.0) -> torch.Tensor:
    """Two-relaxation-time collision, bit-exact.  tensorlbm/solver.py:440."""
    return _ops.collide(9, f, _lib.COLL_TRT, tau_plus, lambda_trt=lambda_trt)


def collide_rlbm(f: torch.Tensor, tau: float) -> torch.Tensor:
    """Regularised BGK (Latt & Chopard 2006), bit-exact.  tensorlbm/solver.py:338."""
    return _ops.collide(9, f, _lib.COLL_RLBM, tau)


def stream(f: torch.Tensor) -> torch.Tensor:
    """Periodic pull streaming.  tensorlbm/solver.py:396."""
    return _ops.stream(9, f)


def correct_mass(f: torch.Tensor, target_mass: float) -> torch.Tensor:
    """tensorlbm/solver.py:420."""
    return _ops.correct_mass(f, target_mass)


__all__ = ["collide_bgk", "collide_bgk_fused", "collide_mrt", "collide_rlbm", "collide_trt", "stream", "correct_mass"]
