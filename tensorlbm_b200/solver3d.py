"""D3Q19 collisions and streaming (tensorlbm/solver3d.py)."""

from __future__ import annotations

import torch

from . import _lib, _ops


def collide_bgk3d(f: torch.Tensor, tau: float) -> torch.Tensor:
    """tensorlbm/solver3d.py:100."""
    return _ops.collide(19, f, _lib.COLL_BGK, tau)


def collide_mrt3d(f: torch.Tensor, tau: float, s_e: float = 1.19, s_eps: float = 1.4, s_q: float = 1.2,
                  s_pi: float | None = None) -> torch.Tensor:
    """d'Humieres D3Q19 MRT.  tensorlbm/solver3d.py:107."""
    return _ops.collide(19, f, _lib.COLL_MRT, tau, s_e=s_e, s_eps=s_eps, s_q=s_q, s_pi=s_pi)


collide_mrt3d_low_memory = collide_mrt3d


def collide_trt3d(f: torch.Tensor, tau_plus: float, lambda_trt: float = 3.0 / 16.0) -> torch.Tensor:
    """Two-relaxation-time collision, bit-exact.  tensorlbm/solver3d.py:303."""
    return _ops.collide(19, f, _lib.COLL_TRT, tau_plus, lambda_trt=lambda_trt)


def collide_rlbm3d(f: torch.Tensor, tau: float) -> torch.Tensor:
    """Regularised BGK (Latt & Chopard 2006), bit-exact.  tensorlbm/solver3d.py:342."""
    return _ops.collide(19, f, _lib.COLL_RLBM, tau)


def stream3d(f: torch.Tensor) -> torch.Tensor:
    """Periodic pull streaming.  tensorlbm/solver3d.py:210."""
    return _ops.stream(19, f)


stream3d_roll = stream3d


def correct_mass3d(f: torch.Tensor, target_mass: float) -> torch.Tensor:
    """tensorlbm/solver3d.py:287."""
    return _ops.correct_mass(f, target_mass)


__all__ = ["collide_bgk3d", "collide_mrt3d", "collide_mrt3d_low_memory", "collide_rlbm3d", "collide_trt3d",
           "stream3d", "stream3d_roll", "correct_mass3d"]
