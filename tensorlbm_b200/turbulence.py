"""Smagorinsky-BGK collisions (tensorlbm/turbulence.py)."""

from __future__ import annotations

import torch

from . import _lib, _ops


def collide_smagorinsky_bgk(f: torch.Tensor, tau: float, C_s: float = 0.1) -> torch.Tensor:
    """D2Q9, tensorlbm/turbulence.py:216."""
    return _ops.collide(9, f, _lib.COLL_SMAGORINSKY, tau, c_smag=C_s)


def collide_smagorinsky_bgk3d(f: torch.Tensor, tau: float, C_s: float = 0.1) -> torch.Tensor:
    """D3Q19, tensorlbm/turbulence.py:245."""
    return _ops.collide(19, f, _lib.COLL_SMAGORINSKY, tau, c_smag=C_s)


def collide_smagorinsky_bgk27(f: torch.Tensor, tau: float, C_s: float = 0.1) -> torch.Tensor:
    """D3Q27, tensorlbm/turbulence.py:472."""
    return _ops.collide(27, f, _lib.COLL_SMAGORINSKY, tau, c_smag=C_s)


__all__ = ["collide_smagorinsky_bgk", "collide_smagorinsky_bgk3d", "collide_smagorinsky_bgk27"]
