"""D2Q9 lattice: tables, equilibrium and moments (tensorlbm/d2q9.py:1-74)."""

from __future__ import annotations

import torch

from . import _ops
from . import lattice as _lat
from ._tables import tables

C, W, _W64, OPPOSITE = tables(_lat.D2Q9)


def equilibrium(rho: torch.Tensor, ux: torch.Tensor, uy: torch.Tensor, device=None) -> torch.Tensor:
    """D2Q9 f_eq for (rho, ux, uy) of shape (ny, nx) -> (9, ny, nx).  tensorlbm/d2q9.py:39."""
    return _ops.equilibrium(9, rho, ux, uy)


def macroscopic(f: torch.Tensor, device=None):
    """(rho, ux, uy) from f of shape (9, ny, nx).  tensorlbm/d2q9.py:61."""
    return _ops.macroscopic(9, f)


__all__ = ["C", "W", "OPPOSITE", "equilibrium", "macroscopic"]
