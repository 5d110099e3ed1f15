"""D3Q19 lattice: tables, equilibrium and moments (tensorlbm/d3q19.py:1-212)."""

from __future__ import annotations

import torch

from . import _ops
from . import lattice as _lat
from ._tables import tables

C, W, W_EXACT64, OPPOSITE = tables(_lat.D3Q19)
WEIGHT_PRECISION_SCHEME = "rational_binary64_cast_to_runtime_dtype_v1"


def equilibrium3d(rho, ux, uy, uz, device=None, *, out: torch.Tensor | None = None) -> torch.Tensor:
    """D3Q19 f_eq, fields (nz, ny, nx) -> (19, nz, ny, nx).  tensorlbm/d3q19.py:83."""
    return _ops.equilibrium(19, rho, ux, uy, uz, out=out)


def macroscopic3d(f: torch.Tensor, device=None):
    """(rho, ux, uy, uz) from f (19, nz, ny, nx).  tensorlbm/d3q19.py:165."""
    return _ops.macroscopic(19, f)


# the low-memory variants of the reference (d3q19.py:128, :189) exist to cap
# torch temporaries; the kernels never materialise any, so they are the same call
equilibrium3d_low_memory = equilibrium3d


def macroscopic3d_low_memory(f: torch.Tensor):
    if not isinstance(f, torch.Tensor) or f.ndim != 4 or f.shape[0] != 19:
        raise ValueError("f must have shape (19,nz,ny,nx)")
    return _ops.macroscopic(19, f)


__all__ = ["C", "W", "W_EXACT64", "OPPOSITE", "equilibrium3d", "macroscopic3d",
           "equilibrium3d_low_memory", "macroscopic3d_low_memory"]
