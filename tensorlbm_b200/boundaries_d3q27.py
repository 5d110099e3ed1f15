"""D3Q27 boundaries (tensorlbm/boundaries_d3q27.py)."""

from __future__ import annotations

import torch

from . import _ops
from .boundaries3d import make_channel_wall_mask_3d as make_channel_wall_mask_27  # same planes (:243)


def bounce_back_cells_27(f: torch.Tensor, mask: torch.Tensor) -> torch.Tensor:
    """tensorlbm/boundaries_d3q27.py:45."""
    return _ops.bounce_back(27, f, mask)


def zou_he_inlet_velocity_27(f: torch.Tensor, u_in: float, uy_in: float = 0.0, uz_in: float = 0.0) -> torch.Tensor:
    """Returns a new tensor (the D3Q27 reference clones).  tensorlbm/boundaries_d3q27.py:107."""
    return _ops.zou_he_inlet_(27, f.clone(memory_format=torch.contiguous_format), u_in, uy_in, uz_in)


def zou_he_outlet_pressure_27(f: torch.Tensor, rho_out: float = 1.0) -> torch.Tensor:
    """tensorlbm/boundaries_d3q27.py:179."""
    return _ops.zou_he_outlet_(27, f.clone(memory_format=torch.contiguous_format), rho_out)


def apply_zou_he_channel_boundaries_27(f, u_in, wall_mask, obstacle_mask):
    """tensorlbm/boundaries_d3q27.py:272."""
    f = zou_he_inlet_velocity_27(f, u_in)
    f = zou_he_outlet_pressure_27(f)
    f = bounce_back_cells_27(f, wall_mask)
    return bounce_back_cells_27(f, obstacle_mask)


def far_field_bc_27(f: torch.Tensor, u_in: float, obstacle_mask: torch.Tensor | None = None, uy: float = 0.0,
                    uz: float = 0.0) -> torch.Tensor:
    """Free-stream far field on the inlet and all four lateral planes,
    zero-gradient outlet, then bounce-back in the obstacle; returns a new
    tensor.  tensorlbm/boundaries_d3q27.py:63."""
    out = _ops.far_field_(27, f.clone(memory_format=torch.contiguous_format), u_in, uy, uz, True)
    return out if obstacle_mask is None else _ops.bounce_back(27, out, obstacle_mask)


__all__ = ["bounce_back_cells_27", "zou_he_inlet_velocity_27", "zou_he_outlet_pressure_27",
           "make_channel_wall_mask_27", "apply_zou_he_channel_boundaries_27", "far_field_bc_27"]
