"""Momentum-exchange forces on stationary obstacles (tensorlbm/obstacles.py)."""

from __future__ import annotations

import torch

from . import _ops


def compute_obstacle_forces_3d(f: torch.Tensor, obstacle_mask: torch.Tensor):
    """(fx, fy, fz) = 2 sum_solid sum_q c_q f_q, float64 accumulation.  tensorlbm/obstacles.py:91."""
    out = _ops.obstacle_force(19, f, obstacle_mask)
    return out[0], out[1], out[2]


def compute_obstacle_forces_27(f: torch.Tensor, obstacle_mask: torch.Tensor):
    """tensorlbm/obstacles.py:197."""
    out = _ops.obstacle_force(27, f, obstacle_mask)
    return out[0], out[1], out[2]


__all__ = ["compute_obstacle_forces_3d", "compute_obstacle_forces_27"]
