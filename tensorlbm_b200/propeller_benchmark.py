"""D3Q19 rotating-body wall operators (tensorlbm/propeller_benchmark.py)."""

from __future__ import annotations

import torch

from . import _ops


def rotating_wall_velocity_3d(obstacle_mask: torch.Tensor, cx: float, cy: float, cz: float,
                              omega: float) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """Rigid rotation about the x-axis, float32, shape (nz, ny, nx): ux_w = 0,
    uy_w = -omega (z - cz), uz_w = omega (y - cy).  tensorlbm/propeller_benchmark.py:195."""
    del cx  # the rotation axis is the x-axis through (cy, cz)
    nz, ny, nx = obstacle_mask.shape
    dev = obstacle_mask.device
    zz, yy, xx = torch.meshgrid(torch.arange(nz, device=dev, dtype=torch.float32),
                                torch.arange(ny, device=dev, dtype=torch.float32),
                                torch.arange(nx, device=dev, dtype=torch.float32), indexing="ij")
    return torch.zeros_like(xx), -omega * (zz - cz), omega * (yy - cy)


def moving_wall_bounce_back_3d(f: torch.Tensor, mask: torch.Tensor, ux_w: torch.Tensor, uy_w: torch.Tensor,
                               uz_w: torch.Tensor) -> torch.Tensor:
    """Ladd moving-wall bounce-back for D3Q19 on the masked cells.
    tensorlbm/propeller_benchmark.py:221."""
    return _ops.moving_wall_bounce_back(19, f, mask, ux_w, uy_w, uz_w)
