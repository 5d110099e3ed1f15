"""D2Q9 rotating-cylinder wall operators (tensorlbm/rotating_cylinder.py)."""

from __future__ import annotations

import torch

from . import _ops


def rotating_wall_velocity(obstacle_mask: torch.Tensor, cx: float, cy: float,
                           omega: float) -> tuple[torch.Tensor, torch.Tensor]:
    """Rigid rotation u_w = omega x r on every cell, float32, shape (ny, nx):
    ux_w = -omega (y - cy), uy_w = omega (x - cx).  tensorlbm/rotating_cylinder.py:112."""
    ny, nx = obstacle_mask.shape
    dev = obstacle_mask.device
    yy, xx = torch.meshgrid(torch.arange(ny, device=dev, dtype=torch.float32),
                            torch.arange(nx, device=dev, dtype=torch.float32), indexing="ij")
    return -omega * (yy - cy), omega * (xx - cx)


def moving_wall_bounce_back(f: torch.Tensor, mask: torch.Tensor, ux_w: torch.Tensor,
                            uy_w: torch.Tensor) -> torch.Tensor:
    """Ladd moving-wall bounce-back on the masked cells: bounce_back(f) +
    2 w_i rho (c_i . u_w) * 3 with rho = sum_i f_i; other cells unchanged.
    tensorlbm/rotating_cylinder.py:140."""
    return _ops.moving_wall_bounce_back(9, f, mask, ux_w, uy_w)
