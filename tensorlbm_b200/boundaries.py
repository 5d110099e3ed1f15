"""D2Q9 boundaries (tensorlbm/boundaries.py)."""

from __future__ import annotations

import torch

from . import _ops


def cylinder_mask(nx: int, ny: int, cx: float, cy: float, radius: float, device) -> torch.Tensor:
    """(x-cx)^2 + (y-cy)^2 <= r^2 in float32, shape (ny, nx).  tensorlbm/boundaries.py:8."""
    return _ops.cylinder_mask(nx, ny, cx, cy, radius, device)


def make_channel_wall_mask(ny: int, nx: int, obstacle_mask: torch.Tensor, device) -> torch.Tensor:
    """Top/bottom rows minus obstacle cells.  tensorlbm/boundaries.py:25."""
    dev = _ops.cuda_device(device)
    wall = torch.zeros((ny, nx), dtype=torch.bool, device=dev)
    wall[0, :] = True
    wall[-1, :] = True
    wall[obstacle_mask.to(dev)] = False
    return wall


def bounce_back_cells(f: torch.Tensor, mask: torch.Tensor) -> torch.Tensor:
    """where(mask, f[opp], f).  tensorlbm/boundaries.py:39."""
    return _ops.bounce_back(9, f, mask)


def zou_he_inlet_velocity(f: torch.Tensor, u_in, uy_in=0.0) -> torch.Tensor:
    """Zou/He velocity inlet at x = 0 (scalar or per-row profile); returns a new tensor.
    tensorlbm/boundaries.py:50."""
    return _ops.zou_he_inlet_(9, f.clone(memory_format=torch.contiguous_format), u_in, uy_in)


def zou_he_outlet_pressure(f: torch.Tensor, rho_out: float = 1.0) -> torch.Tensor:
    """Zou/He pressure outlet at x = nx-1; returns a new tensor.  tensorlbm/boundaries.py:102."""
    return _ops.zou_he_outlet_(9, f.clone(memory_format=torch.contiguous_format), rho_out)


def compute_obstacle_forces(f: torch.Tensor, obstacle_mask: torch.Tensor):
    """Ladd momentum exchange, accumulated in float64: (fx, fy) as 0-dim float64 tensors.
    tensorlbm/boundaries.py:162."""
    out = _ops.obstacle_force(9, f, obstacle_mask)
    return out[0], out[1]


def apply_zou_he_channel_boundaries(f, u_in, wall_mask, obstacle_mask):
    """Zou/He inlet, outlet, then bounce-back on walls and obstacle.  tensorlbm/boundaries.py:360."""
    f = zou_he_inlet_velocity(f, u_in)
    f = zou_he_outlet_pressure(f)
    f = bounce_back_cells(f, wall_mask)
    return bounce_back_cells(f, obstacle_mask)


def far_field_bc_2d(f: torch.Tensor, u_in: float, obstacle_mask: torch.Tensor | None = None) -> torch.Tensor:
    """Free-stream far field: feq(1, u_in, 0) on the inlet and both lateral
    rows, zero-gradient outlet, then bounce-back in the obstacle; returns a new
    tensor.  tensorlbm/boundaries.py:199."""
    out = _ops.far_field_(9, f.clone(memory_format=torch.contiguous_format), u_in, 0.0, 0.0, False)
    return out if obstacle_mask is None else _ops.bounce_back(9, out, obstacle_mask)


def make_sponge_strength(ny: int, nx: int, x0: int, width: int, power: float = 2.0, device=None) -> torch.Tensor:
    """Absorbing-layer strength sigma(x) = clamp((x - x0) / width, 0, 1) ** power
    (float32, shape (ny, nx)); with collide_mrt's tau_field as
    tau (1 + alpha sigma).  tensorlbm/boundaries.py:388."""
    x = torch.arange(nx, device=device, dtype=torch.float32)
    ramp = ((x - x0) / width).clamp(min=0.0, max=1.0) ** power
    return ramp.view(1, nx).expand(ny, nx)


__all__ = ["cylinder_mask", "make_channel_wall_mask", "bounce_back_cells", "zou_he_inlet_velocity",
           "zou_he_outlet_pressure", "compute_obstacle_forces", "apply_zou_he_channel_boundaries", "far_field_bc_2d",
           "make_sponge_strength"]
