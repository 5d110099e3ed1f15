"""D3Q19 boundaries (tensorlbm/boundaries3d.py)."""

from __future__ import annotations

import torch

from . import _ops


def sphere_mask(nx: int, ny: int, nz: int, cx: float, cy: float, cz: float, radius: float, device) -> torch.Tensor:
    """(x-cx)^2 + (y-cy)^2 + (z-cz)^2 <= r^2 in float32, shape (nz, ny, nx).
    tensorlbm/boundaries3d.py:29."""
    return _ops.sphere_mask(nx, ny, nz, cx, cy, cz, radius, device)


def make_channel_wall_mask_3d(nz: int, ny: int, nx: int, obstacle_mask: torch.Tensor, device) -> torch.Tensor:
    """y = 0, ny-1 and z = 0, nz-1 planes minus obstacle cells.  tensorlbm/boundaries3d.py:52."""
    dev = _ops.cuda_device(device)
    wall = torch.zeros((nz, ny, nx), dtype=torch.bool, device=dev)
    wall[:, 0, :] = True
    wall[:, -1, :] = True
    wall[0, :, :] = True
    wall[-1, :, :] = True
    wall[obstacle_mask.to(dev)] = False
    return wall


def bounce_back_cells_3d(f: torch.Tensor, mask: torch.Tensor, f_pre: torch.Tensor | None = None) -> torch.Tensor:
    """where(mask, f[opp], f); f_pre accepted and ignored.  tensorlbm/boundaries3d.py:112."""
    del f_pre
    return _ops.bounce_back(19, f, mask)


def zou_he_inlet_velocity_3d(f: torch.Tensor, u_in: float, uy_in: float = 0.0, uz_in: float = 0.0) -> torch.Tensor:
    """Zou/He velocity inlet at x = 0.  Like the reference it writes into f and
    returns it (tensorlbm/boundaries3d.py:205-266)."""
    if not f.is_contiguous():
        return _ops.zou_he_inlet_(19, f.contiguous(), u_in, uy_in, uz_in)
    return _ops.zou_he_inlet_(19, f, u_in, uy_in, uz_in)


def zou_he_outlet_pressure_3d(f: torch.Tensor, rho_out: float = 1.0) -> torch.Tensor:
    """Zou/He pressure outlet at x = nx-1, in place like tensorlbm/boundaries3d.py:269-321."""
    if not f.is_contiguous():
        return _ops.zou_he_outlet_(19, f.contiguous(), rho_out)
    return _ops.zou_he_outlet_(19, f, rho_out)


def zou_he_moving_lid_3d(f: torch.Tensor, u_lid: float, uy_lid: float = 0.0, uz_lid: float = 0.0) -> torch.Tensor:
    """Zou/He moving lid on the whole y = ny-1 plane; returns a new tensor.
    tensorlbm/boundaries3d.py:324."""
    if uy_lid != 0.0 or uz_lid != 0.0:
        raise NotImplementedError(
            "zou_he_moving_lid_3d currently supports uy=uz=0 (the Ghia cavity case); general uy/uz would "
            "need the (1±uy) density factor and mixed diagonal pairs."
        )
    return _ops.moving_lid_(19, f.clone(memory_format=torch.contiguous_format), u_lid)


def apply_zou_he_channel_boundaries_3d(f, u_in, wall_mask, obstacle_mask):
    """tensorlbm/boundaries3d.py:707."""
    f = zou_he_inlet_velocity_3d(f, u_in)
    f = zou_he_outlet_pressure_3d(f)
    f = bounce_back_cells_3d(f, wall_mask)
    return bounce_back_cells_3d(f, obstacle_mask)


__all__ = ["sphere_mask", "make_channel_wall_mask_3d", "bounce_back_cells_3d", "zou_he_inlet_velocity_3d",
           "zou_he_outlet_pressure_3d", "zou_he_moving_lid_3d", "apply_zou_he_channel_boundaries_3d"]
