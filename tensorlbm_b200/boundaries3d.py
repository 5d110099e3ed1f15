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


def far_field_bc_3d(f: torch.Tensor, u_in: float, obstacle_mask: torch.Tensor | None = None, uy: float = 0.0,
                    uz: float = 0.0, bc_config: dict | None = None) -> torch.Tensor:
    """Free-stream far field: feq(1, (u_in, uy, uz)) on the inlet and the lateral
    planes, zero-gradient outlet, then bounce-back in the obstacle; returns a
    new tensor.  bc_config selects the lateral planes like the reference:
    far-field y planes and z planes each as a pair ("y-" with "y+", "z-" with
    "z+"); a periodic inlet or outlet is not built.  tensorlbm/boundaries3d.py:446."""
    z_faces = True
    if bc_config is not None:
        ff = set(bc_config.get("far_field_faces", []))
        periodic = set(bc_config.get("periodic_faces", []))
        y_planes = {"y-", "y+"} <= ff and not ({"y-", "y+"} & periodic)
        z_pair = ff & {"z-", "z+"}
        if {"x-", "x+"} & periodic or not y_planes or z_pair not in (set(), {"z-", "z+"}) or (z_pair & periodic):
            raise NotImplementedError("far_field_bc_3d: the far field is built for both y planes, optionally both "
                                      "z planes, with the inlet and the outlet")
        z_faces = bool(z_pair)
    out = _ops.far_field_(19, f.clone(memory_format=torch.contiguous_format), u_in, uy, uz, z_faces)
    return out if obstacle_mask is None else _ops.bounce_back(19, out, obstacle_mask)


__all__ = ["sphere_mask", "make_channel_wall_mask_3d", "bounce_back_cells_3d", "zou_he_inlet_velocity_3d",
           "zou_he_outlet_pressure_3d", "zou_he_moving_lid_3d", "apply_zou_he_channel_boundaries_3d",
           "far_field_bc_3d"]
