"""2-D cavity boundary helpers (tensorlbm/lid_driven_cavity.py:404-473)."""

from __future__ import annotations

import torch

from . import _ops


def make_cavity_wall_mask(ny: int, nx: int, device, include_top: bool = True) -> torch.Tensor:
    """tensorlbm/lid_driven_cavity.py:404."""
    dev = _ops.cuda_device(device)
    mask = torch.zeros((ny, nx), dtype=torch.bool, device=dev)
    mask[0, :] = True
    if include_top:
        mask[-1, :] = True
    mask[:, 0] = True
    mask[:, -1] = True
    return mask


def zou_he_moving_lid(f: torch.Tensor, u_lid: float) -> torch.Tensor:
    """Zou/He lid on the whole top row; returns a new tensor.  tensorlbm/lid_driven_cavity.py:431."""
    return _ops.moving_lid_(9, f.clone(memory_format=torch.contiguous_format), u_lid)


__all__ = ["make_cavity_wall_mask", "zou_he_moving_lid"]
