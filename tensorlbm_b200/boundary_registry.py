"""Missing-direction mask and link list (tensorlbm/boundary_registry.py:488-660)."""

from __future__ import annotations

from collections.abc import Sequence

import torch

from . import _ops

_Q = {"D2Q9": 9, "D3Q19": 19, "D3Q27": 27}


def _periodic_bits(periodic) -> int:
    """(z, y, x) sequence, dict with x/y/z keys, or one bool -> bit mask (1=x, 2=y, 4=z).
    Same conventions as tensorlbm/boundary_registry.py:455-485."""
    if isinstance(periodic, bool):
        value = {"z": periodic, "y": periodic, "x": periodic}
    elif isinstance(periodic, dict):
        unknown = set(periodic) - {"x", "y", "z"}
        if unknown:
            raise ValueError(f"unknown periodic axes {sorted(unknown)}")
        value = {k: bool(periodic.get(k, False)) for k in ("x", "y", "z")}
    else:
        seq = tuple(bool(p) for p in periodic)
        if len(seq) != 3:
            raise ValueError("periodic sequence must have 3 entries (z, y, x)")
        value = {"z": seq[0], "y": seq[1], "x": seq[2]}
    return (1 if value["x"] else 0) | (2 if value["y"] else 0) | (4 if value["z"] else 0)


def derive_missing_mask(shape: Sequence[int], *, solid_mask: torch.Tensor | None = None,
                        periodic=False, lattice: str = "D3Q19", device=None) -> torch.Tensor:
    """missing[q, z, y, x] = pull source x - c_q is solid or outside a non-periodic face.
    Returns bool (Q, nz, ny, nx).  tensorlbm/boundary_registry.py:488."""
    if len(shape) != 3 or any(int(n) <= 0 for n in shape):
        raise ValueError(f"shape must be three positive sizes (nz, ny, nx), got {tuple(shape)}")
    nz, ny, nx = (int(n) for n in shape)
    if lattice not in ("D3Q19", "D3Q27"):
        raise ValueError(f"unsupported lattice {lattice!r}")
    if solid_mask is not None:
        if tuple(solid_mask.shape) != (nz, ny, nx) or solid_mask.dtype != torch.bool:
            raise ValueError(f"solid_mask must be boolean with shape {(nz, ny, nx)}, got "
                             f"{tuple(solid_mask.shape)}/{solid_mask.dtype}")
        if device is None:
            device = solid_mask.device
    if device is None:
        device = "cuda"
    return _ops.missing_mask(_Q[lattice], (nx, ny, nz), solid_mask, _periodic_bits(periodic), device)


def link_list(missing: torch.Tensor) -> torch.Tensor:
    """(n_links, ndim) int64 indices of the True entries in row-major order, the
    same as torch.nonzero(missing) (q, z, y, x)."""
    flat = _ops.link_list(missing)
    out = torch.empty((flat.numel(), missing.ndim), dtype=torch.int64, device=flat.device)
    rem = flat
    for axis in range(missing.ndim - 1, -1, -1):
        n = missing.shape[axis]
        out[:, axis] = rem % n
        rem = rem // n
    return out


__all__ = ["derive_missing_mask", "link_list"]
