"""Curved walls: Bouzidi-Firdaouss-Lallemand (BFL) interpolated bounce-back.

Drop-ins for TensorLBM's ``bfl_common.compute_q_sphere_common``,
``interpolated_bc_common.compute_q_sphere_27``,
``bfl_common.bfl_bounce_back_common`` and ``bfl_d3q19.bouzidi_bounce_back_d3q19``
(stationary walls), plus the link tables that put the same update inside the
fused step (``LBMSolver(..., curved_wall=...)``): the curved obstacle then costs
no extra pass, and its force is the BFL ledger of ``bfl_d3q19.py:339-377``
accumulated in float64.
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib, _ops

_Q = {"D3Q19": 19, "D3Q27": 27}


def _lattice_q(lattice: str) -> int:
    q = _Q.get(str(lattice).upper())
    if q is None:
        raise ValueError(f"Unsupported lattice {lattice!r}; supported: {sorted(_Q)}")
    return q


def sphere_links(nx: int, ny: int, nz: int, cx: float, cy: float, cz: float, radius: float, device=None, *,
                 lattice: str = "D3Q19") -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """``(fluid_boundary_mask, q_field, solid)`` of a sphere: the links (x, d)
    from a fluid cell into the sphere, their wall fractions (float32, 0.5 off
    the links) and the solid cells, all by the float64 tests of
    ``bfl_common.py:384-477``."""
    q = _lattice_q(lattice)
    dev = _ops.cuda_device(device)
    mask = torch.empty((q, nz, ny, nx), dtype=torch.uint8, device=dev)
    qf = torch.empty((q, nz, ny, nx), dtype=torch.float32, device=dev)
    solid = torch.empty((nz, ny, nx), dtype=torch.uint8, device=dev)
    st = _lib.load().tlbm_sphere_links(q, int(nx), int(ny), int(nz), float(cx), float(cy), float(cz), float(radius),
                                       mask.data_ptr(), qf.data_ptr(), solid.data_ptr(), _lib.stream_of(dev))
    _lib.check(st, "sphere_links")
    return mask.bool(), qf, solid.bool()


def compute_q_sphere_common(nx: int, ny: int, nz: int, cx: float, cy: float, cz: float, radius: float,
                            device, *, lattice: str = "D3Q19") -> tuple[torch.Tensor, torch.Tensor]:
    """tensorlbm/bfl_common.py:384 (bit-identical mask and float32 q)."""
    mask, qf, _ = sphere_links(nx, ny, nz, cx, cy, cz, radius, device, lattice=lattice)
    return mask, qf


def compute_q_sphere_27(nx: int, ny: int, nz: int, cx: float, cy: float, cz: float, radius: float,
                        device) -> tuple[torch.Tensor, torch.Tensor]:
    """tensorlbm/interpolated_bc_common.py:136."""
    return compute_q_sphere_common(nx, ny, nz, cx, cy, cz, radius, device, lattice="D3Q27")


def _bfl(f, f_prev, mask, q_field, lattice, force: torch.Tensor | None) -> torch.Tensor:
    q = _lattice_q(lattice)
    dev = _lib.require_cuda(f, f_prev, mask, q_field)
    if f.shape[0] != q:
        raise ValueError(f"f has {f.shape[0]} directions but lattice {lattice!r} expects {q}")
    for name, t in (("f_prev", f_prev), ("fluid_boundary_mask", mask), ("q_field", q_field)):
        if tuple(t.shape) != tuple(f.shape):
            raise ValueError(f"{name} shape {tuple(t.shape)} does not match f {tuple(f.shape)}")
    if f_prev.dtype != f.dtype or f.dtype not in (torch.float32, torch.float64):
        raise ValueError("f and f_prev must share a float32 or float64 dtype")
    f, f_prev = f.contiguous(), f_prev.contiguous()
    m = mask.to(torch.uint8).contiguous()
    qf = q_field.to(torch.float32).contiguous()
    out = torch.empty_like(f)
    nz, ny, nx = f.shape[1:]
    d = _ops.make_desc(q, (nx, ny, nz), _lib.real_dtype(f), _lib.COLL_NONE, 1.0)
    st = _lib.load().tlbm_bfl_bounce_back(ctypes.byref(d), f.data_ptr(), f_prev.data_ptr(), m.data_ptr(),
                                          qf.data_ptr(), out.data_ptr(), _lib.ptr(force), _lib.stream_of(dev))
    _lib.check(st, "bfl_bounce_back")
    return out


def bfl_bounce_back_common(f: torch.Tensor, f_prev: torch.Tensor, fluid_boundary_mask: torch.Tensor,
                           q_field: torch.Tensor, *, lattice: str = "D3Q19",
                           wall_correction: torch.Tensor | None = None) -> torch.Tensor:
    """tensorlbm/bfl_common.py:106 (stationary walls; bit-identical)."""
    if wall_correction is not None:
        raise NotImplementedError("the moving-wall BFL correction is not built; stationary walls only")
    return _bfl(f, f_prev, fluid_boundary_mask, q_field, lattice, None)


def bouzidi_bounce_back_d3q19(f: torch.Tensor, f_prev: torch.Tensor, fluid_boundary_mask: torch.Tensor,
                              q_field: torch.Tensor, *, wall_velocity=None, wall_density=None,
                              boundary_fraction=None, return_force: bool = False, force_frame: str = "laboratory",
                              force_normals=None, return_force_decomposition: bool = False):
    """tensorlbm/bfl_d3q19.py:195 for a stationary, fully inserted wall:
    the populations of ``bfl_bounce_back_common`` and, with ``return_force``,
    the laboratory-frame ledger sum c_d (P_d + value) (accumulated in float64,
    returned as three 0-dim tensors of f's dtype)."""
    if force_frame not in ("laboratory", "wall"):
        raise ValueError(f"force_frame must be 'laboratory' or 'wall', got {force_frame!r}")
    if wall_velocity is not None and wall_density is None:
        raise ValueError("wall_velocity requires wall_density for the moving-wall correction")
    if return_force_decomposition and not return_force:
        raise ValueError("return_force_decomposition requires return_force=True")
    if wall_velocity is not None or force_frame != "laboratory" or return_force_decomposition or \
            (boundary_fraction is not None and not (isinstance(boundary_fraction, (int, float))
                                                    and float(boundary_fraction) == 1.0)):
        raise NotImplementedError("moving walls, partial insertion, the wall frame and the force "
                                  "decomposition are not built; stationary walls in the laboratory frame only")
    force = torch.zeros(3, dtype=torch.float64, device=f.device) if return_force else None
    out = _bfl(f, f_prev, fluid_boundary_mask, q_field, "D3Q19", force)
    if not return_force:
        return out
    fo = force.to(f.dtype)
    return out, (fo[0], fo[1], fo[2])


class CurvedWall:
    """Link tables of a curved wall for the fused step.

    ``fluid_boundary_mask`` / ``q_field`` are the (Q, nz, ny, nx) outputs of
    :func:`compute_q_sphere_common` (or any geometry in that format);
    ``solid`` the cells inside the wall (bounced back full-way, not in the
    drag: the drag of a curved wall is its BFL ledger).  The cells with a link
    get ``TLBM_FLAG_CURVED``; their wall fractions are packed into
    ``link_q`` (one row of Q per cell, 0 = no link) indexed by ``link_row``."""

    def __init__(self, fluid_boundary_mask: torch.Tensor, q_field: torch.Tensor, solid: torch.Tensor):
        if tuple(q_field.shape) != tuple(fluid_boundary_mask.shape):
            raise ValueError("q_field and fluid_boundary_mask must have the same shape")
        if tuple(solid.shape) != tuple(fluid_boundary_mask.shape[1:]):
            raise ValueError("solid must have the spatial shape of the link mask")
        mask = fluid_boundary_mask.bool()
        q = mask.shape[0]
        dev = mask.device
        self.q = q
        self.solid = solid.bool()
        self.cells = mask.any(0)                                   # (nz, ny, nx): cells with a link
        if bool((self.cells & self.solid).any()):
            raise ValueError("a link starts in a solid cell")
        flat = self.cells.reshape(-1)
        rows = torch.cumsum(flat.to(torch.int32), 0, dtype=torch.int32) - 1
        self.link_row = torch.where(flat, rows, torch.full_like(rows, -1)).contiguous()
        lq = torch.where(mask, q_field.to(torch.float32), torch.zeros((), dtype=torch.float32, device=dev))
        self.link_q = lq.reshape(q, -1)[:, flat].t().contiguous()  # (rows, Q)
        self.n_links = int(mask.sum())

    def attach(self, desc: _lib.Desc) -> _lib.Desc:
        desc.link_row = self.link_row.data_ptr()
        desc.link_q = self.link_q.data_ptr()
        return desc


def sphere_wall(nx: int, ny: int, nz: int, cx: float, cy: float, cz: float, radius: float, device=None, *,
                lattice: str = "D3Q19") -> CurvedWall:
    """:class:`CurvedWall` of a sphere (links and solid by the same float64 test)."""
    mask, qf, solid = sphere_links(nx, ny, nz, cx, cy, cz, radius, device, lattice=lattice)
    return CurvedWall(mask, qf, solid)
