"""Link-wise momentum-exchange drag (MEM) variants: drop-ins for
``tensorlbm.momentum_exchange`` (momentum_exchange.py:75-360).

All four link-wise variants come from one CUDA pass
(``tlbm_link_momentum_sums``). For every near-wall fluid cell x and every
direction q whose periodic neighbour x + c_q is solid, it adds
(f_q(x) + f_opp(q)(x + c_q)) to a float64 sum for direction q and counts the
link. The force is then Σ_q c_q · sum_q:
- **standard** (Ladd): the sums as they are;
- **Galilean**: times (1 + 1/(2τ));
- **background-subtracted**: minus 2 ρ0 w_q (1 + 4.5 (c_q·u0)² − 1.5 |u0|²)
  per link;
- **BFL**: with each link weighted by 1 / max(q_wall, 1e-6).

The reference loops over the 18 directions with two ``torch.roll`` per
direction. This pass reads the near mask once and touches the populations
only at near cells.

``f`` is the post-streaming field ``(Q, nz, ny, nx)`` (D3Q19 as in the
reference; D3Q27 and D2Q9 ``(9, ny, nx)`` are accepted too), ``solid`` and
``near`` boolean ``(nz, ny, nx)``. The forces are the force on the wall,
drag-positive, as Python floats. The per-direction sums are float64, where
the reference sums in f's dtype.

The surface-integral methods of the same module
(``momentum_exchange_stress``, ``momentum_exchange_pressure_friction``,
``compare_all_methods``) delegate to ``drag_pressure``'s SurfaceMesh
integration, which is not part of this library. They raise
``NotImplementedError``.
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib, _ops
from .lattice import LATTICES


def _shape3(f: torch.Tensor) -> tuple[int, tuple[int, int, int]]:
    q = int(f.shape[0])
    if q not in LATTICES:
        raise ValueError(f"f has {q} directions; expected 9, 19 or 27")
    if q == 9 and f.dim() == 3:
        ny, nx = f.shape[1:]
        return q, (nx, ny, 1)
    if f.dim() != 4:
        raise ValueError(f"expected f of shape (Q, nz, ny, nx), got {tuple(f.shape)}")
    nz, ny, nx = f.shape[1:]
    return q, (nx, ny, nz)


def link_momentum_sums(f: torch.Tensor, solid: torch.Tensor, near: torch.Tensor,
                       q_wall: torch.Tensor | None = None) -> torch.Tensor:
    """The 2Q float64 link sums on f's device: [0, Q) the per-direction sums of
    (f_q(x) + f_opp(x + c_q)) (weighted by 1 / max(q_wall, 1e-6) when given),
    [Q, 2Q) the link counts."""
    dev = _lib.require_cuda(f, solid, near)
    q, (nx, ny, nz) = _shape3(f)
    spatial = tuple(f.shape[1:])
    for name, t in (("solid", solid), ("near", near)):
        if tuple(t.shape) != spatial:
            raise ValueError(f"{name} shape {tuple(t.shape)} does not match the field {spatial}")
    if f.dtype not in (torch.float32, torch.float64):
        raise ValueError(f"f must be float32 or float64, got {f.dtype}")
    per_direction = 0
    qw = None
    if q_wall is not None:
        _lib.require_cuda(q_wall)
        if tuple(q_wall.shape) == tuple(f.shape):
            per_direction = 1
        elif tuple(q_wall.shape) != spatial:
            raise ValueError(f"q_wall must have shape {spatial} or {tuple(f.shape)}, got {tuple(q_wall.shape)}")
        qw = q_wall.to(torch.float32).contiguous()
    f = f.contiguous()
    s = solid.to(torch.uint8).contiguous()
    n = near.to(torch.uint8).contiguous()
    sums = torch.empty(2 * q, dtype=torch.float64, device=dev)
    d = _ops.make_desc(q, (nx, ny, nz), _lib.real_dtype(f), _lib.COLL_NONE, 1.0)
    st = _lib.load().tlbm_link_momentum_sums(ctypes.byref(d), f.data_ptr(), s.data_ptr(), n.data_ptr(), _lib.ptr(qw),
                                             per_direction, sums.data_ptr(), _lib.stream_of(dev))
    _lib.check(st, "link_momentum_sums")
    return sums


def _force(sums: torch.Tensor, factor: float = 1.0, background=None) -> tuple[float, float, float]:
    s = sums.cpu().tolist()
    q = len(s) // 2
    lat = LATTICES[q]
    out = [0.0, 0.0, 0.0]
    for i in range(1, q):
        v = s[i] * factor
        if background is not None:
            v -= background[i] * s[q + i]
        c = lat.c[i]
        for a in range(len(c)):
            out[a] += float(c[a]) * v
    return out[0], out[1], out[2]


def momentum_exchange_standard(f: torch.Tensor, solid: torch.Tensor, near: torch.Tensor) -> tuple[float, float, float]:
    """Ladd sum form: F = Σ links (f_q(x) + f_opp(x + c_q)) c_q (momentum_exchange.py:75)."""
    return _force(link_momentum_sums(f, solid, near))


def momentum_exchange_galilean(f: torch.Tensor, solid: torch.Tensor, near: torch.Tensor,
                               tau: float) -> tuple[float, float, float]:
    """The Ladd sum times 1 + 1/(2 tau) (momentum_exchange.py:138)."""
    return _force(link_momentum_sums(f, solid, near), factor=1.0 + 1.0 / (2.0 * float(tau)))


def momentum_exchange_background_subtracted(f: torch.Tensor, solid: torch.Tensor, near: torch.Tensor,
                                            rho0: float = 1.0, u0=(0.0, 0.0, 0.0)) -> tuple[float, float, float]:
    """The Ladd sum minus the uniform-stream equilibrium background per link,
    2 rho0 w_q (1 + 4.5 (c_q . u0)^2 - 1.5 |u0|^2) with float32 weights, as the
    reference evaluates it (momentum_exchange.py:206)."""
    sums = link_momentum_sums(f, solid, near)
    q = sums.numel() // 2
    lat = LATTICES[q]
    u = [float(v) for v in u0] + [0.0] * (3 - len(u0))
    usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2]
    bg = []
    for i in range(q):
        c = list(lat.c[i]) + [0] * (3 - len(lat.c[i]))
        cu = float(c[0]) * u[0] + float(c[1]) * u[1] + float(c[2]) * u[2]
        w32 = float(lat.w32[i])
        bg.append(2.0 * float(rho0) * w32 * (1.0 + 4.5 * cu * cu - 1.5 * usq))
    return _force(sums, background=bg)


def momentum_exchange_bfl(f: torch.Tensor, solid: torch.Tensor, near: torch.Tensor,
                          q_wall: torch.Tensor) -> tuple[float, float, float]:
    """Each link weighted by 1 / max(q, 1e-6), q_wall scalar (nz, ny, nx) or
    per direction (Q, nz, ny, nx) (momentum_exchange.py:285)."""
    return _force(link_momentum_sums(f, solid, near, q_wall))


def _surface_integral(name: str):
    def fn(*args, **kwargs):
        raise NotImplementedError(f"{name}: surface-integral drag (drag_pressure.py SurfaceMesh) is not part of "
                                  "this library; use the link-wise MEM variants")
    fn.__name__ = name
    fn.__doc__ = f"momentum_exchange.{name}: not built (surface-integral methods)."
    return fn


momentum_exchange_stress = _surface_integral("momentum_exchange_stress")
momentum_exchange_pressure_friction = _surface_integral("momentum_exchange_pressure_friction")
compare_all_methods = _surface_integral("compare_all_methods")

__all__ = [
    "link_momentum_sums",
    "momentum_exchange_standard",
    "momentum_exchange_galilean",
    "momentum_exchange_background_subtracted",
    "momentum_exchange_bfl",
    "momentum_exchange_stress",
    "momentum_exchange_pressure_friction",
    "compare_all_methods",
]
