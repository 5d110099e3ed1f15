"""Scan points of TensorLBM's registered 3-D cavity case, advanced together.

TensorLBM's scan runner runs one design point after the other
(``scan_runner.py:697`` ``run_scan_point``, ``:979`` ``ScanExecutor``): for
each point it builds the registered case (``cases/cavity.py:25-110`` for
``"cavity"``), takes ``case.initial_f()`` and applies ``case.make_step()``
(``cases/base.py:270-289``: collide -> pre-streaming half-way walls -> stream
-> lid) ``plan.steps`` times.  :func:`run_cavity_points` runs the step loop of
many such points as one batched D3Q19 launch per step (or one persistent
launch), every point evolving bit for bit as its own fused run.  The scan's
orchestration (plan files, catalog, HDF5 export, reporters, resume) stays
TensorLBM's: a point's result is its final TensorLBM-phase population field.
"""

from __future__ import annotations

import torch

from . import _ops
from .batch import BatchedSolver, cavity_point


def cavity_initial_f(domain, device=None) -> torch.Tensor:
    """``case.initial_f()`` of the cavity case: the equilibrium at rest, rho = 1."""
    from .d3q19 import equilibrium3d

    dev = _ops.cuda_device(device)
    z = torch.zeros(domain.shape, dtype=torch.float32, device=dev)
    return equilibrium3d(torch.ones_like(z), z, z, z)


def run_cavity_points(points: list[dict], steps: int, *, collision: str = "mrt", device=None,
                      mode: str = "graph", tile: tuple[int, int] = (64, 4),
                      cells_per_thread: int = 2) -> list[torch.Tensor]:
    """Final TensorLBM-phase populations ``(19, nz, ny, nx)`` of every point
    after ``steps`` steps of the cavity case's chain.

    points: the case parameters of each point (``resolution``, ``re``,
    optional ``u_lid`` and ``span``, as ``get_case("cavity", **params)`` takes
    them); collision: the case's collision family ("mrt", the case default,
    or "bgk"), shared by all points of a scan."""
    if steps < 0:
        raise ValueError(f"steps must be >= 0, got {steps}")
    dev = _ops.cuda_device(device)
    domains = [cavity_point(p["resolution"], float(p.get("re", 400.0)), u_lid=float(p.get("u_lid", 0.06)),
                            span=p.get("span"), device=dev) for p in points]
    b = BatchedSolver(domains, collision, device=dev, lattice="D3Q19", mode=mode, tile=tile,
                      cells_per_thread=cells_per_thread)
    b.load([cavity_initial_f(d, dev) for d in domains])
    if steps:
        b.run(steps)
    return [b.f(i) for i in range(len(domains))]


__all__ = ["cavity_initial_f", "run_cavity_points"]
