"""Cavity helpers: the 2-D boundary functions of tensorlbm/lid_driven_cavity.py:404-473,
and TensorLBM's verified 3-D lid-driven cavity benchmark run on the fused kernel
(:func:`cavity_3d_full`)."""

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


def cavity_3d_full(nx: int = 64, re: float = 1000.0, u_lid: float = 0.06, steps: int = 100_000, device=None,
                   chunk: int = 500) -> dict:
    """TensorLBM's verified 3-D lid-driven cavity
    (benchmarks/verified/cavity_3d_full/run.py:80-190) on the fused kernel.

    Cube nz = ny = nx, D3Q19 TRT (Lambda = 3/16), tau = 3 u_lid nx / Re + 1/2;
    the five walls x = 0, x = nx-1, y = 0, z = 0, z = nz-1 bounce back half-way
    before streaming from the pre-collision state; the Zou/He lid moves the
    whole plane y = ny-1 (corners included) at u_lid; rho = 1, u = 0 start.
    After `steps` steps: the centre-plane (z = nz//2) centre lines
    u(x = nx//2, y) and v(x, y = ny//2) divided by u_lid with the wall cells
    zeroed, their u minimum, and the drift of sum(rho) (the benchmark's
    conventions)."""
    import time

    from .d3q19 import equilibrium3d, macroscopic3d
    from .solvers import LBMSolver

    dev = _ops.cuda_device(device)
    n = int(nx)
    tau = 3.0 * u_lid * n / re + 0.5
    wall = torch.zeros((n, n, n), dtype=torch.bool, device=dev)
    wall[:, :, 0] = True
    wall[:, :, -1] = True
    wall[:, 0, :] = True
    wall[0, :, :] = True
    wall[-1, :, :] = True
    rho0 = torch.ones((n, n, n), dtype=torch.float32, device=dev)
    zero = torch.zeros_like(rho0)
    s = LBMSolver("D3Q19", (n, n, n), tau, "trt", device=dev, wall_mask=wall, wall_mode="halfway", u_lid=u_lid)
    s.load(equilibrium3d(rho0, zero, zero, zero))
    mass0 = float(rho0.sum())
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    s.run(steps, chunk=chunk)
    torch.cuda.synchronize(dev)
    secs = time.perf_counter() - t0
    rho, ux, uy, uz = macroscopic3d(s.f)
    ux = ux.masked_fill(wall, 0.0) / u_lid
    uy = uy.masked_fill(wall, 0.0) / u_lid
    z0, xm, ym = n // 2, n // 2, n // 2
    u_cl = ux[z0, :, xm].double().cpu()
    v_cl = uy[z0, ym, :].double().cpu()
    return {"nx": n, "re": re, "u_lid": u_lid, "tau": tau, "steps": steps,
            "u_centerline_mid": u_cl.tolist(), "v_centerline_mid": v_cl.tolist(),
            "u_min_3d_mid": float(u_cl.min()), "mass_drift": float(rho.sum()) - mass0,
            "finite": not s.nonfinite_seen(), "seconds": secs, "mlups": n ** 3 * steps / secs / 1e6}


def cavity_2d(nx: int = 128, re: float = 100.0, u_lid: float = 0.06, steps: int = 100_000, device=None,
              chunk: int = 500, collision: str = "mrt") -> dict:
    """TensorLBM's verified 2-D lid-driven cavity (benchmarks/verified/cavity/re100/run.py:45-150;
    re1000/run.py:45-150 with collision="rlbm") on the fused kernel.

    Square nx x nx, D2Q9 MRT with the library's default rates (Re 100) or the
    regularised BGK (Re 1000, where the MRT diverges), tau = 3 u_lid nx / Re + 1/2;
    the walls y = 0, x = 0, x = nx-1 bounce back half-way before streaming
    from the pre-collision state; the Zou/He lid moves the row y = ny-1 at
    u_lid; rho = 1, u = 0 start.  After `steps` steps: the centre lines
    u(x = nx//2, y) and v(x, y = ny//2) divided by u_lid with the wall cells
    zeroed, and the benchmark's point values u(0.5, 0.5), u(0.5, 0.0625) and
    v(0.5, 0.5), linearly interpolated on the node positions linspace(0, 1, n),
    and the primary vortex centre (re1000/run.py:117-131): the slowest cell of
    x in [0.2, 0.85], y in [0.2, 0.9] in node coordinates rounded to 4 places."""
    import time

    import numpy as np

    from .d2q9 import equilibrium, macroscopic
    from .solvers import LBMSolver

    dev = _ops.cuda_device(device)
    n = int(nx)
    tau = 3.0 * u_lid * n / re + 0.5
    wall = torch.zeros((n, n), dtype=torch.bool, device=dev)
    wall[0, :] = True
    wall[:, 0] = True
    wall[:, -1] = True
    rho0 = torch.ones((n, n), dtype=torch.float32, device=dev)
    zero = torch.zeros_like(rho0)
    s = LBMSolver("D2Q9", (n, n), tau, collision, device=dev, wall_mask=wall, wall_mode="halfway", u_lid=u_lid)
    s.load(equilibrium(rho0, zero, zero))
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    s.run(steps, chunk=chunk)
    torch.cuda.synchronize(dev)
    secs = time.perf_counter() - t0
    _, ux, uy = macroscopic(s.f)
    ux = (ux.masked_fill(wall, 0.0) / u_lid).double().cpu().numpy()
    uy = (uy.masked_fill(wall, 0.0) / u_lid).double().cpu().numpy()
    pos = np.linspace(0.0, 1.0, n)
    u_cl, v_cl = ux[:, n // 2], uy[n // 2, :]
    speed2 = ux * ux + uy * uy
    region = (pos[None, :] >= 0.2) & (pos[None, :] <= 0.85) & (pos[:, None] >= 0.2) & (pos[:, None] <= 0.9)
    iy, ix = np.unravel_index(np.argmin(np.where(region, speed2, np.inf)), speed2.shape)
    return {"nx": n, "re": re, "u_lid": u_lid, "tau": tau, "steps": steps, "collision": collision,
            "primary_vortex": [round(ix / (n - 1), 4), round(iy / (n - 1), 4)],
            "u_centerline": u_cl.tolist(), "v_centerline": v_cl.tolist(),
            "u_mid": float(np.interp(0.5, pos, u_cl)), "u_bot": float(np.interp(0.0625, pos, u_cl)),
            "v_mid": float(np.interp(0.5, pos, v_cl)), "finite": not s.nonfinite_seen(), "seconds": secs,
            "mlups": n * n * steps / secs / 1e6}


__all__ = ["make_cavity_wall_mask", "zou_he_moving_lid", "cavity_3d_full", "cavity_2d"]
