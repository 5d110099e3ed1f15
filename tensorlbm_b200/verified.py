"""TensorLBM's verified benchmarks (benchmarks/verified/*) run on the fused kernel.

Each runner builds the benchmark's case as its run.py does, advances it with
:class:`tensorlbm_b200.LBMSolver` (one fused kernel per step) and returns the
quantities the benchmark records, so that they can be compared with the
values in the reference's own result files:

* :func:`pipe_3d` — Hagen-Poiseuille pipe (poiseuille_3d_pipe/run.py);
* :func:`shear_wave` — decaying 2-D shear wave (shear_wave_decay/run.py);
* :func:`taylor_green_2d` — decaying 2-D Taylor-Green vortex (taylor_green_2d/run.py);
* :func:`cylinder_2d` — free-stream cylinder at Re 100 with a sponge and a
  seeded wake (cylinder/re100/run.py);
* :func:`tensorlbm_b200.lid_driven_cavity.cavity_3d_full` — 3-D cavity, Re 1000;
* :func:`tensorlbm_b200.lid_driven_cavity.cavity_2d` — 2-D cavity, Re 100;
* :func:`tensorlbm_b200.tgv.laminar_decay` — laminar 3-D Taylor-Green decay.
"""

from __future__ import annotations

import time

import numpy as np
import torch

from . import _ops
from .lid_driven_cavity import cavity_2d, cavity_3d_full
from .tgv import laminar_decay


def pipe_3d(R: int, tau: float = 0.8, u_in: float = 0.02, steps: int = 20_000, average: int = 400,
            L_over_R: int = 6, device=None) -> dict:
    """TensorLBM's verified Hagen-Poiseuille pipe in velocity mode
    (benchmarks/verified/poiseuille_3d_pipe/run.py:76-101, :187-300).

    Domain (nz, ny, nx) = (2R + 3, 2R + 3, L_over_R R), axis at y = z = R + 1;
    cells farther than R from the axis (float32 distances) are solid and take
    the full-way swap after streaming; D3Q19 BGK, Zou/He velocity inlet u_in
    at x = 0 and pressure outlet rho = 1 at x = nx - 1 (the chain collide ->
    stream -> inlet -> outlet -> bounce-back); start: the equilibrium of the
    parabola 2 u_in (1 - d^2 / (R + 1/2)^2) in the fluid.  After `steps` steps,
    `average` more steps average u_x on the mid plane x = nx // 2 and rho on the
    inlet plane.  Returns the radial profile (means over the bins
    k <= d < k + 1 of the fluid cells), the centre velocity (mean over d < 1/2),
    the flow rate (sum over the fluid cells), the mean inlet density over the
    fluid cells and the mass drift of sum(f) in percent."""
    from .d3q19 import equilibrium3d, macroscopic3d
    from .solvers import LBMSolver

    dev = _ops.cuda_device(device)
    ny = nz = 2 * R + 3
    nx = L_over_R * R
    yc = zc = R + 1
    iz = torch.arange(nz, device=dev, dtype=torch.float32).view(-1, 1)
    iy = torch.arange(ny, device=dev, dtype=torch.float32).view(1, -1)
    d = torch.sqrt((iy - yc) ** 2 + (iz - zc) ** 2)
    fluid2d = d <= R
    wall = (~fluid2d).unsqueeze(-1).expand(nz, ny, nx).contiguous()
    r_eff = R + 0.5
    d3 = d.unsqueeze(-1)
    ux0 = torch.where(fluid2d.unsqueeze(-1), 2.0 * u_in * (1.0 - d3 ** 2 / r_eff ** 2), torch.zeros_like(d3))
    ux0 = ux0.expand(nz, ny, nx).contiguous()
    rho0 = torch.ones((nz, ny, nx), dtype=torch.float32, device=dev)
    zero = torch.zeros_like(rho0)
    f0 = equilibrium3d(rho0, ux0, zero, zero)
    mass0 = float(f0.sum())
    s = LBMSolver("D3Q19", (nz, ny, nx), tau, "bgk", device=dev, wall_mask=wall, u_in=u_in, rho_out=1.0)
    s.load(f0)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    s.run(steps)
    torch.cuda.synchronize(dev)
    secs = time.perf_counter() - t0
    x_meas = nx // 2
    acc_u = torch.zeros((nz, ny), dtype=torch.float32, device=dev)
    acc_rho = torch.zeros((nz, ny), dtype=torch.float32, device=dev)
    for _ in range(average):
        s.step(1)
        rho, ux, _, _ = macroscopic3d(s.f)
        acc_u += ux[:, :, x_meas]
        acc_rho += rho[:, :, 0]
    acc_u /= float(average)
    acc_rho /= float(average)
    f = s.f
    mass_drift_pct = (float(f.sum()) - mass0) / mass0 * 100.0
    d_np = d.cpu().numpy()
    u_np = acc_u.cpu().numpy().astype(np.float64)
    fluid = d_np <= R
    bins = np.floor(d_np).astype(int)
    profile = [float(u_np[fluid & (bins == k)].mean()) for k in range(R + 1) if (fluid & (bins == k)).any()]
    centre = fluid & (d_np < 0.5)
    return {"R": R, "nx": nx, "ny": ny, "nz": nz, "tau": tau, "u_in": u_in, "steps": steps, "average": average,
            "u_profile": profile, "u_center": float(u_np[centre].mean()), "Q": float(u_np[fluid].sum()),
            "rho_in_measured": float(acc_rho[fluid2d].mean()), "mass_drift_pct": mass_drift_pct,
            "finite": not s.nonfinite_seen(), "seconds": secs, "mlups": nx * ny * nz * steps / secs / 1e6}


def shear_wave(n: int, tau: float = 0.8, u0: float = 0.05, steps: int = 3200, record_every: int = 100,
               device=None) -> dict:
    """TensorLBM's verified decaying shear wave (benchmarks/verified/shear_wave_decay/run.py:46-140)
    on the fused kernel.

    Periodic n x n, D2Q9 BGK in float32, f <- collide(stream(f)); start: the
    equilibrium of u_x = u0 sin(2 pi y / n), rho = 1.  Every record_every
    steps E = <|u|^2> / 2 and the largest |u|; the decay rates are minus the
    slopes of least-squares lines through ln E and ln max|u|, against
    2 nu k^2 and nu k^2 with k = 2 pi / n."""
    from .d2q9 import equilibrium, macroscopic
    from .solvers import LBMSolver

    dev = _ops.cuda_device(device)
    k = 2.0 * np.pi / float(n)
    # the initial field as the benchmark builds it (float32 on the CPU)
    ax = torch.arange(n, dtype=torch.float32)
    y, _ = torch.meshgrid(ax, ax, indexing="ij")
    ux0 = (u0 * torch.sin(k * y)).to(dev)
    zero = torch.zeros_like(ux0)
    f0 = equilibrium(torch.ones_like(ux0), ux0, zero)
    s = LBMSolver("D2Q9", (n, n), tau, "bgk", device=dev)
    # stored state P_0 = f_0, then P_j = collide(stream(P_j-1)) is the
    # benchmark's f_j (load() would store collide(f_0))
    s.resume(f0, stored_state=f0)
    times, energies, umaxs = [], [], []
    for step in range(record_every, steps + 1, record_every):
        s.run(record_every, chunk=record_every)
        _, ux, uy = macroscopic(s.state)
        energies.append(float((0.5 * (ux * ux + uy * uy)).mean()))
        umaxs.append(float((ux * ux + uy * uy).sqrt().max()))
        times.append(step)
    t = np.asarray(times, dtype=np.float64)
    nu = (tau - 0.5) / 3.0
    return {"n": n, "tau": tau, "u0": u0, "steps": steps, "record_every": record_every, "times": times,
            "energies": energies, "umaxs": umaxs,
            "gamma_e_sim": float(-np.polyfit(t, np.log(np.asarray(energies)), 1)[0]),
            "gamma_vel_sim": float(-np.polyfit(t, np.log(np.asarray(umaxs)), 1)[0]),
            "gamma_e_theory": 2.0 * nu * k * k, "gamma_vel_theory": nu * k * k,
            "finite": not s.nonfinite_seen()}


def taylor_green_2d(n: int = 128, re: float = 100.0, u0: float = 0.05, steps: int = 4900, record_every: int = 100,
                    device=None) -> dict:
    """TensorLBM's verified decaying 2-D Taylor-Green vortex
    (benchmarks/verified/taylor_green_2d/run.py:52-160) on the fused kernel.

    Periodic n x n, D2Q9 BGK in float32, nu = u0 n / Re, f <- collide(stream(f));
    start: the equilibrium of u = u0 (-cos kx sin ky, sin kx cos ky), rho = 1,
    built on the CPU as the benchmark builds it.  Every record_every steps
    E = <|u|^2> / 2 and max|u|; the decay rates are minus the slopes of
    least-squares lines through ln E and ln max|u| (theory 4 nu k^2 and
    2 nu k^2); the relative mass drift of sum(f) over the run."""
    from .d2q9 import equilibrium, macroscopic
    from .solvers import LBMSolver

    dev = _ops.cuda_device(device)
    k = 2.0 * np.pi / float(n)
    nu = u0 * float(n) / re
    tau = 0.5 + 3.0 * nu
    ax = torch.arange(n, dtype=torch.float32)
    y, x = torch.meshgrid(ax, ax, indexing="ij")
    ux0 = (-u0 * torch.cos(k * x) * torch.sin(k * y)).to(dev)
    uy0 = (u0 * torch.sin(k * x) * torch.cos(k * y)).to(dev)
    f0 = equilibrium(torch.ones_like(ux0), ux0, uy0)
    mass0 = float(f0.sum())
    s = LBMSolver("D2Q9", (n, n), tau, "bgk", device=dev)
    s.resume(f0, stored_state=f0)  # the benchmark's phase: P_j = collide(stream(P_j-1)), P_0 = f_0
    times, energies, umaxs = [], [], []
    for step in range(record_every, steps + 1, record_every):
        s.run(record_every, chunk=record_every)
        _, ux, uy = macroscopic(s.state)
        energies.append(float((0.5 * (ux * ux + uy * uy)).mean()))
        umaxs.append(float((ux * ux + uy * uy).sqrt().max()))
        times.append(step)
    t = np.asarray(times, dtype=np.float64)
    return {"n": n, "re": re, "u0": u0, "tau": tau, "steps": steps, "times": times, "energies": energies,
            "umaxs": umaxs, "gamma_e_sim": float(-np.polyfit(t, np.log(np.asarray(energies)), 1)[0]),
            "gamma_vel_sim": float(-np.polyfit(t, np.log(np.asarray(umaxs)), 1)[0]),
            "gamma_e_theory": 4.0 * nu * k * k, "gamma_vel_theory": 2.0 * nu * k * k,
            "mass_drift_rel": (float(s.state.sum()) - mass0) / mass0, "finite": not s.nonfinite_seen()}


def lift_strouhal(cl: np.ndarray, D: float, u_in: float) -> float:
    """Strouhal number of a lift-coefficient window as benchmarks/verified/cylinder
    computes it (run.py:150-165): peak of the spectrum of the Hann-windowed,
    mean-removed signal, refined by a parabola through the peak bin and its
    neighbours; NaN for fewer than 256 samples."""
    cl_w = np.asarray(cl, dtype=np.float64)
    cl_w = cl_w - cl_w.mean()
    if cl_w.size < 256:
        return float("nan")
    spec = np.abs(np.fft.rfft(cl_w * np.hanning(cl_w.size)))
    k = int(np.argmax(spec[1:])) + 1
    delta = 0.0
    if 0 < k < spec.size - 1:
        den = spec[k - 1] - 2.0 * spec[k] + spec[k + 1]
        if abs(den) > 1e-30:
            delta = float(0.5 * (spec[k - 1] - spec[k + 1]) / den)
    return float((k + delta) / cl_w.size * D / u_in)


def cylinder_2d(D: int, re: float = 100.0, u_in: float = 0.05, steps: int = 60_000, warmup_frac: float = 0.5,
                domain_d: float = 40.0, cyl_x_d: float = 10.0, sponge_d: float = 10.0, sponge_alpha: float = 10.0,
                st_seed: float = 0.165, seed_ampl: float = 0.10, seed_periods: float = 2.0, device=None,
                return_series: bool = False) -> dict:
    """TensorLBM's verified free-stream cylinder (benchmarks/verified/cylinder/re100/run.py:70-220)
    on the fused kernel.

    Square domain of domain_d D cells, cylinder of diameter D at x = cyl_x_d D,
    y = ny / 2; D2Q9 MRT (library rates) with the sponge tau_field
    tau (1 + alpha sigma), sigma the quadratic ramp over the last sponge_d D
    columns; free-stream far field at u_in (inlet, lateral rows, zero-gradient
    outlet), obstacle bounce-back with the momentum-exchange drag every step;
    start: the free-stream equilibrium.  For the first seed_periods periods of
    St_seed the inlet plane takes u_y = seed_ampl u_in sin(2 pi St_seed u_in
    step / D).  Cd is the mean of F_x / (u_in^2 D / 2) from warmup_frac steps on;
    St is the lift spectrum's peak with parabolic interpolation on a
    Hann-windowed, mean-removed C_l, as the benchmark computes it.  With
    return_series the per-step C_d and C_l come back too."""
    import math

    from .boundaries import cylinder_mask, make_sponge_strength
    from .d2q9 import equilibrium
    from .solvers import LBMSolver

    dev = _ops.cuda_device(device)
    nx = ny = int(domain_d * D)
    tau = 0.5 + 3.0 * (u_in * D / re)
    mask = cylinder_mask(nx, ny, cyl_x_d * D, ny / 2.0, D / 2.0, dev)
    sigma = make_sponge_strength(ny, nx, int(nx - sponge_d * D), int(sponge_d * D), power=2.0, device=dev)
    tau_field = tau * (1.0 + sponge_alpha * sigma)
    rho0 = torch.ones((ny, nx), device=dev)
    f0 = equilibrium(rho0, torch.full_like(rho0, u_in), torch.zeros_like(rho0))
    s = LBMSolver("D2Q9", (ny, nx), tau, "mrt", device=dev, obstacle_mask=mask, u_in=u_in, far_field="y",
                  tau_field=tau_field, track_force=True)
    s.load(f0)
    omega = 2.0 * math.pi * st_seed * u_in / D
    seed_steps = int(round(seed_periods / (st_seed * u_in / D)))
    amp = seed_ampl * u_in
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for k in range(1, min(seed_steps, steps) + 1):
        s.set_inlet_perturbation(0.0, amp * math.sin(omega * k)).step(1)
    s.set_inlet_perturbation(0.0, 0.0, 0.0)
    if steps > seed_steps:
        s.run(steps - seed_steps, chunk=500)
    torch.cuda.synchronize(dev)
    secs = time.perf_counter() - t0
    fh = s.force_history().cpu().numpy()
    q_dyn = 0.5 * u_in * u_in * D
    cd, cl = fh[:, 0] / q_dyn, fh[:, 1] / q_dyn
    w0 = int(warmup_frac * steps)
    cl_w = cl[w0:] - cl[w0:].mean()
    st = lift_strouhal(cl[w0:], D, u_in)
    out = {"D": D, "nx": nx, "ny": ny, "re": re, "u_in": u_in, "tau": tau, "steps": steps, "seed_steps": seed_steps,
           "cd": float(cd[w0:].mean()), "st": st, "cl_amp": float(np.abs(cl_w).max()),
           "finite": not s.nonfinite_seen(), "seconds": secs, "mlups": nx * ny * steps / secs / 1e6}
    if return_series:
        out["cd_series"], out["cl_series"] = cd, cl
    return out


__all__ = ["pipe_3d", "shear_wave", "taylor_green_2d", "cylinder_2d", "lift_strouhal", "cavity_3d_full", "cavity_2d", "laminar_decay"]
