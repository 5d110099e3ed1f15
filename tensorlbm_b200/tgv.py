"""Precision study on the decaying Taylor-Green vortex (D3Q27 cumulant).

Storage formats FP16 / BF16 (shifted deviations f_q - w_q, FP32 collision),
FP32 and FP64 run the same flow; FP64 is the reference of every error:

* kinetic energy K(t) = <rho |u|^2> / 2 and dissipation -dK/dt histories;
* velocity L2 error ||u - u_64|| / ||u_64|| at t = 5, 10, 20 convective times;
* mass drift (M(t) - M(0)) / M(0) from FP64 sums of the stored state;
* MLUPS of each storage format (device time of the stepping only).

Flow: u = u0 sin x cos y cos z, v = -u0 cos x sin y cos z, w = 0,
rho = 1 + 3 (u0^2 / 16) (cos 2x + cos 2y)(cos 2z + 2) on x = 2 pi i / n;
nu = u0 L / Re with L = n / (2 pi); one convective time = L / u0 steps.

    python -m tensorlbm_b200.tgv --n 384 --re 1600 --out <dir>

:func:`laminar_decay` is TensorLBM's verified laminar decay benchmark (D3Q19
BGK, Re 24) on the fused kernel: ``python -m tensorlbm_b200.tgv --laminar 64,96,128``.
"""

from __future__ import annotations

import argparse
import json
import math
import pathlib

import torch

from . import LBMSolver
from .d3q27 import equilibrium27, macroscopic27


def tgv_fields(n: int, u0: float, device, dtype=torch.float64):
    i = torch.arange(n, device=device, dtype=dtype) * (2.0 * math.pi / n)
    z, y, x = torch.meshgrid(i, i, i, indexing="ij")
    ux = u0 * torch.sin(x) * torch.cos(y) * torch.cos(z)
    uy = -u0 * torch.cos(x) * torch.sin(y) * torch.cos(z)
    uz = torch.zeros_like(ux)
    rho = 1.0 + 3.0 * (u0 * u0 / 16.0) * (torch.cos(2 * x) + torch.cos(2 * y)) * (torch.cos(2 * z) + 2.0)
    return rho, ux, uy, uz


def _velocity(s: LBMSolver):
    rho, ux, uy, uz = macroscopic27(s.f)
    return rho.double(), torch.stack([ux.double(), uy.double(), uz.double()])


def _timed(fn, device) -> float:
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    fn()
    e1.record()
    torch.cuda.synchronize(device)
    return e0.elapsed_time(e1) / 1e3


def run(n: int = 384, re: float = 1600.0, u0: float = 0.05, t_end: float = 20.0, checkpoints=(5.0, 10.0, 20.0),
        samples_per_tc: int = 4, storages=("f64", "f32", "f16", "bf16"), collision: str = "cumulant",
        device="cuda:0", log=print) -> dict:
    dev = torch.device(device)
    length = n / (2.0 * math.pi)
    nu = u0 * length / re
    tau = 3.0 * nu + 0.5
    tc = length / u0                       # steps per convective time
    every = max(1, int(round(tc / samples_per_tc)))
    total = int(round(t_end * tc))
    marks = {int(round(c * tc)): c for c in checkpoints}
    res = {"n": n, "re": re, "u0": u0, "nu": nu, "tau": tau, "steps_per_convective_time": tc,
           "collision": collision, "runs": {}}
    ref_u: dict[float, torch.Tensor] = {}
    for storage in storages:
        rho0, ux0, uy0, uz0 = tgv_fields(n, u0, dev)
        cdt = torch.float64 if storage == "f64" else torch.float32
        f0 = equilibrium27(rho0.to(cdt), ux0.to(cdt), uy0.to(cdt), uz0.to(cdt))
        del rho0, ux0, uy0, uz0
        s = LBMSolver("D3Q27", (n, n, n), tau, collision, device=dev, storage=storage)
        s.load(f0)
        del f0
        torch.cuda.empty_cache()
        m0 = float(s.moment_sums()[0])
        hist = {"t": [], "kinetic_energy": [], "energy": [], "mass_drift": []}
        errs = {}
        secs = 0.0
        done = 0
        # sample every `every` steps, at the checkpoints and at the end
        stops = sorted(set(range(every, total, every)) | {m for m in marks if m <= total} | {total})
        for stop in stops:
            step = stop - done
            secs += _timed(lambda: s.run(step), dev)
            done = stop
            rho, u = _velocity(s)
            k = 0.5 * float((rho * (u * u).sum(0)).mean())
            hist["t"].append(done / tc)
            hist["kinetic_energy"].append(k)
            hist["energy"].append(0.5 * float((u * u).sum(0).mean()))
            hist["mass_drift"].append((float(s.moment_sums()[0]) - m0) / m0)
            if done in marks:
                c = marks[done]
                if storage == "f64":
                    ref_u[c] = u.clone()
                elif c in ref_u:
                    ref = ref_u[c]
                    errs[str(c)] = float(torch.linalg.vector_norm(u - ref) / torch.linalg.vector_norm(ref))
            del rho, u
        t = hist["t"]
        # -dK/dt per lattice step by central differences (K rho-weighted); the
        # same for E = <|u|^2>/2, TensorLBM's convention
        for key, src in (("dissipation", "kinetic_energy"), ("dissipation_energy", "energy")):
            e = hist[src]
            hist[key] = [-(e[i + 1] - e[i - 1]) / ((t[i + 1] - t[i - 1]) * tc) if 0 < i < len(t) - 1 else None
                         for i in range(len(t))]
        eps = [(v, t[i]) for i, v in enumerate(hist["dissipation_energy"]) if v is not None]
        peak = max(eps) if eps else (None, None)
        entry = {"mlups": n ** 3 * total / max(secs, 1e-12) / 1e6, "seconds": secs,
                 "finite": not s.nonfinite_seen(), "velocity_l2_vs_f64": errs, "history": hist,
                 "mass_drift_end": hist["mass_drift"][-1],
                 "peak_dissipation": peak[0], "peak_dissipation_t": peak[1]}
        res["runs"][storage] = entry
        log(f"{storage}: {entry['mlups']:.0f} MLUPS, L2 vs f64 {errs}, mass drift {entry['mass_drift_end']:.2e}")
        del s
        torch.cuda.empty_cache()
    f32 = res["runs"].get("f32", {}).get("mlups")
    if f32:
        res["speedup_vs_f32"] = {k: v["mlups"] / f32 for k, v in res["runs"].items()}
    return res


def laminar_decay(n: int, re: float = 24.0, u0: float = 0.05, steps: int = 2000, record_every: int = 50,
                  device="cuda:0") -> dict:
    """TensorLBM's verified laminar Taylor-Green decay
    (benchmarks/verified/taylor_green_3d/run.py:87-230) on the fused kernel.

    D3Q19 BGK in float32, f <- collide(stream(f)) every step on a periodic n^3
    box; nu = u0 n / Re, tau = 1/2 + 3 nu, k = 2 pi / n,
    u = (u0 sin kx cos ky cos kz, -u0 cos kx sin ky cos kz, 0), rho = 1, f = feq.
    Every record_every steps E = <|u|^2> / 2 (no density weight, the
    benchmark's convention); gamma_E is minus the slope of a least-squares line
    through ln E over the recorded steps t >= record_every, against the linear
    viscous rate 6 nu k^2 (modes (+-k, +-k, +-k))."""
    from . import FusedSolver3D
    from .d3q19 import equilibrium3d, macroscopic3d

    dev = torch.device(device)
    nu = u0 * n / re
    tau = 0.5 + 3.0 * nu
    k = 2.0 * math.pi / float(n)
    ax = torch.arange(n, device=dev, dtype=torch.float32)
    z, y, x = torch.meshgrid(ax, ax, ax, indexing="ij")
    ux0 = u0 * torch.sin(k * x) * torch.cos(k * y) * torch.cos(k * z)
    uy0 = -u0 * torch.cos(k * x) * torch.sin(k * y) * torch.cos(k * z)
    uz0 = torch.zeros_like(ux0)
    f = equilibrium3d(torch.ones_like(ux0), ux0, uy0, uz0)
    e0 = float((0.5 * (ux0 * ux0)).mean()) + float((0.5 * (uy0 * uy0)).mean())
    del z, y, x
    s = FusedSolver3D(n, n, n, tau=tau, device=dev)
    times, energies = [0], [e0]
    secs = 0.0
    for step in range(record_every, steps + 1, record_every):
        def advance():
            nonlocal f
            for _ in range(record_every):
                f = s.step(f)
        secs += _timed(advance, dev)
        _, ux, uy, uz = macroscopic3d(f)
        energies.append(float((0.5 * (ux * ux)).mean()) + float((0.5 * (uy * uy)).mean()) +
                        float((0.5 * (uz * uz)).mean()))
        times.append(step)
    import numpy as np

    t = np.asarray(times[1:], dtype=np.float64)
    ln_e = np.log(np.asarray(energies[1:], dtype=np.float64))
    slope, icept = np.polyfit(t, ln_e, 1)
    resid = ln_e - (icept + slope * t)
    gamma_theory = 6.0 * nu * k * k
    return {"n": n, "re": re, "u0": u0, "nu": nu, "tau": tau, "steps": steps, "record_every": record_every,
            "times": times, "energies": energies, "gamma_e_sim": float(-slope), "gamma_e_theory": gamma_theory,
            "err_e_pct": float((-slope - gamma_theory) / gamma_theory * 100.0),
            "r2": 1.0 - float(np.sum(resid ** 2) / np.sum((ln_e - ln_e.mean()) ** 2)),
            "mlups": n ** 3 * steps / max(secs, 1e-12) / 1e6}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description="Taylor-Green precision study (D3Q27 cumulant)")
    ap.add_argument("--n", type=int, default=384)
    ap.add_argument("--re", type=float, default=1600.0)
    ap.add_argument("--t-end", type=float, default=20.0)
    ap.add_argument("--collision", default="cumulant")
    ap.add_argument("--storages", default="f64,f32,f16,bf16")
    ap.add_argument("--out", default="tgv_out")
    ap.add_argument("--laminar", default=None,
                    help="comma list of grid sizes: run TensorLBM's verified laminar decay (Re 24) instead")
    args = ap.parse_args(argv)
    if args.laminar:
        res = {str(n): laminar_decay(int(n), steps=2600 if int(n) >= 128 else 2000) for n in args.laminar.split(",")}
        out = pathlib.Path(args.out)
        out.mkdir(parents=True, exist_ok=True)
        (out / "tgv_laminar.json").write_text(json.dumps(res))
        print(json.dumps({n: {k: v for k, v in r.items() if k not in ("times", "energies")} for n, r in res.items()}))
        return
    res = run(args.n, args.re, t_end=args.t_end, storages=tuple(args.storages.split(",")), collision=args.collision,
              log=lambda s: print(s, flush=True))
    out = pathlib.Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    (out / "tgv_precision.json").write_text(json.dumps(res))
    print(json.dumps({k: {kk: vv for kk, vv in v.items() if kk != "history"} for k, v in res["runs"].items()}))


if __name__ == "__main__":
    main()
