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
        hist = {"t": [], "kinetic_energy": [], "mass_drift": []}
        errs = {}
        secs = 0.0
        done = 0
        while done < total:
            step = min(every, total - done)
            # stop exactly at the next checkpoint
            nxt = [m for m in marks if m > done]
            if nxt:
                step = min(step, min(nxt) - done)
            secs += _timed(lambda: s.run(step), dev)
            done += step
            if done % every == 0 or done in marks or done == total:
                rho, u = _velocity(s)
                k = 0.5 * float((rho * (u * u).sum(0)).mean())
                hist["t"].append(done / tc)
                hist["kinetic_energy"].append(k)
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
        e = hist["kinetic_energy"]
        hist["dissipation"] = [-(e[i + 1] - e[i - 1]) / ((t[i + 1] - t[i - 1]) * tc) if 0 < i < len(t) - 1 else None
                               for i in range(len(t))]
        entry = {"mlups": n ** 3 * total / max(secs, 1e-12) / 1e6, "seconds": secs,
                 "finite": not s.nonfinite_seen(), "velocity_l2_vs_f64": errs, "history": hist,
                 "mass_drift_end": hist["mass_drift"][-1]}
        res["runs"][storage] = entry
        log(f"{storage}: {entry['mlups']:.0f} MLUPS, L2 vs f64 {errs}, mass drift {entry['mass_drift_end']:.2e}")
        del s
        torch.cuda.empty_cache()
    f32 = res["runs"].get("f32", {}).get("mlups")
    if f32:
        res["speedup_vs_f32"] = {k: v["mlups"] / f32 for k, v in res["runs"].items()}
    return res


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description="Taylor-Green precision study (D3Q27 cumulant)")
    ap.add_argument("--n", type=int, default=384)
    ap.add_argument("--re", type=float, default=1600.0)
    ap.add_argument("--t-end", type=float, default=20.0)
    ap.add_argument("--collision", default="cumulant")
    ap.add_argument("--storages", default="f64,f32,f16,bf16")
    ap.add_argument("--out", default="tgv_out")
    args = ap.parse_args(argv)
    res = run(args.n, args.re, t_end=args.t_end, storages=tuple(args.storages.split(",")), collision=args.collision,
              log=lambda s: print(s, flush=True))
    out = pathlib.Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    (out / "tgv_precision.json").write_text(json.dumps(res))
    print(json.dumps({k: {kk: vv for kk, vv in v.items() if kk != "history"} for k, v in res["runs"].items()}))


if __name__ == "__main__":
    main()
