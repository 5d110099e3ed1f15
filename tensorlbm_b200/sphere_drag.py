"""Drag of a sphere against grid resolution: staircase full-way bounce-back
against Bouzidi (BFL) interpolated links.

Channel 8D x 4D x 4D (x streamwise; periodic in y and z), Zou/He velocity
inlet u0 at x = 0 and pressure outlet at x = nx-1, sphere of diameter D with
its centre off the lattice nodes at (2.5 D + 0.3, 2 D + 0.2, 2 D + 0.1),
Re = u0 D / nu fixed, D3Q19 with the chosen collision.  A second sweep moves
the centre by (o, o, o), o = 0 ... 0.5, at one diameter: the staircase shape
changes with o, the BFL wall does not.  The staircase run
uses the float32 sphere mask with the momentum-exchange force of the
obstacle cells (compute_obstacle_forces_3d); the BFL run uses the sphere's
links (compute_q_sphere_common) with the link ledger (bfl_d3q19.py:339).
Cd = F_x / (rho u0^2 pi D^2 / 8), averaged over the second half of the run.

    python -m tensorlbm_b200.sphere_drag --diameters 8,12,16,24,32 --re 20 --out <dir>
"""

from __future__ import annotations

import argparse
import json
import math
import pathlib

import torch

from . import LBMSolver, bfl, boundaries3d
from .d3q19 import equilibrium3d


def drag_coefficient(diameter: int, method: str, re: float = 20.0, u0: float = 0.04, flow_throughs: float = 6.0,
                     collision: str = "mrt", offset=(0.3, 0.2, 0.1), device="cuda:0") -> dict:
    dev = torch.device(device)
    d = int(diameter)
    nx, ny, nz = 8 * d, 4 * d, 4 * d
    cx, cy, cz, r = 2.5 * d + offset[0], 2.0 * d + offset[1], 2.0 * d + offset[2], d / 2.0
    nu = u0 * d / re
    tau = 3.0 * nu + 0.5
    steps = int(round(flow_throughs * nx / u0))
    kw = dict(device=dev, u_in=u0, rho_out=1.0, track_force=True)
    if method == "staircase":
        solid = boundaries3d.sphere_mask(nx, ny, nz, cx, cy, cz, r, dev)
        s = LBMSolver("D3Q19", (nz, ny, nx), tau, collision, obstacle_mask=solid, **kw)
    elif method == "bfl":
        wall = bfl.sphere_wall(nx, ny, nz, cx, cy, cz, r, dev)
        solid = wall.solid
        s = LBMSolver("D3Q19", (nz, ny, nx), tau, collision, curved_wall=wall, **kw)
    else:
        raise ValueError(f"method must be 'staircase' or 'bfl', got {method!r}")
    ux = torch.full((nz, ny, nx), u0, dtype=torch.float32, device=dev)
    ux[solid] = 0.0
    zero = torch.zeros_like(ux)
    s.load(equilibrium3d(torch.ones_like(ux), ux, zero, zero))
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    s.step(steps)
    e1.record()
    torch.cuda.synchronize(dev)
    # the impulsive start leaves acoustic waves between the Zou/He planes;
    # the second half of the run spans many of their periods (2 nx / c_s)
    forces = s.force_history()[:, 0].double()
    tail = forces[-max(1, steps // 2):]
    cd = float(tail.mean()) / (0.5 * u0 * u0 * math.pi * r * r)
    return {"diameter": d, "method": method, "offset": list(offset), "grid": [nx, ny, nz], "tau": tau,
            "steps": steps, "cd": cd,
            "cd_tail_rel_spread": float((tail.max() - tail.min()) / tail.abs().mean()),
            "finite": not s.nonfinite_seen(), "mlups": nx * ny * nz * steps / (e0.elapsed_time(e1) / 1e3) / 1e6,
            "solid_cells": int(solid.sum())}


def run(diameters=(8, 12, 16, 24, 32), re: float = 20.0, collision: str = "mrt", offset_diameter: int = 10,
        offsets=(0.0, 0.1, 0.2, 0.3, 0.4, 0.5), device="cuda:0", log=print) -> dict:
    """Grid sequence at a fixed sub-cell offset, then the spread of Cd over
    sub-cell positions (dx = dy = dz = offset) at one diameter."""
    out = {"re": re, "collision": collision, "runs": [], "offset_runs": []}
    for d in diameters:
        for method in ("staircase", "bfl"):
            r = drag_coefficient(d, method, re=re, collision=collision, device=device)
            out["runs"].append(r)
            log(f"D={d:3d} {method:9s} Cd={r['cd']:.4f} (second-half spread {r['cd_tail_rel_spread']:.1e}, "
                f"{r['steps']} steps, {r['mlups']:.0f} MLUPS)")
    for method in ("staircase", "bfl"):
        cds = [r["cd"] for r in out["runs"] if r["method"] == method]
        out[f"{method}_rel_dev_from_finest"] = [abs(c - cds[-1]) / abs(cds[-1]) for c in cds]
        cds_off = []
        for o in offsets:
            r = drag_coefficient(offset_diameter, method, re=re, collision=collision, offset=(o, o, o), device=device)
            out["offset_runs"].append(r)
            cds_off.append(r["cd"])
        mean = sum(cds_off) / len(cds_off)
        out[f"{method}_offset_cd"] = cds_off
        out[f"{method}_offset_rel_spread"] = (max(cds_off) - min(cds_off)) / abs(mean)
        log(f"D={offset_diameter} {method:9s} Cd over offsets {[round(c, 4) for c in cds_off]}: "
            f"spread {out[f'{method}_offset_rel_spread']:.2%}")
    return out


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description="sphere drag: staircase vs Bouzidi links")
    ap.add_argument("--diameters", default="8,12,16,24,32")
    ap.add_argument("--re", type=float, default=20.0)
    ap.add_argument("--collision", default="mrt")
    ap.add_argument("--out", default="sphere_drag_out")
    args = ap.parse_args(argv)
    res = run(tuple(int(v) for v in args.diameters.split(",")), args.re, args.collision,
              log=lambda m: print(m, flush=True))
    out = pathlib.Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    (out / "sphere_drag.json").write_text(json.dumps(res, indent=1))
    print(json.dumps({k: v for k, v in res.items() if k != "runs"}))


if __name__ == "__main__":
    main()
