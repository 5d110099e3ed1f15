"""Benchmark: MLUPS of the fused LBM step on the D3Q19 MRT channel flow past a sphere.

Workload (one "step" = one fused time step of the whole grid): 512 x 256 x 256
cells, sphere of diameter 32 at (128, 128, 128), Zou/He velocity inlet
u = 0.04, pressure outlet rho = 1, periodic y/z, Re = 300
(tau = 3 u D / Re + 0.5), float32 populations, momentum-exchange drag
accumulated in float64 every step.  Synthetic initial state: the equilibrium
of the inlet velocity (zero inside the sphere), as TensorLBM's sphere runner
starts.  The same grid is also timed with the D3Q27 cumulant collision and
with D3Q19 MRT on float16 shifted storage ("variants").

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun as a z-slab decomposition of one periodic-in-z
domain of 512 x 256 x (256 N) cells with one sphere per slab (weak scaling:
every rank steps a 512 x 256 x 256 slab): each step computes the slab's two
boundary planes, exchanges their crossing populations (5 lanes per face) with
the neighbouring ranks over NCCL while the interior planes are computed, and
the next step waits for that exchange on the stream.  The time is the max over
ranks and the value is the total cell updates of all ranks per second.  Rank 0
prints one JSON line.

--impl reference times TensorLBM's own CPU implementation of the same chain
(its torch operators, unmodified, from baseline/_ref) on every host core, on a
bounded z-slab sample of the workload; the same sample is the cpu_baseline of
our arm.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

NZ, NY, NX = 256, 256, 512
D, CX, CY, CZ = 32, 128, 128, 128
U_IN, RE = 0.04, 300.0
TAU = 3.0 * U_IN * D / RE + 0.5
METRIC = "MLUPS (D3Q19 MRT sphere channel 512x256x256, fused step)"
WORKLOAD = "d3q19_mrt_sphere_channel_512x256x256"
HBM_FALLBACK_GBS = 6650.0
SPEC_HBM_GBS = 8000.0
DATA = "synthetic: equilibrium initial state of the inlet velocity (zero in the sphere)"


def workload_config(world: int) -> dict:
    """The workload both arms report (identical dicts)."""
    return {
        "workload": WORKLOAD,
        "grid": [NX, NY, NZ],
        "lattice": "D3Q19",
        "collision": "mrt",
        "sphere": {"diameter": D, "center": [CX, CY, CZ]},
        "u_in": U_IN, "re": RE, "tau": TAU,
        "boundaries": "zou_he velocity inlet x=0, zou_he pressure outlet x=nx-1, periodic y/z, "
                      "full-way bounce-back + FP64 momentum-exchange drag on the sphere",
        "l2": "no flush: the two population buffers are 5.1 GB, 40x the 126 MB L2",
        "parallelism": (f"z-slabs x{world}: global grid {NX}x{NY}x{NZ * world}, one sphere per slab, "
                        f"NCCL halo exchange of the 5 crossing lanes per face every step "
                        f"({2 * 5 * NX * NY * 4} B sent per rank per step), overlapped with the interior "
                        f"planes") if world > 1 else "single GPU",
    }


def _peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return HBM_FALLBACK_GBS, "fallback"


def _traffic(workload: str):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        return json.loads(p.read_text()).get(workload)
    except Exception:
        return None


class ClockSampler:
    """SM clocks, power and clock-event (throttle) reasons during the timed
    region, polled through NVML every 2 ms in a background thread (a
    20-step region of the headline lasts about 16 ms), plus one sample as the
    region opens and one as it closes.  Falls back to ``nvidia-smi -lms 100``
    when NVML cannot be loaded."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, index: int, period_s: float = 0.002):
        self.index = index
        self.period = period_s
        self.rows: list[tuple[float, float, float, int]] = []   # sm MHz, max MHz, watts, reason bits
        self.smi_rows: list[list[str]] = []
        self.proc = None
        self.thread = None
        self.nvml = None
        self.handle = None
        self.stop = threading.Event()
        self.source = None

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        self.nvml = pynvml
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _sample(self):
        n, h = self.nvml, self.handle
        try:
            reasons = n.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            reasons = n.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        self.rows.append((float(n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM)),
                          float(n.nvmlDeviceGetMaxClockInfo(h, n.NVML_CLOCK_SM)),
                          n.nvmlDeviceGetPowerUsage(h) / 1000.0, int(reasons)))

    def _poll(self):
        while not self.stop.is_set():
            try:
                self._sample()
            except Exception:
                return
            time.sleep(self.period)

    def __enter__(self):
        try:
            self.handle = self._nvml_handle()
            self._sample()
            self.source = "nvml"
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read_smi, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.smi_rows and time.time() - t0 < 3.0:
                time.sleep(0.01)
            self.smi_rows.clear()
            self.source = "nvidia-smi"
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read_smi(self):
        for line in self.proc.stdout:
            self.smi_rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        self.stop.set()
        if self.nvml is not None:
            if self.thread is not None:
                self.thread.join(timeout=2)
            try:
                self._sample()
            except Exception:
                pass
            return
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)

    def summary(self) -> dict:
        sm, smax, watts, reasons = [], None, [], set()
        for mhz, mx, w, bits in self.rows:
            sm.append(mhz)
            smax = mx
            watts.append(w)
            reasons.update(name for name, bit in self.REASONS if bits & bit)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.smi_rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                watts.append(float(r[3]))
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(watts) if watts else None, "source": self.source}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------


def _make_solver(torch, dev, lattice, collision, storage, track_force, pattern="ab", **rates):
    from tensorlbm_b200 import LBMSolver, boundaries3d

    obst = boundaries3d.sphere_mask(NX, NY, NZ, CX, CY, CZ, D / 2, dev)
    s = LBMSolver(lattice, (NZ, NY, NX), TAU, collision, device=dev, storage=storage, obstacle_mask=obst,
                  u_in=U_IN, rho_out=1.0, track_force=track_force, pattern=pattern, **rates)
    return s, obst


def _make_headline(torch, dev, world: int, rank: int, track_force: bool = False):
    """The headline solver: one GPU's domain, or this rank's slab of the
    z-decomposed domain (the same sphere in every slab) with the halo exchange
    over the default process group."""
    if world == 1:
        return _make_solver(torch, dev, "D3Q19", "mrt", "f32", track_force)
    from tensorlbm_b200 import boundaries3d
    from tensorlbm_b200.slabs import SlabSolver

    obst = boundaries3d.sphere_mask(NX, NY, NZ, CX, CY, CZ, D / 2, dev)
    s = SlabSolver("D3Q19", (NZ * world, NY, NX), TAU, "mrt", device=dev, world=world, rank=rank,
                   obstacle_mask=obst.repeat(world, 1, 1), u_in=U_IN, rho_out=1.0, track_force=track_force)
    return s, obst


def _initial_state(torch, dev, lattice, obst):
    from tensorlbm_b200.d3q19 import equilibrium3d
    from tensorlbm_b200.d3q27 import equilibrium27

    ux = torch.full((NZ, NY, NX), U_IN, device=dev)
    ux[obst] = 0.0
    z = torch.zeros_like(ux)
    eq = equilibrium3d if lattice == "D3Q19" else equilibrium27
    return eq(torch.ones_like(ux), ux, z, z)


def _time_steps(torch, s, steps, warmup, force_buf):
    """Device time of `steps` fused launches on the launching stream (CUDA events)."""
    from tensorlbm_b200 import _lib

    cur = torch.cuda.current_stream(s.device)
    for _ in range(warmup):
        s._launch_parity(s._cur, force_buf)
        s._cur = s._next_parity(s._cur)
    torch.cuda.synchronize(s.device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(cur)
    for _ in range(steps):
        s._launch_parity(s._cur, force_buf)
        s._cur = s._next_parity(s._cur)
    e1.record(cur)
    torch.cuda.synchronize(s.device)
    s.steps_done += steps + warmup
    del _lib
    return e0.elapsed_time(e1) / 1e3


def _variant(torch, dev, lattice, collision, storage, steps, warmup, bytes_per_cell, peak, pattern="ab", **rates):
    s, obst = _make_solver(torch, dev, lattice, collision, storage, False, pattern, **rates)
    s.load(_initial_state(torch, dev, lattice, obst))
    force = torch.zeros(3, dtype=torch.float64, device=dev)
    t = _time_steps(torch, s, steps, warmup, force)
    cells = NX * NY * NZ
    mlups = cells * steps / t / 1e6
    gbs = bytes_per_cell * cells / (t / steps) / 1e9
    finite = not s.nonfinite_seen()
    del s
    torch.cuda.empty_cache()
    out = {"mlups": round(mlups, 1), "ms_per_step": round(1e3 * t / steps, 4), "achieved_gbs": round(gbs, 1),
           "roofline_frac": round(gbs / peak, 4), "bytes_per_cell": bytes_per_cell, "finite": finite}
    if pattern == "aa":
        out["pattern"] = "aa (one population buffer, in place)"
    if rates:
        out["rates"] = rates
    return out


def _les_variant(torch, dev, steps, warmup, peak, n_mlp=128, n_smag=256):
    """Forced-turbulence LES steps: the fused learned-closure step (tensor-core
    MLP per cell) at n_mlp^3 against the fused Smagorinsky step at n_smag^3,
    both from a seeded random solenoidal field.  The network has random
    weights and an unbounded training range (no cell takes the fallback): its
    cost does not depend on the weight values."""
    from tensorlbm_b200 import LBMSolver
    from tensorlbm_b200.ai import EddyViscosityMLP3D, LearnedLESSolver
    from tensorlbm_b200.ai.pipeline import equilibrium_field, random_solenoidal_field

    def timed(run):
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / 1e3

    out = {}
    model = EddyViscosityMLP3D(dev, seed=7)
    model.nu_scale = 1e-3
    f0 = equilibrium_field(random_solenoidal_field(n_mlp, 4.0, 0.05, 3, dev))
    s = LearnedLESSolver((n_mlp,) * 3, 0.51, model, force_lin=1e-4, device=dev).load(f0)
    s.step(warmup)
    t = timed(lambda: s.step(steps))
    cells = n_mlp ** 3
    out["mlp"] = {"grid": n_mlp, "mlups": round(cells * steps / t / 1e6, 1), "ms_per_step": round(1e3 * t / steps, 4),
                  "roofline_frac": round(152 * cells / (t / steps) / 1e9 / peak, 4),
                  "finite": not s.nonfinite_seen(), "fallback_cells": int(s.fallback.item())}
    del s, f0
    f0 = equilibrium_field(random_solenoidal_field(n_smag, 4.0, 0.05, 3, dev))
    s = LBMSolver("D3Q19", (n_smag,) * 3, 0.52, "smagorinsky", device=dev, c_smag=0.17, force_lin=1e-4).load(f0)
    s.step(warmup)
    t2 = timed(lambda: s.step(steps))
    cells2 = n_smag ** 3
    out["smagorinsky"] = {"grid": n_smag, "mlups": round(cells2 * steps / t2 / 1e6, 1),
                          "ms_per_step": round(1e3 * t2 / steps, 4),
                          "roofline_frac": round(152 * cells2 / (t2 / steps) / 1e9 / peak, 4)}
    # the same physical time: one n_mlp step covers n_smag / n_mlp steps of the finer grid
    out["wall_time_ratio_same_physical_time"] = round((t2 / steps) * (n_smag / n_mlp) / (t / steps), 2)
    del s, f0
    torch.cuda.empty_cache()
    return out


def _batched_variant(torch, dev, steps, peak):
    """512 D2Q9 BGK cylinder channels (nx ~ U{128..1024}, ny = nx/4, D = ny/8,
    Re ~ U(40, 300), seed 20261203) advanced together, against the same domains
    run one after the other (TensorLBM's scan runner does points sequentially).
    At least 500 steps.  Domains whose BGK run turns non-finite (tau - 1/2
    down to 0.0027; TensorLBM's own chain diverges on them at the same step)
    are retired, as a scan marks a failed point, so the batch's time is spent
    on the live domains; the throughput counts live cell updates only.  The
    sequential sample is 16 domains that stay finite."""
    from tensorlbm_b200 import LBMSolver, batch

    steps = max(steps, 500)
    chunk = 100
    doms = batch.uniform_scan(512, seed=20261203, device=dev)
    f0 = batch.equilibrium_start(doms, dev)
    b = batch.BatchedSolver(doms, "bgk", device=dev, retire=True)
    b.load(f0)
    tune = batch.autotune(b, steps=5)
    cells = torch.tensor([d.nx * d.ny for d in doms], dtype=torch.float64)
    cur = torch.cuda.current_stream(dev)

    def timed_run(record_every):
        b.load(f0)
        b.run(chunk, record_every=record_every)       # warm-up: graphs captured
        b.load(f0)
        t, live_updates = 0.0, 0.0
        for _ in range(0, steps, chunk):
            live = (~b.retired_domains()).cpu()
            live_updates += float(cells[live].sum()) * chunk
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(cur)
            b.run(chunk, record_every=record_every)
            e1.record(cur)
            torch.cuda.synchronize(dev)
            t += e0.elapsed_time(e1) / 1e3
        return t, live_updates

    t, live_updates = timed_run(0)
    finite = (~b.retired_domains()).cpu()
    t_rec, live_rec = timed_run(10)
    total = b.n_cells
    # sequential plain runs of 16 domains that stayed finite (graph-replayed fused steps)
    idx = [i for i in range(len(doms)) if bool(finite[i])]
    pick = [idx[int(k * (len(idx) - 1) / 15)] for k in range(16)] if len(idx) >= 16 else idx
    seq_cells, seq_t = 0, 0.0
    for i in pick:
        d = doms[i]
        s = LBMSolver("D2Q9", (d.ny, d.nx), d.tau, "bgk", device=dev, wall_mask=d.wall_mask,
                      obstacle_mask=d.obstacle_mask, u_in=d.u_in, rho_out=d.rho_out).load(f0[i])
        s.run(64)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        s.run(steps)
        e1.record(cur)
        torch.cuda.synchronize(dev)
        seq_t += e0.elapsed_time(e1) / 1e3
        seq_cells += d.nx * d.ny
    seq_mlups = seq_cells * steps / seq_t / 1e6
    live_mlups = live_updates / t / 1e6
    del b
    torch.cuda.empty_cache()
    return {"steps": steps, "domains": 512, "cells": total,
            "mlups_live": round(live_mlups, 1), "ms_per_step": round(1e3 * t / steps, 4),
            "mlups_all_cells": round(total * steps / t / 1e6, 1),
            "mlups_live_recording_forces_every_10": round(live_rec / t_rec / 1e6, 1),
            "roofline_frac_live": round(72 * live_updates / t / 1e9 / peak, 4), "bytes_per_cell": 72,
            "mode": tune["best"]["mode"], "tile": list(tune["best"]["tile"]), "order": tune["best"]["order"],
            "cells_per_thread": tune["best"]["cells_per_thread"],
            "ctas_per_sm": tune["best"]["ctas_per_sm"],
            "finite_domains": int(finite.sum()), "retired_domains": 512 - int(finite.sum()),
            "sequential_mlups_16_finite_domains": round(seq_mlups, 1),
            "speedup_vs_sequential": round(live_mlups / seq_mlups, 2)}


C2_LONG = "c2_20k_vs_fp64"     # opt-in variant: --variants c2_20k_vs_fp64 [--long-steps N]


def _c2_long_variant(torch, dev, steps, every):
    """Config 2 at its stated length: the 512 x 256 x 256 sphere channel
    (D3Q19 MRT and D3Q27 legacy cumulant) run for `steps` steps with float32
    storage beside the same run with float64 storage (the FP64 oracle run on
    the GPU), the FP64 drag of both recorded every step.  Every `every` steps:
    velocity L2 error ||u32 - u64|| / ||u64|| over the fluid, the largest
    population error relative to max |f64|, the density error, and the drag
    difference."""
    from tensorlbm_b200.d3q19 import macroscopic3d
    from tensorlbm_b200.d3q27 import macroscopic27

    out = {}
    for lattice, coll in (("D3Q19", "mrt"), ("D3Q27", "cumulant")):
        runs = {}
        for st in ("f32", "f64"):
            s, obst = _make_solver(torch, dev, lattice, coll, st, False)
            f0 = _initial_state(torch, dev, lattice, obst)
            s.load(f0.double() if st == "f64" else f0)
            runs[st] = (s, torch.zeros((steps, 3), dtype=torch.float64, device=dev))
            del f0
        fluid = ~obst
        mac = macroscopic3d if lattice == "D3Q19" else macroscopic27
        hist = []
        t = {"f32": 0.0, "f64": 0.0}
        for k0 in range(0, steps, every):
            k1 = min(steps, k0 + every)
            for st, (s, drag) in runs.items():
                torch.cuda.synchronize(dev)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for k in range(k0, k1):
                    s._launch_parity(s._cur, drag[k])
                    s._cur = s._next_parity(s._cur)
                e1.record()
                torch.cuda.synchronize(dev)
                t[st] += e0.elapsed_time(e1) / 1e3
                s.steps_done += k1 - k0
            fa, fb = runs["f32"][0].f, runs["f64"][0].f
            ra, *ua = mac(fa)
            rb, *ub = mac(fb)
            num = sum(float(((a.double() - b)[fluid] ** 2).sum()) for a, b in zip(ua, ub))
            den = sum(float((b[fluid] ** 2).sum()) for b in ub)
            da, db = runs["f32"][1][k1 - 1], runs["f64"][1][k1 - 1]
            hist.append({"step": k1, "velocity_l2": math.sqrt(num / den),
                         "f_max_rel": float((fa.double() - fb).abs().max() / fb.abs().max()),
                         "rho_max_abs": float((ra.double() - rb).abs().max()),
                         "drag_fx_f32": float(da[0]), "drag_fx_f64": float(db[0]),
                         "drag_fx_rel": float(abs(da[0] - db[0]) / abs(db[0])),
                         "finite": bool(torch.isfinite(fa).all())})
            del fa, fb, ra, rb, ua, ub
        d32, d64 = runs["f32"][1], runs["f64"][1]
        tail = slice(steps - steps // 10, steps)
        cells = NX * NY * NZ
        out[f"{lattice.lower()}_{coll}"] = {
            "steps": steps, "tau": TAU, "history": hist,
            "drag_fx_mean_last10pct_f32": float(d32[tail, 0].mean()),
            "drag_fx_mean_last10pct_f64": float(d64[tail, 0].mean()),
            # the instantaneous drag passes near zero in the start-up transient: the
            # difference is scaled by the window's mean |Fx|, not by each step's value
            "drag_fx_max_abs_diff_over_mean_after_1000": float((d32[1000:, 0] - d64[1000:, 0]).abs().max()
                                                                / d64[1000:, 0].abs().mean()) if steps > 1000 else None,
            "mlups_f32": round(cells * steps / t["f32"] / 1e6, 1),
            "mlups_f64": round(cells * steps / t["f64"] / 1e6, 1)}
        del runs, d32, d64
        torch.cuda.empty_cache()
    return out


REF_TRITON = "reference_triton_256"   # opt-in variant: --variants reference_triton_256


def _import_reference_package():
    """TensorLBM's own Triton kernels, from its unmodified install in baseline/_ref."""
    from baseline import reference

    reference.import_reference()
    from tensorlbm import triton_fused, triton_fused_obstacle

    return triton_fused, triton_fused_obstacle


def _reference_triton_variant(torch, dev, steps, warmup, peak, n=256):
    """TensorLBM's own GPU kernels (Triton, JIT-compiled here for the B200)
    against this library on the same n^3 field and step count:

    * `triton_fused` (periodic pull + BGK, D3Q19) in float32 / float16 /
      bfloat16 storage against the periodic fused step in f32 / f16 / bf16
      shifted storage, with one float32 parity check of the stored state after
      `warmup` steps (both sides start from collide(f0));
    * `triton_fused_obstacle_xfar_les` (BGK + Smagorinsky C_s = 0.17 + full-way
      bounce-back + fused drag, its default tiling) against the fused
      Smagorinsky step with bounce-back and FP64 drag, on a sphere of 8 % of
      the cells.
    Both sides launch eagerly, one kernel per step (this library's graph path
    is not used here)."""
    from tensorlbm_b200 import LBMSolver
    from tensorlbm_b200.ai.pipeline import equilibrium_field, random_solenoidal_field

    tf, tfo = _import_reference_package()

    def timed(fn):
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / 1e3

    cells = n ** 3
    tau = 0.53
    f0 = equilibrium_field(random_solenoidal_field(n, 4.0, 0.05, 11, dev))
    out = {"grid": n, "tau": tau, "steps": steps}
    for storage, dt, bpc in (("f32", torch.float32, 152), ("f16", torch.float16, 76), ("bf16", torch.bfloat16, 76)):
        a = tf.triton_collide(f0, tau).to(dt)
        b = torch.empty_like(a)

        def ref_steps(k):
            nonlocal a, b
            for _ in range(k):
                tf.triton_fused(a, tau, out=b)
                a, b = b, a

        ref_steps(warmup)
        s = LBMSolver("D3Q19", (n, n, n), tau, "bgk", device=dev, storage=storage).load(f0)
        s.step(warmup)
        if storage == "f32":
            torch.cuda.synchronize(dev)
            out["f32_state_max_rel_diff_after_warmup"] = float((s.state - a).abs().max() / a.abs().max())
        t_ref = timed(lambda: ref_steps(steps))
        t_us = timed(lambda: s.step(steps))
        out[storage] = {"reference_mlups": round(cells * steps / t_ref / 1e6, 1),
                        "ours_mlups": round(cells * steps / t_us / 1e6, 1),
                        "speedup": round(t_ref / t_us, 2),
                        "reference_roofline_frac": round(bpc * cells * steps / t_ref / 1e9 / peak, 4),
                        "ours_roofline_frac": round(bpc * cells * steps / t_us / 1e9 / peak, 4)}
        if storage != "f32":
            # like for like: this library's triton_fused drop-in on the same plain half storage
            from tensorlbm_b200 import triton_fused as ours_tf

            pa, pb = a.clone(), torch.empty_like(a)

            def plain_steps(k):
                nonlocal pa, pb
                for _ in range(k):
                    ours_tf.triton_fused(pa, tau, out=pb)
                    pa, pb = pb, pa

            plain_steps(warmup)
            t_plain = timed(lambda: plain_steps(steps))
            out[storage]["ours_plain_storage_mlups"] = round(cells * steps / t_plain / 1e6, 1)
            out[storage]["speedup_plain_storage"] = round(t_ref / t_plain, 2)
            del pa, pb
        del a, b, s
        torch.cuda.empty_cache()

    # obstacle + Smagorinsky + drag; sphere radius for an 8 % solid fraction
    r = n * (0.08 * 3.0 / (4.0 * math.pi)) ** (1.0 / 3.0)
    i = torch.arange(n, device=dev, dtype=torch.float32)
    zz, yy, xx = torch.meshgrid(i, i, i, indexing="ij")
    c = (n - 1) / 2.0
    solid = ((xx - c) ** 2 + (yy - c) ** 2 + (zz - c) ** 2) <= r * r
    del zz, yy, xx
    nu = (tau - 0.5) / 3.0
    a = f0.clone()
    b = torch.empty_like(a)
    mask8 = solid.to(torch.int8)
    fbuf = [torch.zeros((), dtype=torch.float32, device=dev) for _ in range(3)]

    def ref_obst(k):
        nonlocal a, b
        for _ in range(k):
            for t in fbuf:
                t.zero_()
            tfo.triton_fused_obstacle_xfar_les(a, nu, mask8, 0.17, 1.0, collision="BGK", out=b,
                                               fx_buf=fbuf[0], fy_buf=fbuf[1], fz_buf=fbuf[2])
            a, b = b, a

    ref_obst(warmup)
    t_ref = timed(lambda: ref_obst(steps))
    del a, b
    s = LBMSolver("D3Q19", (n, n, n), tau, "smagorinsky", device=dev, c_smag=0.17, obstacle_mask=solid,
                  track_force=True).load(f0)
    s.step(warmup)
    t_us = timed(lambda: s.step(steps))
    out["obstacle_smagorinsky_f32"] = {"solid_fraction": round(float(solid.float().mean()), 4),
                                       "reference_mlups": round(cells * steps / t_ref / 1e6, 1),
                                       "ours_mlups": round(cells * steps / t_us / 1e6, 1),
                                       "speedup": round(t_ref / t_us, 2),
                                       "ours_roofline_frac": round(152 * cells * steps / t_us / 1e9 / peak, 4)}
    del s, f0, solid, mask8
    torch.cuda.empty_cache()
    return out


def max_over_ranks(t: float, device) -> float:
    """The slowest rank's time (every rank takes part; a no-op on one process)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return t
    tt = torch.tensor([t], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt)


def whole_job_mlups(world: int, cells_per_rank: int, steps: int, t_max: float) -> float:
    """Cell updates of all ranks (one slab each) per second of the slowest rank, in millions."""
    return world * cells_per_rank * steps / t_max / 1e6


def run_ours(args) -> None:
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    peak, peak_kind = _peaks()
    cells = NX * NY * NZ
    bpc = 2 * 19 * 4

    # ---- headline: D3Q19 MRT float32, one fused kernel per step, FP64 drag ----
    s, obst = _make_headline(torch, dev, world, rank)
    f0 = _initial_state(torch, dev, "D3Q19", obst)
    s.load(f0)                          # N > 1: this rank's owned planes, ghosts exchanged
    force = torch.zeros(3, dtype=torch.float64, device=dev)
    for _ in range(args.warmup):
        s._launch(s._buf[s._cur], s._buf[1 - s._cur], force)
        s._cur ^= 1
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    cur = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        e0.record(cur)
        for _ in range(args.steps):
            s._launch(s._buf[s._cur], s._buf[1 - s._cur], force)
            s._cur ^= 1
        if world > 1:
            s.synchronize()             # the last step's halo has landed
        e1.record(cur)
        torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3, dev)
    s.steps_done += args.steps + args.warmup
    drag = float(force[0])
    finite = not s.nonfinite_seen()
    value = whole_job_mlups(world, cells, args.steps, t)
    per_launch = t / args.steps
    achieved = bpc * cells / per_launch / 1e9
    del s
    torch.cuda.empty_cache()

    # ---- end to end through the public API with host buffers ----
    from tensorlbm_b200 import LBMSolver

    host_f0 = f0.cpu().pin_memory()
    del f0
    host_out = torch.empty(host_f0.shape, dtype=torch.float32).pin_memory()
    host_drag = torch.empty((args.steps, 3), dtype=torch.float64).pin_memory()
    if world == 1:
        s2 = LBMSolver("D3Q19", (NZ, NY, NX), TAU, "mrt", device=dev, obstacle_mask=obst, u_in=U_IN, rho_out=1.0)
    else:
        s2, _ = _make_headline(torch, dev, world, rank)
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    drag_buf = torch.zeros((args.steps, 3), dtype=torch.float64, device=dev)
    e2.record(cur)
    f_dev = host_f0.to(dev, non_blocking=True)
    s2.load(f_dev)
    for k in range(args.steps):
        s2._launch(s2._buf[s2._cur], s2._buf[1 - s2._cur], drag_buf[k])
        s2._cur ^= 1
        s2.steps_done += 1
        host_drag[k].copy_(drag_buf[k], non_blocking=True)  # the step's result, read back every step
    host_out.copy_(s2.f, non_blocking=True)
    e3.record(cur)
    torch.cuda.synchronize(dev)
    t_e2e = max_over_ranks(e2.elapsed_time(e3) / 1e3, dev)
    e2e_value = whole_job_mlups(world, cells, args.steps, t_e2e)
    state_bytes = host_f0.numel() * 4
    del s2, f_dev
    torch.cuda.empty_cache()

    # ---- variants on the same grid (rank 0 device only, N=1 semantics) ----
    variants = {}
    wanted = set(args.variants.split(",")) if args.variants != "all" else None

    def want(name):
        return not args.no_variants and (wanted is None or name in wanted)

    if want("d3q27_cumulant_f32"):
        variants["d3q27_cumulant_f32"] = _variant(torch, dev, "D3Q27", "cumulant", "f32", max(args.steps // 2, 3),
                                                  args.warmup, 2 * 27 * 4, peak)
    if want("d3q19_mrt_f16_shifted"):
        variants["d3q19_mrt_f16_shifted"] = _variant(torch, dev, "D3Q19", "mrt", "f16", args.steps, args.warmup,
                                                     2 * 19 * 2, peak)
    if want("d3q19_bgk_f32"):
        variants["d3q19_bgk_f32"] = _variant(torch, dev, "D3Q19", "bgk", "f32", args.steps, args.warmup, bpc, peak)
    if want("d3q19_rlbm_f32"):
        # regularised BGK (solver3d.py:342), bit-exact arithmetic, same channel
        variants["d3q19_rlbm_f32"] = _variant(torch, dev, "D3Q19", "rlbm", "f32", args.steps, args.warmup, bpc, peak)
    for name, lat, coll, st, bpc_v, steps_v in (
            ("d3q19_bgk_f16_shifted", "D3Q19", "bgk", "f16", 2 * 19 * 2, args.steps),
            ("d3q19_bgk_bf16_shifted", "D3Q19", "bgk", "bf16", 2 * 19 * 2, args.steps),
            ("d3q27_cumulant_f16_shifted", "D3Q27", "cumulant", "f16", 2 * 27 * 2, max(args.steps // 2, 3))):
        if want(name):
            variants[name] = _variant(torch, dev, lat, coll, st, steps_v, args.warmup, bpc_v, peak)
    # the D3Q27 cumulants away from the unit-rate special case: the general
    # moment transform (non-unit omega_b / omega_odd / omega_even) and Geier's
    # cumulant (cumulant.py:935, :1050)
    general = dict(omega_b=1.2, omega_odd=1.5, omega_even=1.5)
    for name, coll, st, bpc_v, rates in (
            ("d3q27_cumulant_general_f32", "cumulant", "f32", 2 * 27 * 4, general),
            ("d3q27_cumulant_general_f16_shifted", "cumulant", "f16", 2 * 27 * 2, general),
            ("d3q27_cumulant_geier_f32", "cumulant_geier", "f32", 2 * 27 * 4, {})):
        if want(name):
            variants[name] = _variant(torch, dev, "D3Q27", coll, st, max(args.steps // 2, 3), args.warmup, bpc_v,
                                      peak, **rates)
    # half storage against float32 for the same collision (MLUPS ratio)
    for half, full in (("d3q19_bgk_f16_shifted", "d3q19_bgk_f32"), ("d3q19_bgk_bf16_shifted", "d3q19_bgk_f32"),
                       ("d3q27_cumulant_f16_shifted", "d3q27_cumulant_f32"),
                       ("d3q27_cumulant_general_f16_shifted", "d3q27_cumulant_general_f32")):
        if half in variants and full in variants:
            variants[half]["speedup_vs_f32"] = round(variants[half]["mlups"] / variants[full]["mlups"], 3)
    if "d3q19_mrt_f16_shifted" in variants:   # against the headline (FP32 MRT, same grid, one GPU's share)
        variants["d3q19_mrt_f16_shifted"]["speedup_vs_f32"] = round(
            variants["d3q19_mrt_f16_shifted"]["mlups"] / (value / world), 3)
    for name, lat, coll, st, bpc_v in (("d3q19_mrt_f32_aa", "D3Q19", "mrt", "f32", bpc),
                                       ("d3q19_bgk_f16_shifted_aa", "D3Q19", "bgk", "f16", 2 * 19 * 2)):
        if want(name):
            variants[name] = _variant(torch, dev, lat, coll, st, args.steps, args.warmup, bpc_v, peak, "aa")
    if want("les_mlp_128_vs_smagorinsky_256"):
        variants["les_mlp_128_vs_smagorinsky_256"] = _les_variant(torch, dev, args.steps, args.warmup, peak)
    if want("d2q9_batched_512_cylinders"):
        variants["d2q9_batched_512_cylinders"] = _batched_variant(torch, dev, args.steps, peak)
    if wanted is not None and REF_TRITON in wanted and not args.no_variants:
        variants[REF_TRITON] = _reference_triton_variant(torch, dev, args.steps, args.warmup, peak)
    if wanted is not None and C2_LONG in wanted and not args.no_variants:
        variants[C2_LONG] = _c2_long_variant(torch, dev, args.long_steps, args.long_every)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(args)

    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC,
        "value": round(value, 1),
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1e3 * t / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": DATA,
        "config": workload_config(world),
        "result": {"drag_fx_last_step": drag, "finite": finite},
        "roofline": {
            "bound": "hbm",
            "achieved": round(achieved, 1),
            "peak": peak,
            "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "peak_kind": peak_kind,
            "frac_of_spec_8tbs": round(achieved / SPEC_HBM_GBS, 4),
            "bytes_per_cell": bpc,
            "traffic": _traffic(WORKLOAD),
        },
        "e2e": {
            "value": round(e2e_value, 1),
            "unit": "MLUPS",
            "h2d_bytes_per_step": int(round(state_bytes / args.steps)),
            "d2h_bytes_per_step": int(round((state_bytes + args.steps * 24) / args.steps)),
            "what": "pinned host f0 -> device, load (collision pass), K fused steps through LBMSolver with the "
                    "float64 drag copied to pinned host memory every step, final TensorLBM-phase f -> host",
        },
        "gpu_launches": args.steps * (3 if world > 1 else 1),
        "clocks": clocks.summary(),
        "variants": variants,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# CPU baseline / reference arm: TensorLBM's own torch chain on the host cores
# ---------------------------------------------------------------------------

CPU_SAMPLE_STEPS_MAX = 30      # timed steps of the CPU sample (both arms), fewer if --steps is smaller
CPU_SAMPLE_BUDGET_S = 90.0     # and no more timed seconds than this


def _reference_chain(nzs: int):
    """The config-2 chain of TensorLBM itself (unmodified, baseline/_ref) on a
    512 x 256 x nzs z-slab of the channel (sphere centred in the slab):
    collide_mrt3d -> stream3d -> compute_obstacle_forces_3d ->
    zou_he_inlet_velocity_3d -> zou_he_outlet_pressure_3d ->
    bounce_back_cells_3d(sphere), the order of d3q27_sphere_flow.py:246-256
    with the D3Q19 MRT operators.  Returns (step, f0)."""
    import torch

    from baseline import reference

    reference.import_reference()
    from tensorlbm.boundaries3d import (bounce_back_cells_3d, sphere_mask, zou_he_inlet_velocity_3d,
                                        zou_he_outlet_pressure_3d)
    from tensorlbm.d3q19 import equilibrium3d
    from tensorlbm.obstacles import compute_obstacle_forces_3d
    from tensorlbm.solver3d import collide_mrt3d, stream3d

    cpu = torch.device("cpu")
    obst = sphere_mask(NX, NY, nzs, CX, CY, nzs / 2, D / 2, cpu)
    ux = torch.full((nzs, NY, NX), U_IN)
    ux[obst] = 0.0
    z = torch.zeros_like(ux)
    f0 = equilibrium3d(torch.ones_like(ux), ux, z, z)

    def step(f):
        f = collide_mrt3d(f, TAU)
        f = stream3d(f)
        fx, _, _ = compute_obstacle_forces_3d(f, obst)
        f = zou_he_inlet_velocity_3d(f, U_IN)
        f = zou_he_outlet_pressure_3d(f, 1.0)
        f = bounce_back_cells_3d(f, obst)
        return f, fx

    return step, f0


def _oracle_chain(nzs: int):
    """The oracle's restatement of the same chain (used when TensorLBM is not installed)."""
    import numpy as np

    from oracle import lbm as O

    obst = O.sphere_mask(NX, NY, nzs, CX, CY, nzs / 2, D / 2)
    ux = np.full((nzs, NY, NX), U_IN, np.float32)
    ux[obst] = 0.0
    z = np.zeros_like(ux)
    f0 = O.equilibrium(19, np.ones_like(ux), ux, z, z)
    return (lambda f: O.channel_step(f, TAU, U_IN, 1.0, None, obst, "mrt")), f0


def cpu_sample(args) -> dict:
    """Time the CPU chain of the headline workload on a z-slab sample: TensorLBM's
    torch operators with every host core (kind "reference"), or the oracle port
    on one core when TensorLBM is not installed (kind "port").  The same slab
    and step count serve the cpu_baseline of our arm and the reference arm."""
    from baseline import reference

    nzs = args.cpu_slab
    want = max(1, min(args.steps, CPU_SAMPLE_STEPS_MAX))
    import contextlib

    with contextlib.ExitStack() as stack:
        if reference.available():
            import torch

            threads_before = torch.get_num_threads()
            torch.set_num_threads(os.cpu_count() or 1)
            stack.callback(torch.set_num_threads, threads_before)
            step, f = _reference_chain(nzs)
            used, kind = torch.get_num_threads(), "reference"
            what = ("TensorLBM's own torch CPU operators (unmodified, baseline/_ref): collide_mrt3d -> stream3d -> "
                    "compute_obstacle_forces_3d -> zou_he_inlet_velocity_3d -> zou_he_outlet_pressure_3d -> "
                    "bounce_back_cells_3d")
        else:
            from threadpoolctl import threadpool_limits

            stack.enter_context(threadpool_limits(1))
            step, f = _oracle_chain(nzs)
            used, kind = 1, "port"
            what = "numpy restatement of the same chain (oracle/), one core"
        f, _ = step(f)                              # warm-up (index caches, allocator)
        done, t = 0, 0.0
        while done < want and t < CPU_SAMPLE_BUDGET_S:
            t0 = time.perf_counter()
            f, _ = step(f)
            t += time.perf_counter() - t0
            done += 1
    cells = NX * NY * nzs
    return {"value": round(cells * done / t / 1e6, 3), "unit": "MLUPS", "cores": used, "kind": kind,
            "host_cpus": os.cpu_count(),
            "sample": f"one {NX}x{NY}x{nzs} z-slab of the sphere channel (sphere centred in the slab, periodic "
                      f"y/z), 1 warm-up step, {done} timed step(s) ({t:.1f} s): {what}"}


def run_reference(args) -> None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sample = cpu_sample(args)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": sample["value"],
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": DATA,
        "config": workload_config(world),
        "cpu_baseline": sample,
        "e2e": {"value": sample["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "TensorLBM is a pure-Python torch package; its CPU path runs here on a bounded z-slab sample of "
                "the workload (see cpu_baseline.sample), on every host core",
    }
    print(json.dumps(line))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--variants", default="all",
                    help="comma list of variants to run (d3q27_cumulant_f32, d3q27_cumulant_f16_shifted, "
                         "d3q19_mrt_f16_shifted, d3q19_bgk_f32, d3q19_rlbm_f32, d3q19_bgk_f16_shifted, "
                         "d3q19_bgk_bf16_shifted, "
                         "les_mlp_128_vs_smagorinsky_256, d2q9_batched_512_cylinders) or 'all'")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-slab", type=int, default=16, help="z-planes of the CPU sample slab")
    ap.add_argument("--long-steps", type=int, default=20000, help="steps of the c2_20k_vs_fp64 variant")
    ap.add_argument("--long-every", type=int, default=2000, help="comparison interval of c2_20k_vs_fp64")
    ap.add_argument("--grid", default=None,
                    help="nx,ny,nz of a smaller channel (profiling only; the sphere keeps its size, centred)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.grid:
        global NX, NY, NZ, CX, CY, CZ, WORKLOAD
        NX, NY, NZ = (int(v) for v in args.grid.split(","))
        CX, CY, CZ = NY // 2, NY // 2, NZ // 2
        WORKLOAD = f"d3q19_mrt_sphere_channel_{NX}x{NY}x{NZ}"
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
