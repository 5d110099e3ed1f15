"""Forced isotropic turbulence: DNS -> filtered training data -> learned
closure -> LES comparisons (ai/pipeline.py:222 run_ai_les_pipeline is the 2-D
original).

Everything is in lattice units of the DNS grid (dx = dt = 1), D3Q19 MRT (the
DNS) or BGK with tau_eff (the LES) with the exact-difference linear (Lundgren)
forcing F = A rho u at constant power: every `force_every` steps
A = epsilon / (2 K) from the current kinetic energy K, so that the injection
rate is the target dissipation whatever the integral scale does (Carroll &
Blanquart 2013).  A grid filtered by a factor r uses dx_r = dt_r = r (acoustic
scaling): nu_r = nu / r, epsilon_r = epsilon r, and one filtered step covers r
DNS steps.  ``HITConfig.les`` lists the LES grids: every grid but the last
runs the learned closure (its nu_t scale calibrated on that grid), Smagorinsky
and no model; the last runs Smagorinsky, the fine-grid reference (a single grid
runs all three).

The a-posteriori error of an LES is mean |ln(E_LES(k) / E_fDNS(k))| over the
shells 1 <= k <= min(m/2, 21), where E_fDNS is the spectrum of the DNS
block-filtered (mean over r^3 cells) to the LES grid m = n / r, both averaged
over the comparison window's spectra.

Run as a module for the full experiment:

    python -m tensorlbm_b200.ai.pipeline --dns 512 --out results/

It writes ``hit_les.json`` (spectra, dissipation, Re_lambda, errors, wall
times) and ``closure.npz`` (the trained network)."""

from __future__ import annotations

import argparse
import json
import math
import pathlib
import time
from dataclasses import asdict, dataclass

import numpy as np
import torch

from .. import LBMSolver
from ..d3q19 import equilibrium3d, macroscopic3d
from .dataset import filtered_moments, les_samples
from .inference import LearnedLESSolver
from .model import EddyViscosityMLP3D
from .train import TrainConfig, train_eddy_viscosity_model3d

C_SMAG = 0.17


# ---------------------------------------------------------------------------
# initial field and spectra
# ---------------------------------------------------------------------------


def random_solenoidal_field(n: int, k0: float, u_rms: float, seed: int, device) -> torch.Tensor:
    """(3, n, n, n) float32 divergence-free field with E(k) ~ k^4 exp(-2 (k/k0)^2):
    complex Gaussian modes of amplitude sqrt(E / (4 pi k^2)) on the rfft half
    space, projected onto k-perpendicular, inverse FFT, scaled to u_rms
    (the construction of benchmarks/pending/dit_turbulence/run.py:95-126,
    generated here on the GPU from a seeded torch generator)."""
    g = torch.Generator(device=device).manual_seed(seed)
    kx = torch.fft.rfftfreq(n, d=1.0 / n, device=device)
    ky = torch.fft.fftfreq(n, d=1.0 / n, device=device)
    kz = torch.fft.fftfreq(n, d=1.0 / n, device=device)
    KZ, KY, KX = torch.meshgrid(kz, ky, kx, indexing="ij")
    K2 = KX * KX + KY * KY + KZ * KZ
    K = torch.sqrt(K2)
    spec = K ** 4 * torch.exp(-2.0 * (K / k0) ** 2)
    amp = torch.where(K > 0, torch.sqrt(spec / (4.0 * math.pi * K2.clamp_min(1e-30))), torch.zeros_like(K))
    uh = []
    for _ in range(3):
        re = torch.randn(KX.shape, generator=g, device=device)
        im = torch.randn(KX.shape, generator=g, device=device)
        uh.append(torch.complex(re, im) * amp)
    kdotu = KX * uh[0] + KY * uh[1] + KZ * uh[2]
    fac = torch.where(K2 > 0, kdotu / K2.clamp_min(1e-30), torch.zeros_like(kdotu))
    uh = [uh[0] - KX * fac, uh[1] - KY * fac, uh[2] - KZ * fac]
    del KX, KY, KZ, K2, K, spec, amp, kdotu, fac
    u = torch.stack([torch.fft.irfftn(c, s=(n, n, n)) for c in uh]).float()
    u *= u_rms / torch.sqrt(torch.mean(u.double() ** 2)).float()
    return u


def energy_spectrum(u: torch.Tensor) -> torch.Tensor:
    """E(k), k = 0 .. round(sqrt(3) n / 2), float64, of a periodic (3, n, n, n)
    field; sum_k E(k) = <|u|^2> / 2 (conventions of dit_turbulence/run.py:158-177)."""
    n = u.shape[-1]
    dev = u.device
    kx = torch.fft.rfftfreq(n, d=1.0 / n, device=dev)
    ky = torch.fft.fftfreq(n, d=1.0 / n, device=dev)
    kz = torch.fft.fftfreq(n, d=1.0 / n, device=dev)
    KZ, KY, KX = torch.meshgrid(kz, ky, kx, indexing="ij")
    idx = torch.round(torch.sqrt(KX * KX + KY * KY + KZ * KZ)).long().reshape(-1)
    w = torch.where((KX > 0) & (KX < n // 2), 2.0, 1.0).reshape(-1).double()
    e = torch.zeros(int(idx.max()) + 1, dtype=torch.float64, device=dev)
    for c in range(3):
        uh = torch.fft.rfftn(u[c].float(), norm="ortho")
        e.scatter_add_(0, idx, 0.5 * (uh.real.double() ** 2 + uh.imag.double() ** 2).reshape(-1) * w)
    return e / n ** 3


def dissipation_from_spectrum(e: torch.Tensor, n: int, nu: float) -> float:
    """epsilon = 2 nu sum_k (2 pi k / n)^2 E(k) in the grid's lattice units."""
    k = torch.arange(e.numel(), dtype=torch.float64, device=e.device)
    return float(2.0 * nu * torch.sum((2.0 * math.pi * k / n) ** 2 * e))


def velocity_of(f: torch.Tensor, force_lin: float) -> torch.Tensor:
    """(3, ...) physical velocity m / rho (1 + A/2) of D3Q19 populations."""
    _, ux, uy, uz = macroscopic3d(f)
    return torch.stack([ux, uy, uz]) * (1.0 + 0.5 * force_lin)


def equilibrium_field(u: torch.Tensor, rho: torch.Tensor | None = None) -> torch.Tensor:
    if rho is None:
        rho = torch.ones_like(u[0])
    return equilibrium3d(rho.contiguous(), u[0].contiguous(), u[1].contiguous(), u[2].contiguous())


# ---------------------------------------------------------------------------
# configuration
# ---------------------------------------------------------------------------


@dataclass
class HITConfig:
    dns: int = 512                  # DNS grid (cells per side)
    les: tuple = (128, 256)         # LES grids (filtered by dns // les)
    u_rms: float = 0.05             # initial rms velocity (Ma = 0.087)
    k0: float = 4.0                 # initial spectrum peak
    re_lambda: float = 100.0        # target Taylor Reynolds number
    seed: int = 20261203
    spinup_turnovers: float = 15.0  # DNS turnovers before the first training snapshot
    snapshots: int = 4              # training snapshots
    snapshot_gap_turnovers: float = 1.0
    window_turnovers: float = 3.0   # LES / DNS comparison window
    spectra_per_window: int = 8
    train_epochs: int = 12
    train_batch: int = 16384
    max_samples_per_grid: int = 3_000_000
    chunk: int = 50                 # steps per CUDA graph replay
    dns_collision: str = "mrt"      # BGK diverges at the DNS's tau ~ 0.515
    calibration: tuple = (1.0, 0.7, 0.5, 0.35, 0.25, 0.15, 0.1, 0.05)  # candidate nu_t scale factors

    force_every: int = 100          # steps between updates of the constant-power force

    @property
    def integral_scale(self) -> float:
        # integral scale assumed when choosing epsilon: 0.1 of the box (between
        # the 0.066 measured after 6 turnovers from the k0 = 4 start and the
        # asymptotic 0.19 of linear forcing, Rosales & Meneveau 2005)
        return 0.1 * self.dns

    @property
    def eps(self) -> float:
        # target dissipation = injected power, epsilon ~ 0.5 u'^3 / L
        return 0.5 * self.u_rms ** 3 / self.integral_scale

    @property
    def force_lin(self) -> float:
        # initial A = epsilon / (2 K), K = 1.5 u'^2
        return self.eps / (3.0 * self.u_rms ** 2)

    @property
    def nu(self) -> float:
        # Re_lambda = u' lambda / nu with lambda^2 = 15 nu u'^2 / epsilon
        return 15.0 * self.u_rms ** 4 / (self.re_lambda ** 2 * self.eps)

    @property
    def tau(self) -> float:
        return 3.0 * self.nu + 0.5

    @property
    def turnover_steps(self) -> int:
        return int(round(self.integral_scale / self.u_rms))


def tau_on(cfg: HITConfig, factor: int) -> float:
    """Molecular tau on a grid filtered by `factor` (nu_r = nu / r)."""
    return 3.0 * cfg.nu / factor + 0.5


def kinetic_energy(state: torch.Tensor) -> float:
    """K = <|u|^2> / 2 of D3Q19 populations."""
    _, ux, uy, uz = macroscopic3d(state)
    return 0.5 * float((ux.double() ** 2 + uy.double() ** 2 + uz.double() ** 2).mean())


def run_forced(solver, steps: int, eps: float, every: int, chunk: int) -> float:
    """Advance `steps` steps at constant injected power eps (grid units): the
    force is reset to A = eps / (2 K) every `every` steps.  Returns the last A."""
    a = 0.0
    done = 0
    while done < steps:
        k = kinetic_energy(solver.state)
        if not (math.isfinite(k) and k > 0.0):
            raise RuntimeError("the flow diverged")
        a = min(eps / (2.0 * k), 0.05)
        solver.set_force_lin(a)
        m = min(every, steps - done)
        solver.run(m, chunk=chunk)
        done += m
    return a


# ---------------------------------------------------------------------------
# the experiment
# ---------------------------------------------------------------------------


def _timed(fn, device) -> float:
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    fn()
    e1.record()
    torch.cuda.synchronize(device)
    return e0.elapsed_time(e1) / 1e3


def _spec_error(e_les: np.ndarray, e_ref: np.ndarray, kmax: int) -> float:
    """mean |log(E_les / E_ref)| over shells 1..kmax."""
    a = np.asarray(e_les[1:kmax + 1], np.float64)
    b = np.asarray(e_ref[1:kmax + 1], np.float64)
    return float(np.mean(np.abs(np.log(np.maximum(a, 1e-300) / np.maximum(b, 1e-300)))))


def collect_samples(cfg: HITConfig, moms: dict, model: EddyViscosityMLP3D | None):
    """Training samples of every stored filtered field (moms: LES grid ->
    list of filtered moments); with a model, tau_eff is that model's own
    prediction (self-consistent pass), else Smagorinsky."""
    xs, ts, ws = [], [], []
    g = torch.Generator(device="cpu").manual_seed(cfg.seed + 7)
    for grid, fields in moms.items():
        per_field = cfg.max_samples_per_grid // max(len(fields), 1)
        for mom in fields:
            tau0 = tau_on(cfg, cfg.dns // grid)
            nu_hat = None
            if model is not None:
                x0, _, _ = les_samples(mom, tau0, C_SMAG)
                nu_hat = model.nu_t(x0)
                del x0
            x, t, w = les_samples(mom, tau0, C_SMAG, nu_hat)
            n = x.shape[0]
            if n > per_field:
                sel = torch.randperm(n, generator=g)[:per_field].to(x.device)
                x, t, w = x[sel], t[sel], w[sel]
            xs.append(x)
            ts.append(t)
            ws.append(w)
    return torch.cat(xs), torch.cat(ts), torch.cat(ws)


def a_priori(model: EddyViscosityMLP3D, x: torch.Tensor, t: torch.Tensor, w: torch.Tensor) -> dict:
    """Weighted MSE of nu_t against nu* (the training objective) for the network
    and for Smagorinsky (nu_s = (tau_s - tau0) / 3, feature 6), plus the
    weighted subgrid dissipation sum w nu relative to sum w nu*."""
    wn = w / w.mean()
    nu_mlp = model.nu_t(x)
    nu_smag = x[:, 6] / 3.0
    scale = model.nu_scale ** 2
    d_true = float((wn * t).mean())
    return {"mse_mlp": float((wn * (nu_mlp - t) ** 2).mean() / scale),
            "mse_smagorinsky": float((wn * (nu_smag - t) ** 2).mean() / scale),
            "dissipation_ratio_mlp": float((wn * nu_mlp).mean()) / d_true,
            "dissipation_ratio_smagorinsky": float((wn * nu_smag).mean()) / d_true}


def run(cfg: HITConfig, out_dir: pathlib.Path, device="cuda:0", log=print) -> dict:
    dev = torch.device(device)
    out_dir = pathlib.Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    res: dict = {"config": asdict(cfg), "derived": {"eps_target": cfg.eps, "force_lin_initial": cfg.force_lin,
                                                    "nu": cfg.nu, "tau": cfg.tau,
                                                    "turnover_steps": cfg.turnover_steps}}
    n = cfg.dns
    # ---- DNS spin-up ----------------------------------------------------
    u0 = random_solenoidal_field(n, cfg.k0, cfg.u_rms, cfg.seed, dev)
    dns = LBMSolver("D3Q19", (n, n, n), cfg.tau, cfg.dns_collision, device=dev, force_lin=cfg.force_lin)
    dns.load(equilibrium_field(u0))
    del u0
    torch.cuda.empty_cache()
    spin = int(cfg.spinup_turnovers * cfg.turnover_steps)
    a_now = [cfg.force_lin]

    def advance(steps):
        a_now[0] = run_forced(dns, steps, cfg.eps, cfg.force_every, cfg.chunk)

    t_spin = _timed(lambda: advance(spin), dev)
    res["dns_mlups"] = n ** 3 * spin / t_spin / 1e6
    log(f"DNS {n}^3 spin-up {spin} steps in {t_spin:.1f} s ({res['dns_mlups']:.0f} MLUPS)")

    def dns_stats():
        f = dns.f
        u = velocity_of(f, a_now[0])
        e = energy_spectrum(u)
        del u
        eps = dissipation_from_spectrum(e, n, cfg.nu)
        k_e = float(e.sum())
        up = math.sqrt(2.0 * k_e / 3.0)
        lam = math.sqrt(15.0 * cfg.nu * up * up / max(eps, 1e-300))
        return f, e, {"kinetic_energy": k_e, "u_prime": up, "epsilon": eps, "lambda": lam,
                      "re_lambda": up * lam / cfg.nu, "eta": (cfg.nu ** 3 / max(eps, 1e-300)) ** 0.25,
                      "force_lin": a_now[0]}

    # ---- training snapshots ------------------------------------------------
    moms: dict = {g: [] for g in cfg.les}
    gap = max(1, int(cfg.snapshot_gap_turnovers * cfg.turnover_steps))
    stats = []
    e = None
    for s in range(cfg.snapshots):
        if s:
            advance(gap)
        f, e, st = dns_stats()
        stats.append(st)
        for g in cfg.les:
            moms[g].append(filtered_moments(f, n // g, a_now[0]))
        del f
        torch.cuda.empty_cache()
        log(f"snapshot {s}: Re_lambda {st['re_lambda']:.1f}, u' {st['u_prime']:.4f}, eps {st['epsilon']:.3e}")
    res["dns_snapshots"] = stats
    res["dns_spectrum"] = e.cpu().numpy().tolist()
    if not math.isfinite(stats[-1]["kinetic_energy"]):
        raise RuntimeError("the DNS diverged")

    # ---- training (two passes: Smagorinsky tau, then the model's own tau) --
    model = EddyViscosityMLP3D(dev, seed=cfg.seed)
    x, t, w = collect_samples(cfg, moms, None)
    t0 = time.time()
    h1 = train_eddy_viscosity_model3d(model, x, t, w, TrainConfig(epochs=cfg.train_epochs, batch=cfg.train_batch,
                                                                    seed=cfg.seed))
    x, t, w = collect_samples(cfg, moms, model)
    h2 = train_eddy_viscosity_model3d(model, x, t, w, TrainConfig(epochs=max(2, cfg.train_epochs // 2),
                                                                    batch=cfg.train_batch, lr=5e-4, lr_final=5e-5,
                                                                    seed=cfg.seed + 1))
    torch.cuda.synchronize(dev)
    res["training"] = {"samples": int(x.shape[0]), "seconds": time.time() - t0, "pass1": h1, "pass2": h2,
                       "nu_scale": model.nu_scale}
    res["a_priori"] = a_priori(model, x, t, w)
    del x, t, w
    log(f"trained on {res['training']['samples']} samples: a-priori {res['a_priori']}")

    # ---- comparison window: filtered DNS spectra ------------------------------
    window = int(cfg.window_turnovers * cfg.turnover_steps)
    init = {g: moms[g][-1] for g in cfg.les}   # LES initial states = filtered DNS now
    every = max(1, window // cfg.spectra_per_window)
    dns_spec = {g: [] for g in cfg.les}
    dns_eps = []
    for _ in range(cfg.spectra_per_window):
        advance(every)
        f, _e, st = dns_stats()
        dns_eps.append(st["epsilon"])
        for g in cfg.les:
            mom = filtered_moments(f, n // g, a_now[0])
            dns_spec[g].append(energy_spectrum(mom[1:4]).cpu().numpy())
        del f
    del dns
    torch.cuda.empty_cache()
    res["dns_window"] = {"epsilon_mean": float(np.mean(dns_eps))}

    # ---- LES runs ------------------------------------------------------------
    def les_run(kind, m, mom, nsamples, steps_per):
        """One LES from the filtered state `mom`; spectra after every steps_per
        steps.  Returns (spectra, device seconds, finite, fallback cells per step)."""
        r = n // m
        tau0 = tau_on(cfg, r)
        eps_r = cfg.eps * r
        a_r = [a_now[0] * r]
        f0 = equilibrium_field(mom[1:4] / (1.0 + 0.5 * a_now[0]), mom[0])
        if kind == "mlp":
            sol = LearnedLESSolver((m, m, m), tau0, model, force_lin=a_r[0], c_s=C_SMAG, device=dev).load(f0)
        else:
            sol = LBMSolver("D3Q19", (m, m, m), tau0, "smagorinsky" if kind == "smag" else "bgk", device=dev,
                            c_smag=C_SMAG, force_lin=a_r[0]).load(f0)
        every_r = max(10, cfg.force_every // r)
        specs, secs, finite = [], 0.0, True

        def advance_les():
            a_r[0] = run_forced(sol, steps_per, eps_r, every_r, cfg.chunk)

        for _ in range(nsamples):
            try:
                secs += _timed(advance_les, dev)
            except RuntimeError:
                finite = False
                break
            state = sol.state if kind == "mlp" else sol.f
            specs.append(energy_spectrum(velocity_of(state, a_r[0])).cpu().numpy())
        finite = finite and not sol.nonfinite_seen() and len(specs) > 0
        fb = int(sol.fallback.item()) / max(sol.steps_done, 1) if kind == "mlp" else None
        del sol
        torch.cuda.empty_cache()
        return specs, secs, finite, fb

    # in-the-loop calibration of the network's scale on the TRAINING window, on
    # every grid that runs the closure: the LES starts from the first training
    # snapshot and is compared with the filtered spectra of the later training
    # snapshots (not the comparison window)
    closure_grids = list(cfg.les[:-1]) if len(cfg.les) > 1 else list(cfg.les)
    base_scale = model.nu_scale
    calib, alpha_of = {}, {}
    for m in closure_grids:
        r = n // m
        train_ref = np.mean([energy_spectrum(mm[1:4]).cpu().numpy() for mm in moms[m][1:]], axis=0)
        errs = {}
        if cfg.snapshots > 1:
            for alpha in cfg.calibration:
                model.nu_scale = base_scale * alpha
                model.invalidate()
                specs, _, fin, _ = les_run("mlp", m, moms[m][0], cfg.snapshots - 1, max(1, gap // r))
                err = _spec_error(np.mean(specs, axis=0), train_ref, min(m // 2, 21)) if fin else float("inf")
                errs[str(alpha)] = err
                log(f"calibration {m}^3 alpha {alpha}: error {err:.4f}")
        calib[str(m)] = errs
        alpha_of[m] = float(min(errs, key=errs.get)) if errs else 1.0
    alpha_best = alpha_of[closure_grids[0]]
    res["calibration"] = {"errors": calib[str(closure_grids[0])], "alpha": alpha_best,
                          "per_grid": {str(m): {"errors": calib[str(m)], "alpha": alpha_of[m]} for m in closure_grids}}
    model.nu_scale = base_scale * alpha_best
    model.invalidate()
    model.save(out_dir / "closure.npz")

    plan = []
    for m in closure_grids:
        plan += [("mlp", m, "mlp", alpha_of[m]), ("mlp_uncalibrated", m, "mlp", 1.0), ("smagorinsky", m, "smag", None),
                 ("no_model", m, "bgk", None)]
    plan.append(("smagorinsky", cfg.les[-1], "smag", None))
    runs: dict = {}
    for name, m, kind, alpha in plan:
        if f"{name}_{m}" in runs:
            continue
        if kind == "mlp":
            model.nu_scale = base_scale * alpha
            model.invalidate()
        r = n // m
        steps_per = max(1, every // r)
        specs, secs, finite, fb = les_run(kind, m, init[m], cfg.spectra_per_window, steps_per)
        if not specs:
            specs = [np.full(len(dns_spec[m][0]), np.nan)]
        e_mean = np.mean(specs, axis=0)
        e_ref = np.mean(dns_spec[m], axis=0)
        kc = m // 2
        entry = {"grid": m, "tau0": tau_on(cfg, r), "steps": steps_per * cfg.spectra_per_window, "seconds": secs,
                 "mlups": m ** 3 * steps_per * cfg.spectra_per_window / max(secs, 1e-12) / 1e6,
                 "finite": finite, "spectrum": e_mean.tolist(), "filtered_dns_spectrum": e_ref.tolist(),
                 "spectrum_error_all": _spec_error(e_mean, e_ref, kc),
                 "spectrum_error_k_le_21": _spec_error(e_mean, e_ref, min(kc, 21)),
                 "kinetic_energy": float(e_mean.sum()), "filtered_dns_kinetic_energy": float(e_ref.sum())}
        if kind == "mlp":
            entry["fallback_cells_per_step"] = fb
            entry["nu_scale_factor"] = alpha
        runs[f"{name}_{m}"] = entry
        log(f"LES {name} {m}^3: err {entry['spectrum_error_all']:.4f} (k<=21 {entry['spectrum_error_k_le_21']:.4f}),"
            f" {secs:.3f} s, finite {finite}")
    model.nu_scale = base_scale * alpha_best
    model.invalidate()
    res["les"] = runs
    m0 = closure_grids[0]
    mlp_key, big_key = f"mlp_{m0}", f"smagorinsky_{cfg.les[-1]}"
    res["summary"] = {
        "mlp_les_error": runs[mlp_key]["spectrum_error_k_le_21"],
        "mlp_uncalibrated_les_error": runs[f"mlp_uncalibrated_{m0}"]["spectrum_error_k_le_21"],
        "smagorinsky_coarse_error": runs[f"smagorinsky_{m0}"]["spectrum_error_k_le_21"],
        "smagorinsky_fine_error": runs[big_key]["spectrum_error_k_le_21"],
        "no_model_coarse_error": runs[f"no_model_{m0}"]["spectrum_error_k_le_21"],
        "calibration_alpha": alpha_best,
        "wall_time_ratio_smagorinsky_fine_over_mlp": runs[big_key]["seconds"] / max(runs[mlp_key]["seconds"], 1e-12),
        "per_grid": {str(m): {k: runs[f"{k}_{m}"]["spectrum_error_k_le_21"]
                              for k in ("mlp", "mlp_uncalibrated", "smagorinsky", "no_model")} for m in closure_grids},
    }
    (out_dir / "hit_les.json").write_text(json.dumps(res))
    return res


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--dns", type=int, default=512)
    ap.add_argument("--les", type=int, nargs="+", default=[128, 256])
    ap.add_argument("--out", default="hit_les_out")
    ap.add_argument("--re-lambda", type=float, default=100.0)
    ap.add_argument("--spinup", type=float, default=15.0, help="turnovers")
    ap.add_argument("--window", type=float, default=3.0, help="turnovers")
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--snapshots", type=int, default=4)
    args = ap.parse_args(argv)
    cfg = HITConfig(dns=args.dns, les=tuple(args.les), re_lambda=args.re_lambda, spinup_turnovers=args.spinup,
                    window_turnovers=args.window, train_epochs=args.epochs, snapshots=args.snapshots)
    res = run(cfg, pathlib.Path(args.out), log=lambda s: print(s, flush=True))
    print(json.dumps(res["summary"]))


if __name__ == "__main__":
    main()
