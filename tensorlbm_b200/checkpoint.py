"""Checkpoint / resume for the fused solvers, in TensorLBM's file formats.

Two formats, both readable and writable by TensorLBM itself:

* the benchmark pair (format_version 1, ``checkpoint.py:27-136``): a
  directory with ``checkpoint_f.pt`` (the population tensor, CPU) and
  ``checkpoint_meta.json`` (step, shape, dtype, Q and caller extras);
* the unified solver-state file (format_version 2, ``checkpoint.py:138-442``):
  one atomically written ``.pt`` envelope tagged
  ``"tensorlbm-solver-checkpoint"``, holding a state dict (``populations``,
  ``step``, lattice / grid / Q, tau, dtype, obstacle mask, precision policy,
  extras), caller metadata, the torch RNG state and SHA-256 digests of the
  tensors, checked on load (fail closed).

The populations written are always the TensorLBM-phase field ``S_n`` in
absolute float32 / float64 (``LBMSolver.f``), whatever the storage format, so
a TensorLBM run can continue from them.  This library adds, under its own
keys, the raw stored state ``P_n`` in the storage format (FP16 ``(f - w)
2^14``, BF16 ``f - w``) so that its own solvers continue bit-exactly, and the
per-domain step counts of the batched runner.
"""

from __future__ import annotations

import hashlib
import json
import os
from collections.abc import Mapping
from dataclasses import dataclass
from datetime import datetime, timezone
from pathlib import Path
from typing import Any

import torch

TENSOR_FILE = "checkpoint_f.pt"
META_FILE = "checkpoint_meta.json"
PAIR_FORMAT_VERSION = 1

SOLVER_CHECKPOINT_FORMAT = "tensorlbm-solver-checkpoint"
SOLVER_CHECKPOINT_VERSION = 2
CASE_CHECKPOINT_FILENAME = "case-checkpoint.pt"

BATCH_FORMAT = "tensorlbm_b200-batch-checkpoint"
BATCH_FORMAT_VERSION = 1
BATCH_MANIFEST = "batch_manifest.json"

# storage format of this library -> TensorLBM precision-policy name (precision.py:72-158)
PRECISION_POLICY = {"f32": "FP32FP32", "f64": "FP64FP64", "f16": "FP32FP16", "bf16": None}


class CheckpointError(ValueError):
    """A checkpoint that cannot be used: missing, torn or corrupt, a digest
    mismatch, an unsupported format version or an identity mismatch."""


# ---------------------------------------------------------------------------
# format 1: tensor + JSON sidecar
# ---------------------------------------------------------------------------

def save_checkpoint(f: torch.Tensor, step: int, run_dir: Path, extra: dict[str, object] | None = None) -> Path:
    """Write ``f`` (moved to the CPU) and its step counter into ``run_dir``.

    Same files and metadata keys as TensorLBM's ``save_checkpoint``
    (``checkpoint.py:27-58``); returns ``run_dir``."""
    out = Path(run_dir)
    out.mkdir(parents=True, exist_ok=True)
    torch.save(f.detach().cpu(), out / TENSOR_FILE)
    meta: dict[str, object] = {
        "format_version": PAIR_FORMAT_VERSION,
        "step": int(step),
        "tensor_shape": list(f.shape),
        "tensor_dtype": str(f.dtype),
        "lattice_directions": int(f.shape[0]) if f.ndim >= 1 else None,
    }
    meta.update(extra or {})
    (out / META_FILE).write_text(json.dumps(meta, indent=2) + "\n", encoding="utf-8")
    return out


def load_checkpoint(run_dir: Path, device: torch.device | None = None, *,
                    expected_shape: tuple[int, ...] | None = None,
                    expected_lattice_directions: int | None = None) -> tuple[torch.Tensor, int, dict[str, object]]:
    """Read a format-1 checkpoint: returns ``(f, step, meta)``.

    Raises ``FileNotFoundError`` for a missing file and ``ValueError`` for bad
    metadata, a newer format version or a shape / Q mismatch, as TensorLBM's
    ``load_checkpoint`` does (``checkpoint.py:61-136``)."""
    src = Path(run_dir)
    tpath, mpath = src / TENSOR_FILE, src / META_FILE
    for p in (tpath, mpath):
        if not p.exists():
            raise FileNotFoundError(f"checkpoint file not found: {p}")
    f = torch.load(tpath, map_location=device or torch.device("cpu"), weights_only=True)
    try:
        meta = json.loads(mpath.read_text(encoding="utf-8"))
    except json.JSONDecodeError as exc:
        raise ValueError(f"checkpoint metadata is not valid JSON: {mpath}") from exc
    if not isinstance(meta, dict) or not all(isinstance(k, str) for k in meta):
        raise ValueError(f"checkpoint metadata must be a JSON object with string keys: {mpath}")
    version = meta.get("format_version", 0)
    if not _is_int(version):
        raise ValueError(f"checkpoint 'format_version' must be an integer: {mpath}")
    if version > PAIR_FORMAT_VERSION:
        raise ValueError(f"unsupported checkpoint format_version={version} "
                         f"(this reader handles up to {PAIR_FORMAT_VERSION}): {mpath}")
    if "step" not in meta:
        raise ValueError(f"checkpoint metadata has no 'step': {mpath}")
    if not _is_int(meta["step"]):
        raise ValueError(f"checkpoint 'step' must be an integer: {mpath}")
    if not isinstance(f, torch.Tensor):
        raise ValueError(f"checkpoint payload is not a tensor: {tpath}")
    shape_meta = meta.get("tensor_shape")
    if isinstance(shape_meta, list) and tuple(shape_meta) != tuple(f.shape):
        raise ValueError(f"checkpoint tensor shape {tuple(f.shape)} differs from its metadata {tuple(shape_meta)}")
    if expected_shape is not None and tuple(f.shape) != tuple(expected_shape):
        raise ValueError(f"checkpoint shape {tuple(f.shape)} does not fit this run ({tuple(expected_shape)})")
    if expected_lattice_directions is not None and f.ndim >= 1 and int(f.shape[0]) != expected_lattice_directions:
        raise ValueError(f"checkpoint has {int(f.shape[0])} lattice directions, this run "
                         f"{expected_lattice_directions}")
    return f, int(meta["step"]), meta


# ---------------------------------------------------------------------------
# format 2: unified solver-state envelope
# ---------------------------------------------------------------------------

@dataclass
class SolverCheckpoint:
    """A validated format-2 checkpoint."""

    state: dict[str, Any]
    step: int
    lattice: str | None
    grid: tuple[int, ...] | None
    q: int | None
    metadata: dict[str, Any]
    format_version: int
    path: Path

    @property
    def populations(self) -> torch.Tensor:
        return self.state["populations"]


def _is_int(v: object) -> bool:
    return isinstance(v, int) and not isinstance(v, bool)


def _digest(t: torch.Tensor) -> str:
    raw = t.detach().to("cpu").contiguous().view(torch.uint8)
    return hashlib.sha256(raw.numpy().tobytes()).hexdigest()


def _checked_state(state: object) -> dict[str, Any]:
    if not isinstance(state, dict):
        raise CheckpointError(f"state must be a dict, got {type(state).__name__}")
    for key in ("populations", "step"):
        if key not in state:
            raise CheckpointError(f"state dict has no {key!r}")
    pop = state["populations"]
    if not isinstance(pop, torch.Tensor) or pop.ndim < 1:
        raise CheckpointError("state['populations'] must be a tensor with a leading lattice dimension")
    if not _is_int(state["step"]) or state["step"] < 0:
        raise CheckpointError(f"state['step'] must be a non-negative integer, got {state['step']!r}")
    lat = state.get("lattice")
    if lat is not None and not isinstance(lat, str):
        raise CheckpointError(f"state['lattice'] must be a string or None, got {lat!r}")
    grid = state.get("grid")
    if grid is not None and (not isinstance(grid, (tuple, list)) or not all(_is_int(n) and n > 0 for n in grid)):
        raise CheckpointError(f"state['grid'] must be positive integers, got {grid!r}")
    q = state.get("q")
    if q is not None and (not _is_int(q) or q <= 0):
        raise CheckpointError(f"state['q'] must be a positive integer or None, got {q!r}")
    return state


def _rng_snapshot(ref: torch.Tensor) -> dict[str, Any]:
    snap: dict[str, Any] = {"cpu": torch.get_rng_state()}
    if ref.device.type == "cuda":
        snap["cuda"] = torch.cuda.get_rng_state(ref.device)
        snap["cuda_device"] = str(ref.device)
    return snap


def _rng_restore(snap: object) -> None:
    if not isinstance(snap, dict) or not isinstance(snap.get("cpu"), torch.Tensor):
        return
    torch.set_rng_state(snap["cpu"])
    cuda_state = snap.get("cuda")
    if not isinstance(cuda_state, torch.Tensor):
        return
    dev = snap.get("cuda_device")
    idx = torch.device(dev).index if isinstance(dev, str) else None
    if not torch.cuda.is_available() or (idx is not None and idx >= torch.cuda.device_count()):
        raise CheckpointError(f"the saved RNG state belongs to CUDA device {dev}, which this host lacks; "
                              "load with restore_rng=False")
    torch.cuda.set_rng_state(cuda_state, dev)


def _atomic_save(obj: Any, path: Path) -> Path:
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_name(f".{path.name}.tmp-{os.getpid()}")
    try:
        torch.save(obj, tmp)
        tmp.replace(path)
    finally:
        if tmp.exists():
            tmp.unlink()
    return path


def save_solver_checkpoint(path: str | Path, state: Mapping[str, Any], *,
                           metadata: Mapping[str, Any] | None = None) -> Path:
    """Write a format-2 envelope (temporary file, then rename).  Tensors are
    stored as CPU copies; populations, obstacle mask and this library's
    stored state get SHA-256 digests."""
    payload = dict(_checked_state(dict(state)))
    digests: dict[str, str] = {}
    for key in ("populations", "obstacle_mask", "stored_state"):
        v = payload.get(key)
        if isinstance(v, torch.Tensor):
            payload[key] = v.detach().to("cpu", copy=True)
            digests[key] = _digest(payload[key])
    grid = payload.get("grid")
    envelope = {
        "format": SOLVER_CHECKPOINT_FORMAT,
        "format_version": SOLVER_CHECKPOINT_VERSION,
        "created_at": datetime.now(timezone.utc).isoformat(),
        "step": int(payload["step"]),
        "lattice": payload.get("lattice"),
        "grid": tuple(grid) if grid is not None else None,
        "q": payload.get("q"),
        "state": payload,
        "metadata": dict(metadata or {}),
        "rng": _rng_snapshot(state["populations"]),
        "digests": digests,
    }
    return _atomic_save(envelope, Path(path))


def load_solver_checkpoint(path: str | Path, *, expected_lattice: str | None = None,
                           expected_grid: tuple[int, ...] | None = None, expected_q: int | None = None,
                           restore_rng: bool = True) -> SolverCheckpoint:
    """Read and validate a format-2 envelope (fail closed: ``CheckpointError``)."""
    src = Path(path)
    if not src.is_file():
        raise CheckpointError(f"checkpoint file not found: {src}")
    try:
        env = torch.load(src, map_location="cpu", weights_only=True)
    except Exception as exc:  # any decode failure means a torn or corrupt file
        raise CheckpointError(f"checkpoint {src} could not be decoded: {type(exc).__name__}: {exc}") from exc
    if not isinstance(env, dict) or env.get("format") != SOLVER_CHECKPOINT_FORMAT:
        raise CheckpointError(f"{src} is not a solver checkpoint (no {SOLVER_CHECKPOINT_FORMAT!r} tag)")
    version = env.get("format_version")
    if version != SOLVER_CHECKPOINT_VERSION:
        raise CheckpointError(f"unsupported checkpoint format_version={version!r} in {src}")
    state = _checked_state(env.get("state"))
    digests = env.get("digests")
    if isinstance(digests, dict):
        for key, want in digests.items():
            v = state.get(key)
            if not isinstance(v, torch.Tensor) or not isinstance(want, str):
                raise CheckpointError(f"checkpoint {src} has a broken digest record for {key!r}")
            if _digest(v) != want:
                raise CheckpointError(f"checkpoint {src}: {key!r} does not match its SHA-256 digest")
    grid = tuple(state["grid"]) if state.get("grid") is not None else None
    if expected_lattice is not None and state.get("lattice") != expected_lattice:
        raise CheckpointError(f"checkpoint lattice {state.get('lattice')!r}, expected {expected_lattice!r}")
    if expected_grid is not None and grid != tuple(expected_grid):
        raise CheckpointError(f"checkpoint grid {grid}, expected {tuple(expected_grid)}")
    if expected_q is not None and state.get("q") != expected_q:
        raise CheckpointError(f"checkpoint Q {state.get('q')}, expected {expected_q}")
    if restore_rng:
        _rng_restore(env.get("rng"))
    lat = state.get("lattice")
    q = state.get("q")
    return SolverCheckpoint(state=state, step=int(state["step"]), lattice=lat if isinstance(lat, str) else None,
                            grid=grid, q=q if _is_int(q) else None, metadata=dict(env.get("metadata") or {}),
                            format_version=int(version), path=src)


# campaign hook: one file per scan point, re-checked against the point's identity

def case_checkpoint_path(directory: str | Path) -> Path:
    return Path(directory) / CASE_CHECKPOINT_FILENAME


def save_case_checkpoint(directory: str | Path, *, f: torch.Tensor, step: int, lattice: str | None,
                         grid: tuple[int, ...] | None, identity: Mapping[str, Any],
                         state_extra: Mapping[str, Any] | None = None,
                         metadata: Mapping[str, Any] | None = None) -> Path:
    """Per-point checkpoint of a scan campaign; ``identity`` (scan / point /
    plan ids) is stored in the metadata and must match on resume."""
    state: dict[str, Any] = {"populations": f, "step": int(step), "lattice": lattice,
                             "grid": tuple(grid) if grid is not None else None,
                             "q": int(f.shape[0]) if f.ndim >= 1 else None}
    state.update(state_extra or {})
    meta = {"identity": dict(identity)}
    meta.update(metadata or {})
    return save_solver_checkpoint(case_checkpoint_path(directory), state, metadata=meta)


def load_case_checkpoint(directory: str | Path, *, identity: Mapping[str, Any]) -> SolverCheckpoint | None:
    """The point's checkpoint, or None (restart from step 0) when it is
    absent, unusable or written for another identity.  The RNG is not restored."""
    path = case_checkpoint_path(directory)
    if not path.is_file():
        return None
    try:
        ck = load_solver_checkpoint(path, restore_rng=False)
    except CheckpointError:
        return None
    saved = ck.metadata.get("identity")
    if not isinstance(saved, dict) or any(saved.get(k) != v for k, v in identity.items()):
        return None
    return ck


# ---------------------------------------------------------------------------
# adapters: this library's solvers <-> state dicts
# ---------------------------------------------------------------------------

_LATTICE_NAME = {9: "D2Q9", 19: "D3Q19", 27: "D3Q27"}
_PARAMS = ("collision", "s_e", "s_eps", "s_q", "s_pi", "omega_b", "omega_odd", "omega_even", "c_smag", "u_lid",
           "u_in", "rho_out", "force_lin", "lambda_trt", "cm_s5", "cm_s6")


def solver_state_dict(solver, *, step: int | None = None, extra: Mapping[str, Any] | None = None) -> dict[str, Any]:
    """State dict of an :class:`~tensorlbm_b200.LBMSolver`.

    ``populations`` is the TensorLBM-phase field ``S_n`` (``solver.f``,
    absolute values in the compute dtype), so TensorLBM's own adapters accept
    it; ``stored_state`` is the raw stored ``P_n`` (storage format) for a
    bit-exact continuation in this library."""
    from . import _lib

    cfg = solver.cfg
    f = solver.f
    obstacle = None
    if solver.flags is not None:
        obstacle = (solver.flags & _lib.FLAG_OBSTACLE) != 0
    state: dict[str, Any] = {
        "populations": f,
        "step": solver.step_index if step is None else int(step),
        "lattice": _LATTICE_NAME[solver.q],
        "grid": tuple(int(n) for n in cfg.shape),
        "q": int(solver.q),
        "tau": float(cfg.tau),
        "dtype": str(f.dtype),
        "obstacle_mask": obstacle,
        "precision_policy": PRECISION_POLICY[solver.storage],
        "storage": solver.storage,
        "storage_dtype": str(solver.buf_dtype),
        "stored_state": solver.state,
        "aa_layout": solver.aa_layout,
        "cell_flags": solver.flags.detach().cpu() if solver.flags is not None else None,
        "solver_params": {k: getattr(cfg, k) for k in _PARAMS},
    }
    if extra:
        state["extra"] = dict(extra)
    return state


def solver_load_state_dict(solver, state: Mapping[str, Any], *, exact: bool = True):
    """Continue ``solver`` from a state dict (fail closed on a lattice, Q,
    grid or tau mismatch).  The raw stored state is used when ``exact`` and
    the storage formats agree; otherwise the state is rebuilt from the
    populations (exact for float32 / float64 storage).  Returns the solver."""
    st = _checked_state(dict(state))
    lat = st.get("lattice")
    if isinstance(lat, str) and lat.upper() != _LATTICE_NAME[solver.q]:
        raise CheckpointError(f"state lattice {lat!r} does not match the solver's {_LATTICE_NAME[solver.q]!r}")
    q = st.get("q")
    if q is not None and int(q) != solver.q:
        raise CheckpointError(f"state Q {q} does not match the solver's {solver.q}")
    grid = st.get("grid")
    if grid is not None and tuple(grid) != tuple(solver.cfg.shape):
        raise CheckpointError(f"state grid {tuple(grid)} does not match the solver's {tuple(solver.cfg.shape)}")
    tau = st.get("tau")
    if tau is not None and float(tau) != float(solver.cfg.tau):
        raise CheckpointError(f"state tau {tau} does not match the solver's {solver.cfg.tau}")
    pop = st["populations"]
    if tuple(pop.shape) != (solver.q,) + tuple(solver.cfg.shape):
        raise CheckpointError(f"populations {tuple(pop.shape)} do not fit the solver")
    raw = st.get("stored_state")
    # the raw state fits when the storage format and the memory pattern (two
    # buffers, or one AA buffer with its layout) are the solver's
    same_pattern = (st.get("aa_layout") is None) == (solver.aa_layout is None)
    use_raw = exact and isinstance(raw, torch.Tensor) and st.get("storage") == solver.storage and same_pattern
    return solver.resume(pop.to(device=solver.device, dtype=solver.compute_dtype), step=int(st["step"]),
                         stored_state=raw if use_raw else None, aa_layout=st.get("aa_layout"))


def save_solver(solver, path: str | Path, *, metadata: Mapping[str, Any] | None = None) -> Path:
    """``save_solver_checkpoint(path, solver_state_dict(solver))``."""
    return save_solver_checkpoint(path, solver_state_dict(solver), metadata=metadata)


def load_solver(path: str | Path, solver, *, exact: bool = True, restore_rng: bool = False):
    """Read a format-2 file and continue ``solver`` from it."""
    ck = load_solver_checkpoint(path, restore_rng=restore_rng)
    return solver_load_state_dict(solver, ck.state, exact=exact)


# TensorLBM's duck-typed adapters (checkpoint.py:544-652) for callers that own
# the populations tensor (functional make_step, FusedSolver3D)

def _duck_grid(solver) -> tuple[int, ...] | None:
    dims = [getattr(solver, n, None) for n in ("nz", "ny", "nx")]
    return tuple(int(d) for d in dims) if all(_is_int(d) for d in dims) else None


def _duck_q(solver) -> int | None:
    for n in ("Q", "_Q", "q"):
        v = getattr(solver, n, None)
        if _is_int(v):
            return int(v)
    return None


def eager_state_dict(solver, f: torch.Tensor, *, step: int | None = None,
                     extra: Mapping[str, Any] | None = None) -> dict[str, Any]:
    """State dict from any object with ``tau`` (and optionally ``nz/ny/nx``,
    ``Q``, ``lattice``, ``mask``) plus the caller's populations ``f``."""
    if not isinstance(f, torch.Tensor):
        raise TypeError(f"populations must be a tensor, got {type(f).__name__}")
    tau = getattr(solver, "tau", None)
    grid = _duck_grid(solver)
    q = _duck_q(solver)
    mask = next((v for n in ("mask", "_mask", "solid_mask", "_solid_mask")
                 if isinstance(v := getattr(solver, n, None), torch.Tensor)), None)
    policy = getattr(solver, "precision_policy", None)
    state = {"populations": f.detach(),
             "step": int(step) if step is not None else int(getattr(solver, "_report_step", 0) or 0),
             "lattice": getattr(solver, "lattice", None),
             "grid": grid if grid is not None else tuple(int(n) for n in f.shape[1:]),
             "q": q if q is not None else int(f.shape[0]),
             "tau": float(tau) if tau is not None else None,
             "dtype": str(f.dtype), "obstacle_mask": mask,
             "precision_policy": getattr(policy, "name", policy)}
    if extra:
        state["extra"] = dict(extra)
    return state


def eager_load_state_dict(solver, state: Mapping[str, Any], *, device=None) -> torch.Tensor:
    """The populations of ``state`` on the solver's device, after checking
    lattice, Q, grid and tau against the solver."""
    st = _checked_state(dict(state))
    f = st["populations"]
    lat, mine = st.get("lattice"), getattr(solver, "lattice", None)
    if isinstance(lat, str) and isinstance(mine, str) and lat.upper() != mine.upper():
        raise CheckpointError(f"state lattice {lat!r} does not match the solver's {mine!r}")
    q = _duck_q(solver)
    if q is not None and int(st.get("q") or f.shape[0]) != q:
        raise CheckpointError(f"state Q {st.get('q')} does not match the solver's {q}")
    grid = _duck_grid(solver)
    if grid is not None and tuple(st.get("grid") or ()) != grid:
        raise CheckpointError(f"state grid {st.get('grid')} does not match the solver's {grid}")
    tau, mtau = st.get("tau"), getattr(solver, "tau", None)
    if tau is not None and mtau is not None and float(tau) != float(mtau):
        raise CheckpointError(f"state tau {tau} does not match the solver's {mtau}")
    if isinstance(getattr(solver, "_report_step", None), int):
        solver._report_step = int(st["step"])
    target = device if device is not None else getattr(solver, "device", None)
    return f.to(device=target) if target is not None else f


def triton_fused_state_dict(solver, f: torch.Tensor, *, step: int | None = None,
                            extra: Mapping[str, Any] | None = None) -> dict[str, Any]:
    """``eager_state_dict`` plus the storage dtype (lattice defaults to D3Q19)."""
    state = eager_state_dict(solver, f, step=step, extra=extra)
    state["lattice"] = state["lattice"] or "D3Q19"
    state["storage_dtype"] = str(getattr(solver, "dtype", f.dtype))
    return state


def triton_fused_load_state_dict(solver, state: Mapping[str, Any], *, device=None) -> torch.Tensor:
    """``eager_load_state_dict`` that also rejects a storage dtype or
    precision policy other than the solver's (either would change the trajectory)."""
    policy = getattr(solver, "precision_policy", None)
    if state.get("precision_policy") != getattr(policy, "name", policy):
        raise CheckpointError(f"state precision policy {state.get('precision_policy')!r} does not match "
                              f"the solver's {getattr(policy, 'name', policy)!r}")
    dt = getattr(solver, "dtype", None)
    saved = state.get("storage_dtype") or state.get("dtype")
    if dt is not None and str(saved) != str(dt):
        raise CheckpointError(f"state storage dtype {saved} does not match the solver's {dt}")
    return eager_load_state_dict(solver, state, device=device)


# ---------------------------------------------------------------------------
# batched runner: one format-1 directory per domain plus a manifest
# ---------------------------------------------------------------------------

def save_batch_checkpoint(batch, run_dir: str | Path, *, extra: Mapping[str, Any] | None = None) -> Path:
    """Checkpoint a :class:`~tensorlbm_b200.batch.BatchedSolver`.

    Each domain is a format-1 directory (``domain_NNNNN/``): its
    TensorLBM-phase float32 field, its own step count and its parameters, so
    any domain can be continued alone by TensorLBM; the domain masks sit
    beside it, and ``batch_manifest.json`` lists the domains."""
    out = Path(run_dir)
    out.mkdir(parents=True, exist_ok=True)
    steps = batch.step_counts
    entries = []
    for i, d in enumerate(batch.domains):
        sub = f"domain_{i:05d}"
        params = {"lattice": "D2Q9", "grid": [d.ny, d.nx], "tau": float(d.tau), "u_in": d.u_in,
                  "rho_out": d.rho_out, "collision": batch.collision, "domain_index": i}
        save_checkpoint(batch.f(i), steps[i], out / sub, extra=params)
        torch.save({"wall_mask": None if d.wall_mask is None else d.wall_mask.detach().cpu(),
                    "obstacle_mask": None if d.obstacle_mask is None else d.obstacle_mask.detach().cpu()},
                   out / sub / "domain_masks.pt")
        entries.append({"index": i, "dir": sub, "nx": d.nx, "ny": d.ny, "tau": float(d.tau), "u_in": d.u_in,
                        "rho_out": d.rho_out, "step": steps[i]})
    manifest = {"format": BATCH_FORMAT, "format_version": BATCH_FORMAT_VERSION,
                "created_at": datetime.now(timezone.utc).isoformat(), "collision": batch.collision,
                "n_domains": len(entries), "domains": entries, "extra": dict(extra or {})}
    tmp = out / f".{BATCH_MANIFEST}.tmp-{os.getpid()}"
    tmp.write_text(json.dumps(manifest, indent=2) + "\n", encoding="utf-8")
    tmp.replace(out / BATCH_MANIFEST)
    return out


def load_batch_checkpoint(run_dir: str | Path, device=None, *, collision: str | None = None, **solver_kwargs):
    """Rebuild the batched solver of a :func:`save_batch_checkpoint`
    directory and continue it (float32 storage: the continuation is exact).
    ``solver_kwargs`` go to :class:`~tensorlbm_b200.batch.BatchedSolver`."""
    from .batch import BatchedSolver, DomainSpec

    src = Path(run_dir)
    mpath = src / BATCH_MANIFEST
    if not mpath.is_file():
        raise CheckpointError(f"batch manifest not found: {mpath}")
    try:
        man = json.loads(mpath.read_text(encoding="utf-8"))
    except json.JSONDecodeError as exc:
        raise CheckpointError(f"batch manifest is not valid JSON: {mpath}") from exc
    if not isinstance(man, dict) or man.get("format") != BATCH_FORMAT:
        raise CheckpointError(f"{mpath} is not a batch checkpoint manifest")
    if man.get("format_version") != BATCH_FORMAT_VERSION:
        raise CheckpointError(f"unsupported batch checkpoint version {man.get('format_version')!r}")
    specs, fields, steps = [], [], []
    for e in man["domains"]:
        f, step, _ = load_checkpoint(src / e["dir"], expected_shape=(9, e["ny"], e["nx"]),
                                     expected_lattice_directions=9)
        masks = torch.load(src / e["dir"] / "domain_masks.pt", map_location="cpu", weights_only=True)
        specs.append(DomainSpec(int(e["nx"]), int(e["ny"]), float(e["tau"]), e["u_in"], e["rho_out"],
                                masks.get("wall_mask"), masks.get("obstacle_mask")))
        fields.append(f)
        steps.append(step)
    b = BatchedSolver(specs, collision or man["collision"], device=device, **solver_kwargs)
    return b.resume(fields, steps)
