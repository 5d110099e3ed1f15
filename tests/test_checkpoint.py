"""Checkpoint formats on the CPU: TensorLBM's format-1 pair and format-2
solver-state envelope, read from files the reference itself wrote
(tests/golden/checkpoint_ref, made by make_golden.py --only checkpoints),
written and read back, and rejected when broken."""

import json
import pathlib
import types

import numpy as np
import pytest
import torch

from tensorlbm_b200 import checkpoint as C

REF = pathlib.Path(__file__).parent / "golden" / "checkpoint_ref"


def test_reads_reference_pair():
    exp = np.load(REF / "expected.npz")
    f, step, meta = C.load_checkpoint(REF / "pair", expected_shape=(19, 2, 3, 4), expected_lattice_directions=19)
    assert step == 123 and meta["case"] == "golden" and meta["tau"] == 0.6
    assert np.array_equal(f.numpy(), exp["f"])


def test_reads_reference_solver_file():
    exp = np.load(REF / "expected.npz")
    ck = C.load_solver_checkpoint(REF / "solver_v2.pt", expected_lattice="D3Q19", expected_grid=(2, 3, 4),
                                  expected_q=19, restore_rng=True)
    assert ck.step == 77 and ck.format_version == 2 and ck.metadata == {"run": "golden"}
    assert np.array_equal(ck.populations.numpy(), exp["f2"])
    assert np.array_equal(ck.state["obstacle_mask"].numpy(), exp["mask"])
    assert ck.state["tau"] == 0.55 and ck.state["extra"] == {"note": "golden"}
    # the saved RNG state is the one right after torch.manual_seed(7)
    assert np.array_equal(torch.rand(4).numpy(), exp["rng_after_seed7"])


def test_pair_round_trip_same_files(tmp_path):
    f = torch.arange(19 * 6, dtype=torch.float64).reshape(19, 2, 3)
    C.save_checkpoint(f, 9, tmp_path, extra={"who": "us"})
    g, step, meta = C.load_checkpoint(tmp_path)
    assert torch.equal(f, g) and step == 9 and meta["who"] == "us"
    ref_meta = json.loads((REF / "pair" / "checkpoint_meta.json").read_text())
    ours = json.loads((tmp_path / "checkpoint_meta.json").read_text())
    fixed = {"format_version", "step", "tensor_shape", "tensor_dtype", "lattice_directions"}
    assert fixed <= set(ours) and fixed <= set(ref_meta)
    assert sorted((p.name for p in tmp_path.iterdir())) == sorted(p.name for p in (REF / "pair").iterdir())


def test_pair_rejects(tmp_path):
    with pytest.raises(FileNotFoundError):
        C.load_checkpoint(tmp_path / "nothing")
    C.save_checkpoint(torch.zeros(9, 2, 2), 1, tmp_path)
    with pytest.raises(ValueError, match="does not fit"):
        C.load_checkpoint(tmp_path, expected_shape=(9, 2, 3))
    with pytest.raises(ValueError, match="lattice directions"):
        C.load_checkpoint(tmp_path, expected_lattice_directions=19)
    meta = json.loads((tmp_path / C.META_FILE).read_text())
    (tmp_path / C.META_FILE).write_text(json.dumps(dict(meta, format_version=3)))
    with pytest.raises(ValueError, match="format_version"):
        C.load_checkpoint(tmp_path)
    (tmp_path / C.META_FILE).write_text("{not json")
    with pytest.raises(ValueError, match="JSON"):
        C.load_checkpoint(tmp_path)
    (tmp_path / C.META_FILE).write_text(json.dumps({"format_version": 1}))
    with pytest.raises(ValueError, match="step"):
        C.load_checkpoint(tmp_path)


def test_solver_file_round_trip_and_envelope(tmp_path):
    f = torch.randn(27, 3, 4, 5)
    raw = torch.randn(27, 3, 4, 5).to(torch.float16)
    state = {"populations": f, "step": 5, "lattice": "D3Q27", "grid": (3, 4, 5), "q": 27, "tau": 0.6,
             "obstacle_mask": torch.zeros(3, 4, 5, dtype=torch.bool), "stored_state": raw, "storage": "f16"}
    p = C.save_solver_checkpoint(tmp_path / "a.pt", state, metadata={"k": 1})
    ck = C.load_solver_checkpoint(p, expected_grid=(3, 4, 5), restore_rng=False)
    assert torch.equal(ck.populations, f) and torch.equal(ck.state["stored_state"], raw) and ck.metadata == {"k": 1}
    env = torch.load(p, weights_only=True)
    ref_env = torch.load(REF / "solver_v2.pt", weights_only=True)
    assert set(ref_env) <= set(env) and env["format"] == ref_env["format"]
    assert env["format_version"] == ref_env["format_version"]
    assert set(env["digests"]) == {"populations", "obstacle_mask", "stored_state"}
    assert not any(pp.name.startswith(".") for pp in tmp_path.iterdir())  # no temporary file left


def test_solver_file_fails_closed(tmp_path):
    f = torch.randn(19, 2, 2, 2)
    p = C.save_solver_checkpoint(tmp_path / "a.pt", {"populations": f, "step": 1, "lattice": "D3Q19", "q": 19})
    with pytest.raises(C.CheckpointError, match="lattice"):
        C.load_solver_checkpoint(p, expected_lattice="D3Q27", restore_rng=False)
    with pytest.raises(C.CheckpointError, match="Q"):
        C.load_solver_checkpoint(p, expected_q=27, restore_rng=False)
    env = torch.load(p, weights_only=True)
    env["state"]["populations"] = f + 1.0                     # payload changed after the digest
    torch.save(env, tmp_path / "b.pt")
    with pytest.raises(C.CheckpointError, match="digest"):
        C.load_solver_checkpoint(tmp_path / "b.pt", restore_rng=False)
    (tmp_path / "c.pt").write_bytes(p.read_bytes()[: len(p.read_bytes()) // 2])   # torn write
    with pytest.raises(C.CheckpointError, match="decoded"):
        C.load_solver_checkpoint(tmp_path / "c.pt")
    env = torch.load(p, weights_only=True)
    env["format_version"] = 3
    torch.save(env, tmp_path / "d.pt")
    with pytest.raises(C.CheckpointError, match="format_version"):
        C.load_solver_checkpoint(tmp_path / "d.pt")
    with pytest.raises(C.CheckpointError):
        C.save_solver_checkpoint(tmp_path / "e.pt", {"populations": f, "step": -1})
    with pytest.raises(C.CheckpointError, match="not found"):
        C.load_solver_checkpoint(tmp_path / "missing.pt")


def test_case_checkpoint_identity(tmp_path):
    f = torch.randn(9, 4, 4)
    C.save_case_checkpoint(tmp_path, f=f, step=3, lattice="D2Q9", grid=(4, 4), identity={"scan": "s1", "point": 2})
    ck = C.load_case_checkpoint(tmp_path, identity={"scan": "s1", "point": 2})
    assert ck is not None and ck.step == 3 and torch.equal(ck.populations, f)
    assert C.load_case_checkpoint(tmp_path, identity={"scan": "s1", "point": 3}) is None
    assert C.load_case_checkpoint(tmp_path / "other", identity={}) is None


def test_duck_typed_adapters():
    solver = types.SimpleNamespace(tau=0.6, nz=2, ny=2, nx=3, Q=19, lattice="D3Q19", dtype=torch.float16,
                                   precision_policy=types.SimpleNamespace(name="FP32FP16"), _report_step=0)
    f = torch.randn(19, 2, 2, 3).to(torch.float16)
    st = C.triton_fused_state_dict(solver, f, step=11)
    assert st["lattice"] == "D3Q19" and st["storage_dtype"] == "torch.float16" and st["precision_policy"] == "FP32FP16"
    g = C.triton_fused_load_state_dict(solver, st)
    assert torch.equal(g, f) and solver._report_step == 11
    other = types.SimpleNamespace(**{**vars(solver), "precision_policy": types.SimpleNamespace(name="FP32FP32")})
    with pytest.raises(C.CheckpointError, match="precision"):
        C.triton_fused_load_state_dict(other, st)
    wrong_tau = types.SimpleNamespace(**{**vars(solver), "tau": 0.7})
    with pytest.raises(C.CheckpointError, match="tau"):
        C.eager_load_state_dict(wrong_tau, st)


def _reference_checkpoint_module():
    """TensorLBM's own checkpoint module from baseline/_ref, or skip."""
    import importlib
    import sys

    ref = pathlib.Path(__file__).resolve().parents[1] / "baseline" / "_ref"
    if not (ref / "tensorlbm" / "checkpoint.py").is_file():
        pytest.skip("TensorLBM is not installed in baseline/_ref")

    class _Stub(types.ModuleType):
        def __getattr__(self, name):
            if name.startswith("__"):
                raise AttributeError(name)
            return _Stub(f"{self.__name__}.{name}")

        def __call__(self, *a, **k):
            return self

    for name in ("matplotlib", "matplotlib.pyplot", "h5py"):
        sys.modules.setdefault(name, _Stub(name))
    if str(ref) not in sys.path:
        sys.path.append(str(ref))
    try:
        return importlib.import_module("tensorlbm.checkpoint")
    except Exception as exc:  # the package pulls in optional modules
        pytest.skip(f"TensorLBM does not import here: {exc}")


def test_reference_reads_our_files(tmp_path):
    ref = _reference_checkpoint_module()
    f = torch.randn(19, 2, 3, 4)
    C.save_checkpoint(f, 42, tmp_path / "pair", extra={"x": 1})
    g, step, meta = ref.load_checkpoint(tmp_path / "pair", expected_shape=(19, 2, 3, 4))
    assert torch.equal(f, g) and step == 42 and meta["x"] == 1
    state = {"populations": f, "step": 8, "lattice": "D3Q19", "grid": (2, 3, 4), "q": 19, "tau": 0.6,
             "stored_state": f.to(torch.float16), "storage": "f16"}
    C.save_solver_checkpoint(tmp_path / "s.pt", state)
    ck = ref.load_solver_checkpoint(tmp_path / "s.pt", expected_lattice="D3Q19", expected_grid=(2, 3, 4),
                                    restore_rng=False)
    assert ck.step == 8 and torch.equal(ck.populations, f)
