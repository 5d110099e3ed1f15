"""The drop-in, end to end: TensorLBM's own runners (the unmodified package
from baseline/_ref) on CUDA tensors after install(), against the same runners
on the CPU with TensorLBM's torch operators.

- run_sphere_flow_d3q27 (d3q27_sphere_flow.py:134, loop :246-289):
  collide_bgk27 -> stream27 -> compute_obstacle_forces_27 ->
  apply_zou_he_channel_boundaries_27, all bound at the runner's import.  Every
  replaced operator is bit-exact, so the final populations must be identical
  and the drag coefficient equal to float32 summation order.
- run_sphere_flow (sphere_flow.py:256-296): collide_bgk3d -> stream3d ->
  apply_simple_channel_boundaries_3d (TensorLBM's own torch code, now calling
  the replaced macroscopic3d / equilibrium3d) -> correct_mass3d every output
  interval.  The mass correction sums in float64 on the GPU and in float32 on
  the CPU, so the runs may part by float32 rounding: 1e-5 relative.
"""

from __future__ import annotations

import json

import numpy as np
import pytest
import torch

from baseline import reference

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not reference.available(), reason="TensorLBM is not installed in baseline/_ref")]


def _run(runner, cfg_cls, device, tmp, install):
    import tensorlbm_b200 as tb

    tl = reference.import_reference()
    from tensorlbm.checkpoint import load_checkpoint

    kw = dict(nx=48, ny=24, nz=24, u_in=0.04, re=20.0, radius=4.0, n_steps=40, output_interval=10,
              output_root=tmp / device, run_name="run", device=device, overwrite=True)
    det = torch.are_deterministic_algorithms_enabled()
    try:
        if install:
            tb.install(tl)
        run_dir = runner(cfg_cls(**kw))
    finally:
        tb.uninstall()
        torch.use_deterministic_algorithms(det)
    meta = json.loads((run_dir / "run_metadata.json").read_text())
    f, step, _ = load_checkpoint(run_dir)
    return meta["diagnostics"], f.detach().cpu().numpy(), step


def test_reference_d3q27_sphere_runner_on_kernels(cuda, tmp_path):
    reference.import_reference()
    from tensorlbm.d3q27_sphere_flow import SphereFlowD3Q27Config, run_sphere_flow_d3q27

    d_cpu, f_cpu, s_cpu = _run(run_sphere_flow_d3q27, SphereFlowD3Q27Config, "cpu", tmp_path, install=False)
    d_gpu, f_gpu, s_gpu = _run(run_sphere_flow_d3q27, SphereFlowD3Q27Config, "cuda", tmp_path, install=True)
    assert s_cpu == s_gpu == 40 and len(d_cpu) == len(d_gpu) == 4
    assert np.isfinite(f_cpu).all()
    assert np.array_equal(f_gpu, f_cpu)                      # bit-exact chain
    for a, b in zip(d_gpu, d_cpu):
        assert a["step"] == b["step"]
        assert abs(a["cd"] - b["cd"]) <= 1e-5 * abs(b["cd"]), (a["cd"], b["cd"])
        for key in ("mass", "mean_rho", "max_speed"):
            assert abs(a[key] - b[key]) <= 1e-6 * abs(b[key]), key


def test_reference_d3q19_sphere_runner_on_kernels(cuda, tmp_path):
    reference.import_reference()
    from tensorlbm.sphere_flow import SphereFlowConfig, run_sphere_flow

    d_cpu, f_cpu, s_cpu = _run(run_sphere_flow, SphereFlowConfig, "cpu", tmp_path, install=False)
    d_gpu, f_gpu, s_gpu = _run(run_sphere_flow, SphereFlowConfig, "cuda", tmp_path, install=True)
    assert s_cpu == s_gpu == 40 and len(d_cpu) == len(d_gpu) == 4
    assert np.isfinite(f_cpu).all()
    assert np.max(np.abs(f_gpu - f_cpu)) <= 1e-5 * np.max(np.abs(f_cpu))
    for a, b in zip(d_gpu, d_cpu):
        assert a["step"] == b["step"]
        for key in ("mass", "mean_rho", "max_speed"):
            assert abs(a[key] - b[key]) <= 1e-5 * abs(b[key]), key
