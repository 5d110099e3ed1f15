"""The tensorlbm.triton_fused drop-in: periodic D3Q19 pull + BGK, its halves
and the solver class, in float32 (bit-exact with the torch path) and in plain
float16 / bfloat16 storage (float32 arithmetic, rounded to nearest on store)."""

import numpy as np
import pytest
import torch

from oracle import lbm as O

pytestmark = pytest.mark.gpu


def _field(shape=(6, 8, 16), seed=4):
    rng = np.random.default_rng(seed)
    rho = (1 + 0.03 * rng.uniform(-1, 1, shape)).astype(np.float32)
    u = [(0.05 * rng.uniform(-1, 1, shape)).astype(np.float32) for _ in range(3)]
    f = O.equilibrium(19, rho, *u) * (1 + 0.01 * rng.uniform(-1, 1, (19,) + shape))
    return f.astype(np.float32)


def test_float32_bitwise(cuda):
    from tensorlbm_b200 import triton_fused as tf

    f = _field()
    t = torch.from_numpy(f).to(cuda)
    assert np.array_equal(tf.triton_stream(t).cpu().numpy(), O.stream(f))
    assert np.array_equal(tf.triton_collide(t, 0.6).cpu().numpy(), O.collide_bgk(f, 0.6))
    assert np.array_equal(tf.triton_fused(t, 0.6).cpu().numpy(), O.collide_bgk(O.stream(f), 0.6))
    out = torch.empty_like(t)
    assert tf.triton_fused(t, 0.6, out=out) is out
    with pytest.raises(ValueError, match="alias"):
        tf.triton_fused(t, 0.6, out=t)            # the pull must not run in place


@pytest.mark.parametrize("dtype,tol", [(torch.float16, 1e-3), (torch.bfloat16, 8e-3)])
def test_plain_half_storage(cuda, dtype, tol):
    from tensorlbm_b200 import triton_fused as tf

    f = _field()
    h = torch.from_numpy(f).to(cuda).to(dtype)
    ref = O.collide_bgk(O.stream(h.float().cpu().numpy()), 0.6)
    got = tf.triton_fused(h, 0.6)
    assert got.dtype == dtype
    # one rounding to nearest of the float32 result (computed in the fused form)
    assert np.all(np.abs(got.float().cpu().numpy() - ref) <= tol * np.abs(ref) + 1e-6)


def test_solver_class_and_precision(cuda):
    from tensorlbm_b200 import FusedSolver3D
    from tensorlbm_b200.triton_fused import TritonFusedSolver3D

    assert FusedSolver3D is TritonFusedSolver3D
    f = torch.from_numpy(_field()).to(cuda)
    s32 = TritonFusedSolver3D(6, 8, 16, 0.6, device=cuda)
    s16 = TritonFusedSolver3D(6, 8, 16, 0.6, device=cuda, precision="FP32FP16")
    assert s16.dtype == torch.float16 and s16.transient_memory_bytes() == 2 * 6 * 8 * 16 * 19 * 2
    a, _ = s32.run(f, 10)
    b, diags = s16.run(f.half(), 10)
    assert len(diags) == 10 and s16._report_step == 10
    assert (b.float() - a).abs().max().item() < 5e-3 * a.abs().max().item()
    with pytest.raises(NotImplementedError):
        TritonFusedSolver3D(6, 8, 16, 0.6, device=cuda, precision="FP64FP64")
    with pytest.raises(ValueError):
        TritonFusedSolver3D(6, 8, 16, 0.6, device=cuda, dtype=torch.bfloat16, precision="FP32FP16")
    with pytest.raises(ValueError):
        s16.step(f)                                   # float32 input to a float16 solver
    assert s32.benchmark(n_steps=3, warmup=1) > 0
