"""Checkpoint / resume on the GPU: a run saved at step n and continued to
2n must equal the uninterrupted run bit for bit (float32 from the
TensorLBM-phase populations alone; FP16/BF16 from the stored state), and the
batched runner continues every domain exactly with its own step count."""

import numpy as np
import pytest
import torch

from oracle import lbm as O
from tensorlbm_b200 import checkpoint as C

pytestmark = pytest.mark.gpu


def _channel(cuda, storage, coll="mrt"):
    from tensorlbm_b200 import LBMSolver, boundaries3d

    nz, ny, nx = 10, 12, 24
    obst = boundaries3d.sphere_mask(nx, ny, nz, 8.0, 6.0, 5.0, 2.5, cuda)
    ux = np.full((nz, ny, nx), 0.04, np.float32)
    ux[obst.cpu().numpy()] = 0.0
    z = np.zeros_like(ux)
    f0 = torch.from_numpy(O.equilibrium(19, np.ones_like(ux), ux, z, z)).to(cuda)

    def make():
        return LBMSolver("D3Q19", (nz, ny, nx), 0.53, coll, device=cuda, storage=storage, obstacle_mask=obst,
                         u_in=0.04, rho_out=1.0)

    return make, f0


@pytest.mark.parametrize("coll", ["mrt", "bgk"])
def test_float32_resume_from_populations_is_exact(cuda, tmp_path, coll):
    make, f0 = _channel(cuda, "f32", coll)
    full = make().load(f0).step(40)
    half = make().load(f0).step(20)
    C.save_checkpoint(half.f, half.step_index, tmp_path / "pair")
    C.save_solver(half, tmp_path / "s.pt")
    f, step, _ = C.load_checkpoint(tmp_path / "pair", expected_lattice_directions=19)
    a = make().resume(f.to(cuda), step=step).step(20)
    b = C.load_solver(tmp_path / "s.pt", make(), exact=False).step(20)
    assert a.step_index == 40 and b.step_index == 40
    assert torch.equal(a.state, full.state) and torch.equal(b.state, full.state)
    assert torch.equal(a.f, full.f)


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_half_storage_resume_from_stored_state_is_exact(cuda, tmp_path, storage):
    make, f0 = _channel(cuda, storage, "bgk")
    full = make().load(f0).step(30)
    half = make().load(f0).step(15)
    C.save_solver(half, tmp_path / "s.pt")
    ck = C.load_solver_checkpoint(tmp_path / "s.pt", expected_q=19, restore_rng=False)
    assert ck.state["storage"] == storage and ck.state["populations"].dtype == torch.float32
    exact = C.solver_load_state_dict(make(), ck.state).step(15)
    assert torch.equal(exact.state, full.state)
    # from the absolute populations alone the half formats are re-rounded once:
    # the same flow to storage precision, not the same bits
    approx = C.solver_load_state_dict(make(), ck.state, exact=False).step(15)
    assert (approx.f - full.f).abs().max().item() < 1e-3 * full.f.abs().max().item()


def test_resume_rejects_other_grid(cuda, tmp_path):
    from tensorlbm_b200 import LBMSolver

    make, f0 = _channel(cuda, "f32")
    s = make().load(f0).step(2)
    C.save_solver(s, tmp_path / "s.pt")
    other = LBMSolver("D3Q19", (10, 12, 26), 0.53, "mrt", device=cuda)
    with pytest.raises(C.CheckpointError, match="grid"):
        C.load_solver(tmp_path / "s.pt", other)
    wrong_tau = LBMSolver("D3Q19", (10, 12, 24), 0.6, "mrt", device=cuda)
    with pytest.raises(C.CheckpointError, match="tau"):
        C.load_solver(tmp_path / "s.pt", wrong_tau)


def test_batched_resume_is_exact(cuda, tmp_path):
    from tensorlbm_b200 import batch

    doms = [batch.cylinder_channel(nx, re, device=cuda) for nx, re in ((128, 20.0), (160, 30.0), (192, 25.0))]
    f0 = batch.equilibrium_start(doms, cuda)
    full = batch.BatchedSolver(doms, "bgk", device=cuda).load(f0)
    full.step(40)
    half = batch.BatchedSolver(doms, "bgk", device=cuda).load(f0)
    half.step(25)
    C.save_batch_checkpoint(half, tmp_path / "b")
    # any one domain is a plain format-1 checkpoint
    f1, step1, meta1 = C.load_checkpoint(tmp_path / "b" / "domain_00001", expected_shape=(9, 40, 160))
    assert step1 == 25 and meta1["tau"] == doms[1].tau and torch.equal(f1.to(cuda), half.f(1))
    res = C.load_batch_checkpoint(tmp_path / "b", cuda)
    assert res.step_counts == [25, 25, 25]
    res.step(15)
    assert res.step_counts == [40, 40, 40]
    for i in range(len(doms)):
        assert torch.equal(res.f(i), full.f(i)), i
