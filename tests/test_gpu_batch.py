"""Batched multi-domain D2Q9 runner: every domain must evolve bit for bit as
the single-domain fused solver advances it, in every execution mode."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from tests.conftest import same

pytestmark = pytest.mark.gpu


def _domains(dev):
    from tensorlbm_b200 import batch

    # uneven sizes (ny = nx/4); Reynolds numbers low enough that tau >= 0.53
    # keeps BGK stable on these coarse cylinders (D = 2..6 cells)
    return [batch.cylinder_channel(nx, re, 0.05, dev) for nx, re in ((64, 8.0), (136, 20.0), (96, 12.0),
                                                                    (200, 25.0), (128, 16.0))]


def _alone(dom, f0, steps, dev):
    from tensorlbm_b200 import LBMSolver

    s = LBMSolver("D2Q9", (dom.ny, dom.nx), dom.tau, "bgk", device=dev, wall_mask=dom.wall_mask,
                  obstacle_mask=dom.obstacle_mask, u_in=dom.u_in, rho_out=dom.rho_out, track_force=True)
    s.load(f0).step(steps)
    return s


@pytest.mark.parametrize("mode,tile", [("launch", (64, 4)), ("graph", (32, 8)), ("persistent", (128, 2))])
def test_batched_domains_equal_single_runs(cuda, mode, tile):
    from tensorlbm_b200 import batch

    doms = _domains(cuda)
    f0 = batch.equilibrium_start(doms, cuda)
    steps = 120
    b = batch.BatchedSolver(doms, "bgk", device=cuda, tile=tile, mode=mode).load(f0)
    rec = 3 if mode == "graph" else 1  # graph mode: an odd record period exercises the slot counter
    hist = b.run(steps, record_every=rec)
    assert int(b.status.item()) == 0
    for i, d in enumerate(doms):
        ref = _alone(d, f0[i], steps, cuda)
        assert same(b.f(i).cpu().numpy(), ref.f.cpu().numpy()), f"domain {i}"
        got = hist[:, i, :].cpu().numpy()
        want = ref.force_history().cpu().numpy()[::rec]
        assert got.shape == want.shape
        assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


def test_persistent_barrier_timeout_reports_status(cuda):
    """A barrier that cannot complete within its spin budget makes every CTA
    return and sets status bit 1; nothing hangs and the context stays usable."""
    from tensorlbm_b200 import batch

    doms = _domains(cuda)
    b = batch.BatchedSolver(doms, "bgk", device=cuda, tile=(32, 1), mode="persistent")
    b.load(batch.equilibrium_start(doms, cuda))
    b.sync[2] = 1  # error flag already raised: the first barrier gives up at once
    b.run(50, max_spins=1)
    torch.cuda.synchronize(cuda)
    assert int(b.status.item()) & 2
    # recover: clear the sync words and status, reload, run normally
    b.sync.zero_()
    b.status.zero_()
    b.load(batch.equilibrium_start(doms, cuda))
    b.run(10)
    torch.cuda.synchronize(cuda)
    assert int(b.status.item()) == 0


def test_autotune_and_strouhal_smoke(cuda):
    from tensorlbm_b200 import batch

    # Re low enough for BGK at these resolutions (tau >= 0.52)
    doms = batch.uniform_scan(6, seed=20261203, device=cuda, nx_range=(128, 256), re_range=(8.0, 25.0))
    b = batch.BatchedSolver(doms, "bgk", device=cuda)
    b.load(batch.equilibrium_start(doms, cuda))
    res = batch.autotune(b, steps=5)
    assert res["best"]["mlups"] > 0 and len(res["trials"]) >= 2
    b.load(batch.equilibrium_start(doms, cuda))
    hist = b.run(400, record_every=1)
    assert hist.shape == (400, 6, 3)
    assert torch.isfinite(hist).all()
