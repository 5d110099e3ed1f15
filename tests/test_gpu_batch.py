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


@pytest.mark.parametrize("mode,tile,cpt", [("launch", (64, 4), 1), ("graph", (32, 8), 1), ("persistent", (128, 2), 1),
                                          ("launch", (128, 2), 2), ("graph", (64, 4), 2), ("persistent", (256, 2), 2)])
def test_batched_domains_equal_single_runs(cuda, mode, tile, cpt):
    """cpt = 2: two cells per thread (the pair update; the odd-nx domain takes
    two single-cell updates), still bit for bit the single runs."""
    from tensorlbm_b200 import batch

    doms = _domains(cuda)
    if cpt == 2:   # one domain of odd nx for the per-cell fallback of the pair tiles
        odd = batch.cylinder_channel(96, 12.0, 0.05, cuda)
        odd = batch.DomainSpec(95, odd.ny, odd.tau, odd.u_in, odd.rho_out, odd.wall_mask[:, :95].contiguous(),
                               odd.obstacle_mask[:, :95].contiguous())
        doms.append(odd)
    f0 = batch.equilibrium_start(doms, cuda)
    steps = 120
    b = batch.BatchedSolver(doms, "bgk", device=cuda, tile=tile, mode=mode, cells_per_thread=cpt).load(f0)
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


def test_scan_divergence_matches_reference(cuda):
    """The 21 smallest design points of the seeded 512-domain scan (nx <= 160,
    BGK tau - 1/2 between 0.0027 and 0.0068 on cylinders of D = 4-5 cells)
    turn non-finite in TensorLBM's own D2Q9 cylinder chain at steps 54-64
    (golden c4_divergence, generated from the unmodified reference).  The
    batched runner must reach the same onset step on every one of them, and
    the same populations bit for bit on the last finite state the fixture
    holds."""
    from tensorlbm_b200 import batch

    from tests.conftest import golden

    g = golden("c4_divergence")
    pick = [int(i) for i in g["domains"]]
    design = batch.uniform_scan(512, seed=20261203, device=cuda)
    doms = [design[i] for i in pick]
    for k, i in enumerate(pick):
        assert doms[k].tau == pytest.approx(float(g[f"tau_{i}"]), rel=0, abs=1e-15)
    b = batch.BatchedSolver(doms, "bgk", device=cuda).load(batch.equilibrium_start(doms, cuda))
    onset = {i: -1 for i in pick}
    last = max(int(g[f"nan_step_{i}"]) for i in pick)
    assert 0 < last < 100
    for step in range(1, last + 1):
        b.step()
        for k, i in enumerate(pick):
            if onset[i] >= 0:
                continue
            f = b.f(k)
            if not bool(torch.isfinite(f).all()):
                onset[i] = step
            elif f"check_step_{i}" in g and step == int(g[f"check_step_{i}"]):
                assert same(f.cpu().numpy(), g[f"check_{i}"]), i
    assert onset == {i: int(g[f"nan_step_{i}"]) for i in pick}


@pytest.mark.parametrize("mode", ["graph", "persistent"])
def test_cavity_scan_points_match_reference_case(cuda, mode):
    """Scan points of TensorLBM's registered cavity case (cases/cavity.py),
    advanced as one batch, against the case's own chain run by the reference
    (golden cavity_case): BGK bit for bit, MRT to float32 rounding of the
    reference's BLAS products (1e-5 relative)."""
    from tensorlbm_b200 import batch, scan

    from tests.conftest import golden

    g = golden("cavity_case")
    res = {"bgk32": 32, "mrt24": 24, "mrt6x20x40": (6, 20, 40)}
    for collision, tags in (("bgk", ["bgk32"]), ("mrt", ["mrt24", "mrt6x20x40"])):
        pts = [dict(resolution=res[t], re=float(g[f"{t}_re"]), u_lid=float(g[f"{t}_u_lid"])) for t in tags]
        for t, p in zip(tags, pts):
            d = batch.cavity_point(p["resolution"], p["re"], u_lid=p["u_lid"], device=cuda)
            assert d.tau == float(g[f"{t}_tau"]) and d.shape == tuple(int(v) for v in g[f"{t}_shape"])
        steps = int(g[f"{tags[0]}_steps"])
        fs = scan.run_cavity_points(pts, steps, collision=collision, device=cuda, mode=mode)
        for t, f in zip(tags, fs):
            mid = f[:, f.shape[1] // 2].cpu().numpy()
            qsum = f.double().sum(dim=(1, 2, 3)).cpu().numpy()
            if collision == "bgk":
                assert same(mid, g[f"{t}_mid"]), t
                np.testing.assert_allclose(qsum, g[f"{t}_qsum"], rtol=1e-12)
            else:
                assert float(np.max(np.abs(mid - g[f"{t}_mid"]))) <= 1e-5 * float(np.max(np.abs(g[f"{t}_mid"]))), t
                # the MRT chain tolerance: float32 rounding of the BLAS products over 300 steps
                np.testing.assert_allclose(qsum, g[f"{t}_qsum"], rtol=1e-5)


@pytest.mark.parametrize("mode", ["launch", "graph", "persistent"])
def test_retire_skips_diverged_domains(cuda, mode):
    """With retire=True a domain that turns non-finite is skipped from then on
    (its own status word); the other domains still evolve bit for bit as
    without it."""
    from tensorlbm_b200 import batch

    from tests.conftest import golden

    g = golden("c4_divergence")
    design = batch.uniform_scan(512, seed=20261203, device=cuda)
    bad = [int(i) for i in g["domains"]][:4]
    good = [batch.cylinder_channel(nx, re, 0.05, cuda) for nx, re in ((128, 10.0), (160, 12.0))]
    doms = [design[i] for i in bad] + good
    f0 = batch.equilibrium_start(doms, cuda)
    b = batch.BatchedSolver(doms, "bgk", device=cuda, mode=mode, retire=True).load(f0)
    b.run(128)
    assert b.retired_domains().tolist() == [True] * 4 + [False] * 2
    ref = batch.BatchedSolver(good, "bgk", device=cuda, mode=mode).load(f0[4:])
    ref.run(128)
    for k in range(2):
        assert torch.equal(b.f(4 + k), ref.f(k))
    # the next run() drops the retired domains' tiles from the tile list
    n_all = b.ntiles
    b.run(64)
    ref.run(64)
    assert b.ntiles == ref.ntiles < n_all
    for k in range(2):
        assert torch.equal(b.f(4 + k), ref.f(k))
    torch.cuda.synchronize(cuda)
    assert int(b.status.item()) == 0          # the non-finite bits went to the domains' own words
