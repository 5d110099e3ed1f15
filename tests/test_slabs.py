"""Z-slab decomposition host logic on CPU: the crossing-lane tables, the
ghost-plane layout and the halo exchange over gloo ranks (2 and 3) and within
one process.  The per-slab step here is the oracle's periodic pull + collision
over the padded slab (only the owned planes are kept, as the slab kernel
does), so the test isolates what the slab layer adds: after every exchange the
owned planes must equal the undivided oracle run exactly."""

from __future__ import annotations

import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import lbm as O


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _field(q, nz, ny, nx, seed=5):
    rng = np.random.default_rng(seed)
    shape = (nz, ny, nx)
    ux, uy, uz = (0.03 * rng.standard_normal(shape) for _ in range(3))
    rho = 1.0 + 0.01 * rng.standard_normal(shape)
    return O.equilibrium(q, rho, ux, uy, uz).astype(np.float64)


def _slab_step(geom, local: np.ndarray, tau: float, collision: str) -> np.ndarray:
    """The owned planes of collide(stream(local)) over the padded slab; ghost
    planes are left stale (the exchange refills them)."""
    new = O.COLLIDERS[collision](O.stream(local), tau)
    out = local.copy()
    out[:, 1:geom.nz_local + 1] = new[:, 1:geom.nz_local + 1]
    return out


def _reference_run(f, steps, tau, collision):
    for _ in range(steps):
        f = O.COLLIDERS[collision](O.stream(f), tau)
    return f


def test_crossing_tables_and_layout():
    from tensorlbm_b200.slabs import SlabGeometry, crossing_face_indices

    g = SlabGeometry(19, 12, 3, 4, world=3, rank=0)
    assert g.n_cross == 5 and len(g.cross_dn) == 5
    assert all(O.C[19][q][2] == 1 for q in g.cross_up) and all(O.C[19][q][2] == -1 for q in g.cross_dn)
    assert g.padded_planes().tolist() == [11, 0, 1, 2, 3, 4]
    assert (g.left_neighbor, g.right_neighbor) == (2, 1)
    assert SlabGeometry(27, 4, 2, 2).n_cross == 9
    assert g.local_shape == (19, 6, 3, 4) and g.owned_slice() == (1, 5)
    with pytest.raises(ValueError):
        SlabGeometry(19, 10, 3, 4, world=3)
    with pytest.raises(ValueError):
        crossing_face_indices([0, 1, -1], 2)


@pytest.mark.parametrize("collision", ["bgk", "mrt"])
def test_ring_in_one_process_matches_undivided(collision):
    from tensorlbm_b200.slabs import SlabGeometry, exchange_ring

    q, nz, ny, nx, world, steps, tau = 19, 12, 5, 6, 3, 4, 0.6
    f = _field(q, nz, ny, nx)
    geoms = [SlabGeometry(q, nz, ny, nx, world, r) for r in range(world)]
    locals_ = [g.local_from_global(torch.from_numpy(f), dim=1).numpy().copy() for g in geoms]
    for _ in range(steps):
        locals_ = [_slab_step(g, x, tau, collision) for g, x in zip(geoms, locals_)]
        t = [torch.from_numpy(x) for x in locals_]
        exchange_ring(geoms, t)
    ref = _reference_run(f, steps, tau, collision)
    got = np.concatenate([x[:, 1:g.nz_local + 1] for g, x in zip(geoms, locals_)], axis=1)
    assert np.array_equal(got, ref)


def _gloo_rank(rank, world, port, q, shape, steps, wire, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from tensorlbm_b200.slabs import ProcessGroupTransport, SlabGeometry, StagedTransport

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        nz, ny, nx = shape
        f = _field(q, nz, ny, nx)
        g = SlabGeometry(q, nz, ny, nx, world, rank)
        tr = ProcessGroupTransport() if wire is None else StagedTransport(wire)
        local = g.local_from_global(torch.from_numpy(f), dim=1).numpy().copy()
        for _ in range(steps):
            local = _slab_step(g, local, 0.6, "bgk")
            t = torch.from_numpy(local)
            tr.wait(tr.start(g, t))
        out[rank] = local
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,q", [(2, 19), (3, 27)])
def test_gloo_ranks_match_undivided(world, q):
    shape, steps = (4 * world, 4, 5), 3
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, q, shape, steps, None, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
            assert p.exitcode == 0
        res = dict(out)
    ref = _reference_run(_field(q, *shape), steps, 0.6, "bgk")
    got = np.concatenate([res[r][:, 1:shape[0] // world + 1] for r in range(world)], axis=1)
    assert np.array_equal(got, ref)


def test_gloo_float16_wire_is_close():
    world, shape, steps = 2, (8, 4, 5), 3
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, 19, shape, steps, torch.float16, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
            assert p.exitcode == 0
        res = dict(out)
    ref = _reference_run(_field(19, *shape), steps, 0.6, "bgk")
    got = np.concatenate([res[r][:, 1:shape[0] // world + 1] for r in range(world)], axis=1)
    err = np.abs(got - ref).max()
    assert 0 < err < 1e-3                      # the float16 wire rounds the crossing lanes
