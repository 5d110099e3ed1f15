"""Z-slab decomposition on the GPU: several slabs driven by one process on
cuda:0 (the ranks' kernels never wait on one another: the lanes are copied
between steps) against the undivided LBMSolver run, bit for bit in float32,
with a sphere obstacle, Zou/He planes and the drag; the one-slab loopback path;
the DistributedTritonFusedSolver3D surface against triton_fused; and
tlbm_step_planes' argument checks."""

import ctypes

import numpy as np
import pytest
import torch

from oracle import lbm as O

pytestmark = pytest.mark.gpu


def _channel(q, shape, cuda, seed=1):
    from tensorlbm_b200 import boundaries3d

    nz, ny, nx = shape
    obst = boundaries3d.sphere_mask(nx, ny, nz, nx / 3 + 0.3, ny / 2 - 0.4, nz / 2 + 0.2, min(ny, nz) / 4, cuda)
    rng = np.random.default_rng(seed)
    ux = 0.04 + 0.005 * rng.standard_normal(shape)
    ux[obst.cpu().numpy()] = 0.0
    uy, uz = (0.005 * rng.standard_normal(shape) for _ in range(2))
    f0 = torch.from_numpy(O.equilibrium(q, np.ones(shape), ux, uy, uz).astype(np.float32)).to(cuda)
    return obst, f0


@pytest.mark.parametrize("q,coll,nx", [(19, "mrt", 24), (19, "bgk", 23), (27, "cumulant", 16)])
@pytest.mark.parametrize("n_slabs", [2, 3])
def test_slabs_equal_undivided(cuda, q, coll, nx, n_slabs):
    from tensorlbm_b200 import LBMSolver
    from tensorlbm_b200.slabs import MultiSlabSolver

    shape = (6 * n_slabs, 10, nx)
    obst, f0 = _channel(q, shape, cuda)
    kw = dict(obstacle_mask=obst, u_in=0.04, rho_out=1.0, track_force=True)
    ref = LBMSolver(q, shape, 0.56, coll, device=cuda, **kw).load(f0).step(7)
    ms = MultiSlabSolver(q, shape, 0.56, coll, devices=(cuda,), n_slabs=n_slabs, **kw).load(f0).step(7)
    assert torch.equal(ms.gather(), ref.f)
    fr, fm = ref.force_history(), ms.force_history()
    assert torch.allclose(fm, fr, rtol=1e-12, atol=1e-12 * float(fr.abs().max()))
    assert not ms.nonfinite_seen()


def test_one_slab_loopback_with_overlap(cuda):
    from tensorlbm_b200 import LBMSolver
    from tensorlbm_b200.slabs import SlabSolver

    shape = (12, 10, 24)
    obst, f0 = _channel(19, shape, cuda, seed=2)
    kw = dict(obstacle_mask=obst, u_in=0.04, rho_out=1.0, track_force=True)
    ref = LBMSolver("D3Q19", shape, 0.58, "mrt", device=cuda, **kw).load(f0).step(9)
    s = SlabSolver("D3Q19", shape, 0.58, "mrt", device=cuda, world=1, rank=0, **kw).load(f0).step(9)
    assert torch.equal(s.f, ref.f)
    assert torch.allclose(s.global_force_history(), ref.force_history(), rtol=1e-12, atol=1e-15)
    owned = torch.from_numpy(np.ascontiguousarray(ref.f.cpu().numpy())).to(cuda)
    s2 = SlabSolver("D3Q19", shape, 0.58, "mrt", device=cuda, world=1, rank=0, **kw).load(owned)
    assert torch.equal(s2.step(3).f, LBMSolver("D3Q19", shape, 0.58, "mrt", device=cuda, **kw).load(owned).step(3).f)


def test_half_storage_slabs_close(cuda):
    from tensorlbm_b200 import LBMSolver
    from tensorlbm_b200.slabs import MultiSlabSolver

    shape = (12, 10, 24)
    obst, f0 = _channel(19, shape, cuda, seed=3)
    kw = dict(obstacle_mask=obst, u_in=0.04, rho_out=1.0, storage="f16")
    ref = LBMSolver("D3Q19", shape, 0.56, "bgk", device=cuda, **kw).load(f0).step(10).f
    got = MultiSlabSolver("D3Q19", shape, 0.56, "bgk", devices=(cuda,), n_slabs=2, **kw).load(f0).step(10).gather()
    # the stochastic rounding bits hash the local cell index: not the same bits
    assert float((got - ref).abs().max()) < 2e-4


def test_distributed_surface_single_rank(cuda):
    from tensorlbm_b200 import triton_fused
    from tensorlbm_b200.triton_fused_distributed import DistributedTritonFusedSolver3D

    nz, ny, nx = 16, 12, 20
    g = torch.Generator(cuda).manual_seed(7)
    f = 1.0 / 19 + 1e-3 * torch.randn((19, nz, ny, nx), device=cuda, generator=g)
    sol = DistributedTritonFusedSolver3D(nz, ny, nx, 0.6, cuda)
    loc = sol.from_global(f)
    assert loc.shape == sol.local_shape == (19, nz + 2, ny, nx)
    ref = f
    for _ in range(6):
        loc = sol.step(loc)
        ref = triton_fused.triton_fused(ref, 0.6)
    sol.synchronize()
    assert torch.equal(sol.to_global(loc), ref)
    assert sol.halo_bytes_per_step() == 0 and sol.staging_bytes() == 0 and sol.grid_size_cells() == nz * ny * nx


def test_step_planes_checks(cuda):
    from tensorlbm_b200 import _lib, _ops

    f = torch.zeros((19, 6, 4, 8), device=cuda)
    out = torch.empty_like(f)
    d = _ops.make_desc(19, (8, 4, 6), _lib.F32, _lib.COLL_BGK, 0.6)
    lib = _lib.load()
    s = _lib.stream_of(torch.device(cuda))
    for z0, nz in ((0, 0), (-1, 2), (5, 2), (0, 7)):
        assert lib.tlbm_step_planes(ctypes.byref(d), f.data_ptr(), out.data_ptr(), None, None, None, None,
                                    z0, nz, s) == _lib.ERR_SHAPE
    assert lib.tlbm_step_planes(ctypes.byref(d), f.data_ptr(), f.data_ptr(), None, None, None, None, 1, 4, s) \
        == _lib.ERR_ALIAS
