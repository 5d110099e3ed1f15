"""AA pattern (one buffer, in place) against the two-buffer step: the same
TensorLBM-phase populations bit for bit in float32 after odd and even step
counts, with obstacles, Zou/He planes, walls and the drag; half storage to
storage precision; graph replay, moment sums and an exact checkpoint resume."""

import numpy as np
import pytest
import torch

from oracle import lbm as O
from tests.conftest import golden

pytestmark = pytest.mark.gpu


def T(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _sphere_channel(cuda, q, coll, steps, storage="f32", nx=24, **kw):
    from tensorlbm_b200 import LBMSolver, boundaries3d

    nz, ny = 9, 10
    obst = boundaries3d.sphere_mask(nx, ny, nz, 8.0, 5.0, 4.0, 2.3, cuda)
    ux = np.full((nz, ny, nx), 0.04, np.float32)
    ux[obst.cpu().numpy()] = 0.0
    z = np.zeros_like(ux)
    f0 = T(O.equilibrium(q, np.ones_like(ux), ux, z, z), cuda)
    out = {}
    for pattern in ("ab", "aa"):
        s = LBMSolver(q, (nz, ny, nx), 0.56, coll, device=cuda, storage=storage, obstacle_mask=obst, u_in=0.04,
                      rho_out=1.0, track_force=True, pattern=pattern, **kw)
        s.load(f0).step(steps)
        out[pattern] = s
    return out["ab"], out["aa"]


@pytest.mark.parametrize("steps", [7, 8])
@pytest.mark.parametrize("q,coll", [(19, "mrt"), (19, "bgk"), (27, "cumulant"), (19, "trt"), (27, "cascaded")])
def test_aa_equals_two_buffers_float32(cuda, q, coll, steps):
    ab, aa = _sphere_channel(cuda, q, coll, steps)
    assert aa.aa_layout == 1 - steps % 2 and ab.aa_layout is None
    assert torch.equal(aa.f, ab.f)
    fa, fb = aa.force_history(), ab.force_history()
    assert fa.shape == fb.shape
    assert torch.allclose(fa, fb, rtol=1e-12, atol=1e-12 * float(fb.abs().max()))
    assert aa.state.data_ptr() == aa._buf[0].data_ptr() and len(aa._buf) == 1


def test_aa_forced_and_odd_nx(cuda):
    """Linear forcing (load and steps) and an odd nx (the two-buffer run then
    uses one cell per thread as well)."""
    ab, aa = _sphere_channel(cuda, 19, "bgk", 9, nx=23, force_lin=1e-4)
    assert torch.equal(aa.f, ab.f)


@pytest.mark.parametrize("q,coll,steps", [(19, "mrt", 7), (27, "cumulant", 8)])
def test_aa_one_cell_per_thread(cuda, q, coll, steps):
    """Odd nx: the AA steps take one cell per thread, the even-nx runs above
    two; both match the two-buffer step bit for bit."""
    ab, aa = _sphere_channel(cuda, q, coll, steps, nx=23)
    assert torch.equal(aa.f, ab.f)


def test_aa_pair_forced_rows(cuda):
    """Forced steps on an even nx keep one cell per thread; the unforced pair
    steps around them must agree with it."""
    ab, aa = _sphere_channel(cuda, 19, "mrt", 10, force_lin=2e-5)
    assert torch.equal(aa.f, ab.f)


def test_aa_d2q9_walls(cuda):
    from tensorlbm_b200 import LBMSolver

    g = golden("chain_cylinder_d2q9_bgk")
    sp = g["obstacle"].shape
    res = {}
    for pattern in ("ab", "aa"):
        s = LBMSolver("D2Q9", sp, float(g["tau"]), "bgk", device=cuda, wall_mask=T(g["wall"], cuda),
                      obstacle_mask=T(g["obstacle"], cuda), u_in=float(g["u_in"]), rho_out=1.0, pattern=pattern)
        res[pattern] = s.load(T(g["f0"], cuda)).step(int(g["steps"])).f
    assert torch.equal(res["aa"], res["ab"])
    assert np.array_equal(res["aa"].cpu().numpy(), g["f"])    # and the reference's own chain


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_aa_half_storage(cuda, storage):
    ab, aa = _sphere_channel(cuda, 19, "bgk", 12, storage=storage)
    tol = 2e-4 if storage == "f16" else 1e-3
    assert float((aa.f - ab.f).abs().max() / ab.f.abs().max()) < tol


def test_aa_graph_and_exact_resume(cuda, tmp_path):
    from tensorlbm_b200 import checkpoint as C

    ab, aa = _sphere_channel(cuda, 19, "mrt", 0)
    ref = _sphere_channel(cuda, 19, "mrt", 0)[1]
    ref.track_force = False
    ref.step(41)
    aa.track_force = False
    aa.run(41, chunk=10)                                   # graph replays of 10 steps, then 1 eager
    assert torch.equal(aa.f, ref.f)
    C.save_solver(aa, tmp_path / "aa.pt")
    again = _sphere_channel(cuda, 19, "mrt", 0)[1]
    again.track_force = False
    C.load_solver(tmp_path / "aa.pt", again)
    assert again.aa_layout == aa.aa_layout == 0 and again.step_index == 41
    again.step(9)
    ref.step(9)
    assert torch.equal(again.f, ref.f)
