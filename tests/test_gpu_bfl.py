"""Curved walls (Bouzidi / BFL) on the GPU: the sphere link fields and the
stand-alone update against the reference's own outputs, and the fused step
with the links against the reference's chain (bfl_step order)."""

import numpy as np
import pytest
import torch

from oracle import lbm as O
from tests.conftest import golden, same

pytestmark = pytest.mark.gpu


def N(t):
    return t.detach().cpu().numpy()


def T(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def test_sphere_links_bitwise(cuda):
    from tensorlbm_b200 import bfl

    g = golden("bfl")
    m19, q19 = bfl.compute_q_sphere_common(16, 14, 12, 7.3, 6.6, 5.8, 3.7, cuda, lattice="D3Q19")
    m27, q27 = bfl.compute_q_sphere_27(12, 11, 10, 5.4, 5.1, 4.7, 2.9, cuda)
    assert same(N(m19), g["m19"]) and same(N(q19), g["q19"])
    assert same(N(m27), g["m27"]) and same(N(q27), g["q27"])
    _, _, solid = bfl.sphere_links(16, 14, 12, 7.3, 6.6, 5.8, 3.7, cuda)
    zz, yy, xx = np.meshgrid(*(np.arange(n, dtype=np.float64) for n in (12, 14, 16)), indexing="ij")
    assert same(N(solid), ((xx - 7.3) ** 2 + (yy - 6.6) ** 2 + (zz - 5.8) ** 2) <= 3.7 ** 2)


def test_bfl_update_and_force(cuda):
    from tensorlbm_b200 import bfl

    g = golden("bfl")
    for q in (19, 27):
        out = bfl.bfl_bounce_back_common(T(g[f"f{q}"], cuda), T(g[f"fprev{q}"], cuda), T(g[f"m{q}"], cuda),
                                         T(g[f"q{q}"], cuda), lattice=f"D3Q{q}")
        assert same(N(out), g[f"bfl{q}"])
    out, force = bfl.bouzidi_bounce_back_d3q19(T(g["f19"], cuda), T(g["fprev19"], cuda), T(g["m19"], cuda),
                                               T(g["q19"], cuda), return_force=True)
    assert same(N(out), g["bfl19"])
    got = np.array([float(v) for v in force])
    assert np.max(np.abs(got - g["force19"])) < 1e-5 * np.max(np.abs(g["force19"]))
    assert np.max(np.abs(got - O.bfl_force(g["fprev19"], g["m19"], g["q19"]))) < 1e-6 * np.max(np.abs(got))
    f64 = bfl.bfl_bounce_back_common(T(g["f19"], cuda).double(), T(g["fprev19"], cuda).double(),
                                     T(g["m19"], cuda), T(g["q19"], cuda))
    ref64 = O.bfl_bounce_back(g["f19"].astype(np.float64), g["fprev19"].astype(np.float64), g["m19"], g["q19"])
    assert same(N(f64), ref64)
    with pytest.raises(NotImplementedError):
        bfl.bfl_bounce_back_common(T(g["f19"], cuda), T(g["fprev19"], cuda), T(g["m19"], cuda),
                                   T(g["q19"], cuda), wall_correction=T(g["f19"], cuda))


@pytest.mark.parametrize("coll", ["bgk", "mrt"])
def test_fused_step_with_curved_wall(cuda, coll):
    """The fused step with Bouzidi links against the reference's chain (BGK,
    golden) and the oracle's (MRT): every fluid cell, and the BFL force."""
    from tensorlbm_b200 import LBMSolver, bfl

    g = golden("bfl")
    tau = float(g["chain_tau"])
    wall = bfl.CurvedWall(T(g["chain_mask"], cuda), T(g["chain_q"], cuda), T(g["chain_solid"], cuda))
    s = LBMSolver("D3Q19", (16, 16, 24), tau, coll, device=cuda, curved_wall=wall, track_force=True)
    s.load(T(g["chain_f0"], cuda)).step(8)
    fluid = ~g["chain_solid"]
    if coll == "bgk":
        ref, ref_forces = g["chain_f"], g["chain_forces"]
        assert same(N(s.f)[:, fluid], ref[:, fluid])
    else:
        ref, forces = g["chain_f0"], []
        for _ in range(8):
            ref, fo = O.bfl_chain_step(ref, tau, g["chain_solid"], g["chain_mask"], g["chain_q"], "mrt")
            forces.append(fo)
        ref_forces = np.array(forces)
        err = np.max(np.abs(N(s.f)[:, fluid] - ref[:, fluid])) / np.max(np.abs(ref))
        assert err < 1e-5
    got = N(s.force_history())
    assert np.max(np.abs(got - ref_forces)) < 1e-5 * np.max(np.abs(ref_forces))


def test_curved_wall_half_storage_and_d3q27(cuda):
    """FP16 storage and D3Q27 with a curved sphere: finite, close to float32."""
    from tensorlbm_b200 import LBMSolver, bfl

    for q in (19, 27):
        wall = bfl.sphere_wall(32, 20, 20, 10.3, 9.6, 10.2, 4.1, cuda, lattice=f"D3Q{q}")
        ux = torch.full((20, 20, 32), 0.04, device=cuda)
        ux[wall.solid] = 0.0
        z = torch.zeros_like(ux)
        f0 = T(O.equilibrium(q, np.ones((20, 20, 32), np.float32), N(ux), N(z), N(z)), cuda)
        runs = {}
        for storage in ("f32", "f16"):
            s = LBMSolver(q, (20, 20, 32), 0.55, "bgk", device=cuda, storage=storage, curved_wall=wall,
                          u_in=0.04, rho_out=1.0, track_force=True)
            s.load(f0).step(30)
            assert not s.nonfinite_seen()
            runs[storage] = (N(s.f), N(s.force_history()))
        fluid = ~N(wall.solid)
        assert np.max(np.abs(runs["f16"][0][:, fluid] - runs["f32"][0][:, fluid])) < 2e-4
        assert np.max(np.abs(runs["f16"][1] - runs["f32"][1])) < 2e-2 * np.max(np.abs(runs["f32"][1]))
