"""Link-wise momentum exchange (tlbm_link_momentum_sums) against the reference's
MEM variants (golden vectors of momentum_exchange.py) and the oracle, plus a
property at a size the oracle would be slow on: on a periodic domain whose near
mask holds every fluid neighbour of the solid, links in q and opp(q) are equally
many, so the uniform background cancels exactly."""

import numpy as np
import pytest
import torch

from oracle import lbm as O
from tests.conftest import golden

pytestmark = pytest.mark.gpu


def T(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_mem_variants_match_reference(cuda, tag):
    from tensorlbm_b200 import momentum_exchange as me

    g = golden("mem")
    f, solid, near = T(g[f"f_{tag}"], cuda), T(g["solid"], cuda), T(g["near"], cuda)
    qs, qd = T(g["q_scalar"], cuda), T(g["q_dir"], cuda)
    got = {"standard": me.momentum_exchange_standard(f, solid, near),
           "galilean": me.momentum_exchange_galilean(f, solid, near, 0.6),
           "background": me.momentum_exchange_background_subtracted(f, solid, near, rho0=1.02, u0=(0.05, 0.01, -0.02)),
           "bfl_scalar": me.momentum_exchange_bfl(f, solid, near, qs),
           "bfl_dir": me.momentum_exchange_bfl(f, solid, near, qd)}
    # the reference sums each direction in f's dtype; the bound is a few ulp of
    # the per-direction sums (the oracle's own golden test uses the same one)
    eps = 2e-7 if tag == "f32" else 1e-13
    for name, val in got.items():
        qw = {"bfl_scalar": g["q_scalar"], "bfl_dir": g["q_dir"]}.get(name)
        scale = 2.0 * np.abs(O.link_momentum_sums(g[f"f_{tag}"], g["solid"], g["near"], qw)[:19]).sum()
        assert np.abs(np.array(val) - g[f"{name}_{tag}"]).max() <= eps * scale, name


@pytest.mark.parametrize("q,shape", [(9, (1, 40, 48)), (19, (12, 14, 16)), (27, (10, 12, 14))])
@pytest.mark.parametrize("weighted", [False, True])
def test_link_sums_match_oracle(cuda, q, shape, weighted):
    from tensorlbm_b200 import momentum_exchange as me

    rng = np.random.default_rng(q + 100 * weighted)
    f = rng.random((q,) + shape).astype(np.float32)
    solid = rng.random(shape) < 0.15
    near = (~solid) & (rng.random(shape) < 0.7)
    qw = rng.random((q,) + shape).astype(np.float32) if weighted else None
    if q == 9:
        f, solid, near = f[:, 0], solid[0], near[0]
        qw = None if qw is None else qw[:, 0]
    ref = O.link_momentum_sums(f, solid, near, qw)
    got = me.link_momentum_sums(T(f, cuda), T(solid, cuda), T(near, cuda),
                                None if qw is None else T(qw, cuda)).cpu().numpy()
    assert np.array_equal(got[q:], ref[q:])                                   # link counts exact
    assert np.allclose(got[:q], ref[:q], rtol=1e-12, atol=1e-9)               # float64 sums, other order


def test_background_cancels_on_closed_periodic_surface(cuda):
    from tensorlbm_b200 import boundaries3d
    from tensorlbm_b200 import momentum_exchange as me

    nz, ny, nx = 128, 160, 192
    solid = boundaries3d.sphere_mask(nx, ny, nz, 70.3, 80.2, 63.9, 21.0, cuda)
    nb = torch.zeros_like(solid)
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                nb |= torch.roll(solid, (dz, dy, dx), dims=(0, 1, 2))
    near = nb & ~solid
    f = 0.05 + 0.01 * torch.rand((19, nz, ny, nx), device=cuda, generator=torch.Generator(cuda).manual_seed(3))
    sums = me.link_momentum_sums(f, solid, near).cpu().numpy()
    opp = O.opposite(19)
    assert sums[19:].sum() > 1000 and np.array_equal(sums[19 + 1:], sums[19 + opp[1:]])
    std = np.array(me.momentum_exchange_standard(f, solid, near))
    bg = np.array(me.momentum_exchange_background_subtracted(f, solid, near, rho0=1.0, u0=(0.04, 0.0, 0.0)))
    assert np.allclose(bg, std, rtol=0, atol=1e-9 * np.abs(sums[:19]).sum())
    gal = np.array(me.momentum_exchange_galilean(f, solid, near, 0.55))
    assert np.allclose(gal, std * (1.0 + 1.0 / 1.1), rtol=1e-12, atol=1e-12)


def test_argument_errors(cuda):
    from tensorlbm_b200 import momentum_exchange as me

    f = torch.zeros((19, 4, 5, 6), device=cuda)
    m = torch.zeros((4, 5, 6), dtype=torch.bool, device=cuda)
    with pytest.raises(ValueError):
        me.link_momentum_sums(f, m[:, :, :5], m)
    with pytest.raises(ValueError):
        me.momentum_exchange_bfl(f, m, m, torch.ones((3, 4, 5, 6), device=cuda))
    with pytest.raises(NotImplementedError):
        me.compare_all_methods(f, m, m, None, 1.0, 0.1, 0.6)
