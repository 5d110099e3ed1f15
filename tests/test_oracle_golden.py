"""Pin the numpy oracle to TensorLBM: every oracle function against the golden
vectors produced by the unmodified reference (tests/golden/make_golden.py).

The oracle restates the reference's arithmetic order, including torch's CPU
summation order over the direction axis (oracle.lbm.sum0), so on the golden
shapes (inner sizes that are multiples of 32) it reproduces TensorLBM bit for
bit: operators, boundary planes and whole multi-step chains.  CPU only."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import lbm as O
from tests.conftest import golden


def same(a, b):
    """bitwise equality, NaN == NaN"""
    a = np.asarray(a)
    b = np.asarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("q", [9, 19, 27])
def test_moments_and_equilibrium(q, tag):
    g = golden(f"moments_d{'2' if q == 9 else '3'}q{q}_{tag}")
    rho, ux, uy, uz = O.macroscopic(g["f"])
    assert same(rho, g["rho"]) and same(ux, g["ux"]) and same(uy, g["uy"])
    if q != 9:
        assert same(uz, g["uz"])
    assert same(O.equilibrium(q, g["rho_in"], g["ux_in"], g["uy_in"], None if q == 9 else g["uz_in"]), g["feq"])


def test_collide_d2q9():
    g = golden("collide_d2q9_f32")
    f, tau = g["f"], float(g["tau"])
    assert same(O.collide_bgk(f, tau), g["bgk"])
    assert same(O.collide_mrt(f, tau), g["mrt"])
    assert same(O.collide_mrt(f, tau, tau_field=g["tau_field"]), g["mrt_field"])
    assert same(O.collide_smagorinsky(f, tau, 0.17), g["smag"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_collide_d3q19(tag):
    g = golden(f"collide_d3q19_{tag}")
    f, tau = g["f"], float(g["tau"])
    assert same(O.collide_bgk(f, tau), g["bgk"])
    assert same(O.collide_smagorinsky(f, tau, 0.17), g["smag"])
    assert same(O.collide_cumulant_d3q19(f, tau, omega_b=1.2, omega_even=0.8), g["cum19"])
    assert same(O.collide_cumulant_d3q19(f, tau, omega_b=1.2, omega_even=0.8, c_s=0.17), g["cum19_smag"])
    if "mrt" in g:
        assert same(O.collide_mrt(f, tau), g["mrt"])
        assert same(O.collide_mrt(f, tau, s_e=1.3, s_eps=1.5, s_q=1.1, s_pi=1.25), g["mrt_custom"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_collide_d3q27(tag):
    g = golden(f"collide_d3q27_{tag}")
    f, tau = g["f"], float(g["tau"])
    assert same(O.collide_bgk(f, tau), g["bgk"])
    assert same(O.collide_smagorinsky(f, tau, 0.17), g["smag"])
    assert same(O.collide_cumulant_d3q27(f, tau, 1.1, 1.2, 0.9), g["cum"])
    assert same(O.collide_cumulant_geier_d3q27(f, tau, 1.1, 1.2, 0.9), g["geier"])
    if "mrt" in g:
        assert same(O.collide_mrt(f, tau), g["mrt"])


def test_stream_canary_bitwise():
    g = golden("stream")
    for q in (9, 19, 27):
        assert same(O.stream(g[f"f{q}"]), g[f"s{q}"])


@pytest.mark.parametrize("q", [9, 19, 27])
def test_boundaries(q):
    g = golden(f"bc_d{'2' if q == 9 else '3'}q{q}")
    f, m = g["f"], g["mask"]
    assert same(O.bounce_back(f, m), g["bb"])
    if q == 9:
        assert same(O.zou_he_inlet(f, 0.05, 0.01), g["inlet"])
        assert same(O.zou_he_outlet(f, 1.02), g["outlet"])
        assert same(O.moving_lid(f, 0.07), g["lid"])
    else:
        assert same(O.zou_he_inlet(f, 0.04, 0.01, -0.005), g["inlet"])
        assert same(O.zou_he_outlet(f, 0.98), g["outlet"])
        if q == 19:
            assert same(O.moving_lid(f, 0.05), g["lid"])
    # the reference sums the force in float32, the oracle in float64
    ref = g["force"].astype(np.float64)
    got = O.obstacle_force(f, m)[: len(ref)]
    assert np.max(np.abs(got - ref)) < 1e-6 * max(np.max(np.abs(ref)), 1.0)


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_moving_wall(tag):
    g = golden("moving_wall")
    for f, m, uw, key in ((g[f"f9_{tag}"], g["disc"], (g["ux2"], g["uy2"]), f"mw9_{tag}"),
                          (g[f"f19_{tag}"], g["rotor"], (g["ux3"], g["uy3"], g["uz3"]), f"mw19_{tag}")):
        out = O.moving_wall_bounce_back(f, m, *uw)
        assert same(out[:, m], g[key])
        assert same(out[:, ~m], f[:, ~m])


def test_masks_bitwise():
    g = golden("masks")
    assert np.array_equal(O.sphere_mask(32, 16, 16, 12.0, 8.0, 8.0, 4.5), g["sphere"])
    assert np.array_equal(O.sphere_mask(40, 24, 20, 17.3, 11.7, 9.1, 6.35), g["sphere_odd"])
    assert np.array_equal(O.cylinder_mask(200, 50, 25.0, 25.0, 3.125), g["cylinder"])
    assert np.array_equal(O.cylinder_mask(97, 31, 20.4, 15.5, 4.7), g["cylinder_odd"])
    big = O.sphere_mask(512, 256, 256, 128, 128, 128, 16)
    assert int(big.sum()) == int(g["big_count"])
    assert np.array_equal(np.flatnonzero(big), g["big_index"])


def test_missing_mask_and_links():
    g = golden("masks")
    sph = g["sphere"]
    m19 = O.missing_mask(19, sph.shape, sph, periodic=(True, True, False))
    ref19 = np.unpackbits(g["missing19"])[: m19.size].reshape(tuple(g["missing19_shape"])).astype(bool)
    assert np.array_equal(m19, ref19)
    assert np.array_equal(np.argwhere(m19), g["links19"])
    m27 = O.missing_mask(27, sph.shape, sph, periodic=(False, False, False))
    ref27 = np.unpackbits(g["missing27"])[: m27.size].reshape(tuple(g["missing27_shape"])).astype(bool)
    assert np.array_equal(m27, ref27)


@pytest.mark.parametrize("coll", ["bgk", "mrt"])
@pytest.mark.parametrize("mode", ["fullway", "halfway", "fullway_window"])
def test_chain_cavity(coll, mode):
    """12^3 cavity chains.  Where the reference diverges (NaN) inside the
    window the oracle must diverge at the same step."""
    g = golden(f"chain_cavity_d3q19_{coll}_{mode}")
    f = g["f0"]
    nan_step = -1
    with np.errstate(all="ignore"):
        for s in range(1, int(g["steps"]) + 1):
            f = O.cavity_step(f, float(g["tau"]), g["wall"], float(g["u_lid"]), coll,
                              mode="halfway" if mode == "halfway" else "fullway")
            if nan_step < 0 and not np.isfinite(f).all():
                nan_step = s
    assert nan_step == int(g.get("nan_step", -1))
    assert same(f, g["f"])


def test_chain_cylinder_d2q9():
    g = golden("chain_cylinder_d2q9_bgk")
    f = g["f0"]
    forces = []
    for _ in range(int(g["steps"])):
        f, fo = O.channel_step(f, float(g["tau"]), float(g["u_in"]), 1.0, g["wall"], g["obstacle"], "bgk")
        forces.append(fo[:2])
    assert same(f, g["f"])
    ref = g["forces"].astype(np.float64)
    assert np.max(np.abs(np.array(forces) - ref)) < 1e-5 * np.max(np.abs(ref))


@pytest.mark.parametrize("name,coll", [("d3q19_mrt", "mrt"), ("d3q19_bgk", "bgk"), ("d3q27_cumulant", "cumulant"),
                                       ("d3q27_geier", "cumulant_geier"), ("d3q27_bgk", "bgk")])
def test_chain_sphere(name, coll):
    g = golden(f"chain_sphere_{name}")
    f = g["f0"]
    forces = []
    for _ in range(int(g["steps"])):
        f, fo = O.channel_step(f, float(g["tau"]), float(g["u_in"]), 1.0, None, g["obstacle"], coll)
        forces.append(fo)
    assert same(f, g["f"])
    ref = g["forces"].astype(np.float64)
    assert np.max(np.abs(np.array(forces)[:, :3] - ref)) < 1e-5 * np.max(np.abs(ref[:, 0]))


def test_collide_trt():
    """TRT (solver.py:440, solver3d.py:303, d3q27.py:438): the oracle against
    the reference's own outputs, bit for bit, default and custom Lambda."""
    g = golden("collide_trt")
    assert same(O.collide_trt(g["f9"], 0.6), g["trt9"])
    assert same(O.collide_trt(g["f9"], 0.57, 0.25), g["trt9_lam"])
    for tag in ("f32", "f64"):
        for q in (19, 27):
            assert same(O.collide_trt(g[f"f{q}_{tag}"], 0.6), g[f"trt{q}_{tag}"])
            assert same(O.collide_trt(g[f"f{q}_{tag}"], 0.57, 0.25), g[f"trt{q}_lam_{tag}"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("q", [9, 19, 27])
def test_collide_rlbm(q, tag):
    """Regularised BGK (solver.py:338, solver3d.py:342, d3q27.py:481): the
    oracle against the reference's own outputs, bit for bit, near equilibrium
    (tau 0.6 and 0.5046) and with 5 % seeded ghost-mode content (tau 0.53)."""
    g = golden("collide_rlbm")
    assert same(O.collide_rlbm(g[f"f{q}_{tag}"], 0.6), g[f"rlbm{q}_{tag}"])
    assert same(O.collide_rlbm(g[f"f{q}_{tag}"], 0.5046), g[f"rlbm{q}_low_{tag}"])
    assert same(O.collide_rlbm(g[f"fr{q}_{tag}"], 0.53), g[f"rlbmr{q}_{tag}"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_far_field(tag):
    """Free-stream far field (boundaries.py:199, boundaries3d.py:446,
    boundaries_d3q27.py:63): the oracle against the reference's outputs, bit
    for bit, with the obstacle bounce-back after it."""
    g = golden("far_field")
    ob9, ob3 = g["ob9"], g["ob3"]
    assert same(O.bounce_back(O.far_field(g[f"f9_{tag}"], 0.07), ob9), g[f"ff9_{tag}"])
    assert same(O.bounce_back(O.far_field(g[f"f19_{tag}"], 0.06), ob3), g[f"ff19_{tag}"])
    assert same(O.far_field(g[f"f19_{tag}"], 0.06, z_faces=False), g[f"ff19y_{tag}"])
    assert same(O.far_field(g[f"f19_{tag}"], 0.06, 0.01, -0.02), g[f"ff19uv_{tag}"])
    assert same(O.bounce_back(O.far_field(g[f"f27_{tag}"], 0.05), ob3), g[f"ff27_{tag}"])


def test_bfl_links_update_and_chain():
    """Bouzidi links of a sphere (bfl_common.py:384, interpolated_bc_common.py:136),
    the link update (bfl_common.py:106) and the 8-step chain in bfl_step's
    order: bit for bit against the reference; the force ledger (float64 here,
    float32 sums there) to float32 rounding."""
    g = golden("bfl")
    m19, q19 = O.sphere_links(19, 16, 14, 12, 7.3, 6.6, 5.8, 3.7)
    m27, q27 = O.sphere_links(27, 12, 11, 10, 5.4, 5.1, 4.7, 2.9)
    assert same(m19, g["m19"]) and same(q19, g["q19"]) and same(m27, g["m27"]) and same(q27, g["q27"])
    assert same(O.bfl_bounce_back(g["f19"], g["fprev19"], g["m19"], g["q19"]), g["bfl19"])
    assert same(O.bfl_bounce_back(g["f27"], g["fprev27"], g["m27"], g["q27"]), g["bfl27"])
    fo = O.bfl_force(g["fprev19"], g["m19"], g["q19"])
    assert np.max(np.abs(fo - g["force19"])) < 1e-5 * np.max(np.abs(g["force19"]))
    f, forces = g["chain_f0"], []
    for _ in range(8):
        f, fo = O.bfl_chain_step(f, float(g["chain_tau"]), g["chain_solid"], g["chain_mask"], g["chain_q"])
        forces.append(fo)
    assert same(f, g["chain_f"])
    assert np.max(np.abs(np.array(forces) - g["chain_forces"])) < 1e-5 * np.max(np.abs(g["chain_forces"]))


def test_collide_cascaded():
    """Cascaded central-moment collisions (cascaded_collision.py:445, :512): the
    oracle against the reference's outputs (its float32 matrix products are
    restated with numpy's, equal here to rounding)."""
    g = golden("collide_cascaded")
    for tag, tol in (("f32", 1e-6), ("f64", 1e-13)):
        for q in (19, 27):
            f = g[f"f{q}_{tag}"]
            assert np.max(np.abs(O.collide_cascaded(f, 0.6) - g[f"c{q}_{tag}"])) < tol * np.max(np.abs(f))
            kw = dict(s_bulk=1.2, s_3=0.9, s_4=1.3) if q == 19 else dict(s_bulk=1.2, s_3=0.9, s_4=1.3, s_5=1.1, s_6=0.8)
            assert np.max(np.abs(O.collide_cascaded(f, 0.57, **kw) - g[f"c{q}r_{tag}"])) < tol * np.max(np.abs(f))


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_mem_variants_against_reference(tag):
    """Standard, Galilean, background-subtracted and BFL-weighted link-wise
    momentum exchange (momentum_exchange.py:75-360).  The reference sums each
    direction in the populations' dtype, the oracle in float64: the bound is a
    few units in the last place of the per-direction sums."""
    g = golden("mem")
    f, solid, near = g[f"f_{tag}"], g["solid"], g["near"]
    eps = 2e-7 if tag == "f32" else 1e-13
    cases = {"standard": (None, dict()), "galilean": (None, dict(variant="galilean", tau=0.6)),
             "background": (None, dict(variant="background", rho0=1.02, u0=(0.05, 0.01, -0.02))),
             "bfl_scalar": (g["q_scalar"], dict(variant="bfl")), "bfl_dir": (g["q_dir"], dict(variant="bfl"))}
    for name, (qw, kw) in cases.items():
        sums = O.link_momentum_sums(f, solid, near, qw)
        got = O.mem_force(sums, **kw)
        tol = eps * 2.0 * np.abs(sums[:19]).sum()
        assert np.abs(got - g[f"{name}_{tag}"]).max() <= tol, name
    assert O.link_momentum_sums(f, solid, near)[19:].sum() > 100          # links on the sphere and the x wall


def c2_links_decoded(g, tag):
    """Flat row-major (q, z, y, x) indices of the 512x256x256 link list."""
    return np.cumsum(g[f"delta_{tag}"].astype(np.int64))


@pytest.mark.parametrize("tag", ["q19", "q27"])
def test_links_c2_full_size(tag):
    """The full-size sphere-channel link list (512x256x256, sphere D = 32 at
    (128, 128, 128), periodic y/z, closed x) that torch.nonzero returned for
    the reference's missing mask: the stored digest of its int64 rows, and the
    oracle's missing mask over the whole grid.  The oracle runs on the band of
    48 planes around the sphere (a periodic-z subdomain holds the same links
    there, since no solid lies near the band's edges); every other plane is an
    empty periodic slice, checked against the oracle's own empty-slab mask."""
    import hashlib

    g = golden("links_c2")
    nz, ny, nx = (int(v) for v in g["shape"])
    q = int(g[f"q_{tag}"])
    flat = c2_links_decoded(g, tag)
    assert flat.size == int(g[f"count_{tag}"])
    rows = np.stack(np.unravel_index(flat, (q, nz, ny, nx)), axis=1).astype(np.int64)
    assert hashlib.sha256(np.ascontiguousarray(rows).tobytes()).digest() == g[f"sha256_{tag}"].tobytes()

    z0, z1 = 104, 152
    band = O.missing_mask(q, (z1 - z0, ny, nx), O.sphere_mask(nx, ny, z1 - z0, 128, 128, 128 - z0, 16),
                          periodic=(True, True, False))
    empty = O.missing_mask(q, (2, ny, nx), None, periodic=(True, True, False))[:, 0]
    expect = []
    for i in range(q):
        full = np.broadcast_to(empty[i], (nz, ny, nx)).copy()
        full[z0:z1] = band[i]
        expect.append(np.flatnonzero(full) + i * nz * ny * nx)
    assert np.array_equal(np.concatenate(expect), flat)


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("q", [9, 19, 27])
def test_correct_mass(q, tag):
    """Global mass correction (solver.py:420, solver3d.py:287, d3q27.py:729).
    The reference sums in the field dtype in torch's order, the oracle in
    float64: the bound is the rounding of the sum."""
    g = golden("mass")
    ref = g[f"m{q}_{tag}"]
    got = O.correct_mass(g[f"f{q}_{tag}"], float(g[f"t{q}_{tag}"]))
    tol = 1e-6 if tag == "f32" else 1e-14
    assert got.dtype == ref.dtype and np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
    assert same(O.correct_mass(np.zeros((19, 2, 3, 4), np.float32), 5.0), g["zero_out"])


def test_c4_divergence_onset():
    """The oracle's D2Q9 cylinder chain on the smallest design points of the
    batched scan: bit-exact to TensorLBM up to the last finite state the
    fixture holds, and non-finite at the same step as TensorLBM."""
    g = golden("c4_divergence")
    for i in (118, 364):
        nx = 128
        ny = nx // 4
        d = ny / 8.0
        tau = float(g[f"tau_{i}"])
        obst = O.cylinder_mask(nx, ny, ny / 2.0, ny / 2.0, d / 2.0)
        wall = np.zeros((ny, nx), bool)
        wall[0, :] = wall[-1, :] = True
        wall[obst] = False
        ux = np.full((ny, nx), 0.05, np.float32)
        ux[obst] = 0.0
        f = O.equilibrium(9, np.ones((ny, nx), np.float32), ux, np.zeros_like(ux))
        onset = -1
        with np.errstate(all="ignore"):
            for step in range(1, 100):
                f, _ = O.channel_step(f, tau, 0.05, 1.0, wall, obst)
                if step == int(g[f"check_step_{i}"]):
                    assert same(f, g[f"check_{i}"])
                if not np.isfinite(f).all():
                    onset = step
                    break
        assert onset == int(g[f"nan_step_{i}"])
