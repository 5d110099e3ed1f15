"""GPU parity of the stand-alone operators against TensorLBM's outputs (golden
vectors) and the numpy oracle.  Every call goes through libtlbm.so."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import lbm as O
from tests.conftest import golden, rel_err, same

pytestmark = pytest.mark.gpu

F32_TOL = 2e-6
F64_TOL = 1e-12


def T(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def N(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("q", [9, 19, 27])
def test_moments_equilibrium(cuda, q, tag):
    from tensorlbm_b200 import d2q9, d3q19, d3q27

    g = golden(f"moments_d{'2' if q == 9 else '3'}q{q}_{tag}")
    tol = F32_TOL if tag == "f32" else F64_TOL
    f = T(g["f"], cuda)
    if q == 9:
        rho, ux, uy = d2q9.macroscopic(f)
        feq = d2q9.equilibrium(T(g["rho_in"], cuda), T(g["ux_in"], cuda), T(g["uy_in"], cuda))
    else:
        mod = d3q19 if q == 19 else d3q27
        mac = mod.macroscopic3d if q == 19 else mod.macroscopic27
        eqf = mod.equilibrium3d if q == 19 else mod.equilibrium27
        rho, ux, uy, uz = mac(f)
        assert same(N(uz), g["uz"])
        feq = eqf(*(T(g[k], cuda) for k in ("rho_in", "ux_in", "uy_in", "uz_in")))
    assert feq.dtype == f.dtype
    # bit-exact: same summation order, rounding and IEEE division as torch
    assert same(N(rho), g["rho"]) and same(N(ux), g["ux"]) and same(N(uy), g["uy"])
    assert same(N(feq), g["feq"])


def test_collide_d2q9(cuda):
    from tensorlbm_b200 import solver, turbulence

    g = golden("collide_d2q9_f32")
    f, tau = T(g["f"], cuda), float(g["tau"])
    assert same(N(solver.collide_bgk(f, tau)), g["bgk"])
    assert same(N(turbulence.collide_smagorinsky_bgk(f, tau, C_s=0.17)), g["smag"])
    # MRT: the reference multiplies by float32 M and M^-1 with BLAS; the kernel
    # applies M^-1 S M (f - feq), the same operator with other rounding
    assert rel_err(N(solver.collide_mrt(f, tau)), g["mrt"]) < F32_TOL
    assert rel_err(N(solver.collide_mrt(f, tau, tau_field=T(g["tau_field"], cuda))), g["mrt_field"]) < F32_TOL


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_collide_d3q19(cuda, tag):
    from tensorlbm_b200 import cumulant, solver3d, turbulence

    g = golden(f"collide_d3q19_{tag}")
    tol = F32_TOL if tag == "f32" else F64_TOL
    f, tau = T(g["f"], cuda), float(g["tau"])
    assert same(N(solver3d.collide_bgk3d(f, tau)), g["bgk"])
    assert same(N(turbulence.collide_smagorinsky_bgk3d(f, tau, C_s=0.17)), g["smag"])
    assert same(N(cumulant.collide_cumulant_d3q19(f, tau, omega_b=1.2, omega_even=0.8)), g["cum19"])
    assert same(N(cumulant.collide_cumulant_d3q19(f, tau, omega_b=1.2, omega_even=0.8, C_s=0.17)), g["cum19_smag"])
    if "mrt" in g:
        assert rel_err(N(solver3d.collide_mrt3d(f, tau)), g["mrt"]) < F32_TOL
        assert rel_err(N(solver3d.collide_mrt3d(f, tau, s_e=1.3, s_eps=1.5, s_q=1.1, s_pi=1.25)),
                       g["mrt_custom"]) < F32_TOL


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_collide_d3q27(cuda, tag):
    from tensorlbm_b200 import cumulant, d3q27, turbulence

    g = golden(f"collide_d3q27_{tag}")
    tol = F32_TOL if tag == "f32" else F64_TOL
    f, tau = T(g["f"], cuda), float(g["tau"])
    assert same(N(d3q27.collide_bgk27(f, tau)), g["bgk"])
    assert same(N(turbulence.collide_smagorinsky_bgk27(f, tau, C_s=0.17)), g["smag"])
    assert rel_err(N(cumulant.collide_cumulant_d3q27(f, tau, 1.1, 1.2, 0.9)), g["cum"]) < 5 * tol
    assert rel_err(N(cumulant.collide_cumulant_geier_d3q27(f, tau, 1.1, 1.2, 0.9)), g["geier"]) < 5 * tol
    if "mrt" in g:
        assert rel_err(N(d3q27.collide_mrt27(f, tau)), g["mrt"]) < 5 * F32_TOL


@pytest.mark.parametrize("seed", [0, 1])
def test_collisions_vs_oracle_larger(cuda, seed):
    """Seeded 12x10x8 fields (beyond the golden sizes) against the oracle."""
    from tensorlbm_b200 import cumulant, d3q27, solver3d

    rng = np.random.default_rng(seed)
    for q, fns in ((19, [(solver3d.collide_bgk3d, O.collide_bgk), (solver3d.collide_mrt3d, O.collide_mrt)]),
                   (27, [(cumulant.collide_cumulant_d3q27, O.collide_cumulant_d3q27),
                         (cumulant.collide_cumulant_geier_d3q27, O.collide_cumulant_geier_d3q27),
                         (d3q27.collide_mrt27, O.collide_mrt)])):
        sp = (8, 10, 12)
        rho = (1 + 0.05 * rng.uniform(-1, 1, sp)).astype(np.float32)
        u = [(0.08 * rng.uniform(-1, 1, sp)).astype(np.float32) for _ in range(3)]
        f = O.equilibrium(q, rho, *u) * (1 + 0.02 * rng.uniform(-1, 1, (q,) + sp)).astype(np.float32)
        f = f.astype(np.float32)
        for ours, ref in fns:
            assert rel_err(N(ours(T(f, cuda), 0.57)), ref(f, 0.57)) < 5 * F32_TOL, ours.__name__


def test_stream_canary_bitwise(cuda):
    from tensorlbm_b200 import d3q27, solver, solver3d

    g = golden("stream")
    assert np.array_equal(N(solver.stream(T(g["f9"], cuda))), g["s9"])
    assert np.array_equal(N(solver3d.stream3d(T(g["f19"], cuda))), g["s19"])
    assert np.array_equal(N(d3q27.stream27(T(g["f27"], cuda))), g["s27"])


def test_stream_full_size_roundtrip(cuda):
    """Size-independent: streaming then streaming the reversed directions is the identity."""
    from tensorlbm_b200 import solver3d
    from tensorlbm_b200.d3q19 import OPPOSITE

    f = torch.rand((19, 64, 96, 128), device=cuda)
    s = solver3d.stream3d(f)
    back = solver3d.stream3d(s[OPPOSITE.to(cuda)])[OPPOSITE.to(cuda)]
    assert torch.equal(back, f)


@pytest.mark.parametrize("q", [9, 19, 27])
def test_boundaries(cuda, q):
    from tensorlbm_b200 import boundaries, boundaries3d, boundaries_d3q27, lid_driven_cavity, obstacles

    g = golden(f"bc_d{'2' if q == 9 else '3'}q{q}")
    f, m = T(g["f"], cuda), T(g["mask"], cuda)
    if q == 9:
        assert np.array_equal(N(boundaries.bounce_back_cells(f, m)), g["bb"])
        assert same(N(boundaries.zou_he_inlet_velocity(f, 0.05, 0.01)), g["inlet"])
        assert same(N(boundaries.zou_he_inlet_velocity(f, T(g["profile"], cuda))), g["inlet_profile"])
        assert same(N(boundaries.zou_he_outlet_pressure(f, 1.02)), g["outlet"])
        assert same(N(lid_driven_cavity.zou_he_moving_lid(f, 0.07)), g["lid"])
        force = torch.stack(boundaries.compute_obstacle_forces(f, m))
        assert np.array_equal(N(f), g["f"])  # functional: input untouched
    elif q == 19:
        assert np.array_equal(N(boundaries3d.bounce_back_cells_3d(f, m)), g["bb"])
        fin = f.clone()
        out = boundaries3d.zou_he_inlet_velocity_3d(fin, 0.04, 0.01, -0.005)
        assert out.data_ptr() == fin.data_ptr()  # in place, like the reference
        assert same(N(out), g["inlet"])
        assert same(N(boundaries3d.zou_he_outlet_pressure_3d(f.clone(), 0.98)), g["outlet"])
        assert same(N(boundaries3d.zou_he_moving_lid_3d(f, 0.05)), g["lid"])
        force = torch.stack(obstacles.compute_obstacle_forces_3d(f, m))
    else:
        assert np.array_equal(N(boundaries_d3q27.bounce_back_cells_27(f, m)), g["bb"])
        assert same(N(boundaries_d3q27.zou_he_inlet_velocity_27(f, 0.04, 0.01, -0.005)), g["inlet"])
        assert same(N(boundaries_d3q27.zou_he_outlet_pressure_27(f, 0.98)), g["outlet"])
        force = torch.stack(obstacles.compute_obstacle_forces_27(f, m))
    ref = g["force"].astype(np.float64)
    assert force.dtype == torch.float64
    assert np.max(np.abs(N(force) - ref)) < 1e-6 * max(np.max(np.abs(ref)), 1.0)


def test_errors(cuda):
    from tensorlbm_b200 import boundaries3d, d3q19, solver3d

    f = torch.rand((19, 4, 5, 6), device=cuda)
    with pytest.raises(ValueError):
        solver3d.collide_bgk3d(torch.rand((18, 4, 5, 6), device=cuda), 0.6)
    with pytest.raises(ValueError):
        d3q19.equilibrium3d(*(torch.ones((4, 5, 6), device=cuda),) * 3, torch.ones((4, 5, 7), device=cuda))
    with pytest.raises(ValueError):
        solver3d.collide_bgk3d(f.half(), 0.6)
    with pytest.raises(NotImplementedError):
        boundaries3d.zou_he_moving_lid_3d(f, 0.05, uy_lid=0.01)
    with pytest.raises(RuntimeError):
        solver3d.collide_bgk3d(f.cpu(), 0.6)


def test_masks_bitwise(cuda):
    from tensorlbm_b200 import boundaries, boundaries3d

    g = golden("masks")
    assert np.array_equal(N(boundaries3d.sphere_mask(32, 16, 16, 12.0, 8.0, 8.0, 4.5, cuda)), g["sphere"])
    assert np.array_equal(N(boundaries3d.sphere_mask(40, 24, 20, 17.3, 11.7, 9.1, 6.35, cuda)), g["sphere_odd"])
    assert np.array_equal(N(boundaries.cylinder_mask(200, 50, 25.0, 25.0, 3.125, cuda)), g["cylinder"])
    assert np.array_equal(N(boundaries.cylinder_mask(97, 31, 20.4, 15.5, 4.7, cuda)), g["cylinder_odd"])
    big = boundaries3d.sphere_mask(512, 256, 256, 128, 128, 128, 16, cuda)
    assert int(big.sum()) == int(g["big_count"])
    assert np.array_equal(N(torch.nonzero(big.reshape(-1))[:, 0]), g["big_index"])


def test_missing_mask_and_links(cuda):
    from tensorlbm_b200 import boundary_registry as br

    g = golden("masks")
    sph = T(g["sphere"], cuda)
    m19 = br.derive_missing_mask((16, 16, 32), solid_mask=sph, periodic={"y": True, "z": True, "x": False},
                                 lattice="D3Q19")
    ref19 = np.unpackbits(g["missing19"])[: int(np.prod(g["missing19_shape"]))].reshape(tuple(g["missing19_shape"]))
    assert np.array_equal(N(m19), ref19.astype(bool))
    links = br.link_list(m19)
    assert np.array_equal(N(links), g["links19"])
    m27 = br.derive_missing_mask((16, 16, 32), solid_mask=sph, periodic=False, lattice="D3Q27")
    ref27 = np.unpackbits(g["missing27"])[: int(np.prod(g["missing27_shape"]))].reshape(tuple(g["missing27_shape"]))
    assert np.array_equal(N(m27), ref27.astype(bool))


def test_link_list_large_and_empty(cuda):
    from tensorlbm_b200 import _ops

    m = torch.rand((19, 40, 50, 60), device=cuda) < 0.01
    assert torch.equal(_ops.link_list(m), torch.nonzero(m.reshape(-1))[:, 0])
    assert _ops.link_list(torch.zeros(1000, dtype=torch.bool, device=cuda)).numel() == 0


@pytest.mark.parametrize("lat", ["D3Q19", "D3Q27"])
def test_links_c2_full_size(cuda, lat):
    """The 512x256x256 sphere channel's solid mask, missing mask and link list,
    built on the GPU, against the list torch.nonzero returned for the
    reference's derive_missing_mask (periodic y/z, closed x): every index, and
    the SHA-256 of the (n, 4) int64 rows."""
    import hashlib

    from tensorlbm_b200 import _ops, boundaries3d
    from tensorlbm_b200 import boundary_registry as br

    g = golden("links_c2")
    tag = lat[2:].lower()
    nz, ny, nx = (int(v) for v in g["shape"])
    solid = boundaries3d.sphere_mask(nx, ny, nz, 128, 128, 128, 16, cuda)
    miss = br.derive_missing_mask((nz, ny, nx), solid_mask=solid, periodic={"y": True, "z": True, "x": False},
                                  lattice=lat)
    assert tuple(miss.shape) == (int(g[f"q_{tag}"]), nz, ny, nx)
    flat = N(_ops.link_list(miss))
    assert flat.size == int(g[f"count_{tag}"])
    assert np.array_equal(flat, np.cumsum(g[f"delta_{tag}"].astype(np.int64)))
    rows = N(br.link_list(miss))
    assert rows.dtype == np.int64 and rows.shape == (flat.size, 4)
    assert hashlib.sha256(np.ascontiguousarray(rows).tobytes()).digest() == g[f"sha256_{tag}"].tobytes()


def test_correct_mass(cuda):
    from tensorlbm_b200 import solver3d

    f = torch.rand((19, 8, 9, 10), device=cuda, dtype=torch.float64)
    out = solver3d.correct_mass3d(f, 123.0)
    assert abs(float(out.sum()) - 123.0) < 1e-9
    assert torch.equal(solver3d.correct_mass3d(torch.zeros_like(f), 5.0), torch.zeros_like(f))


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_correct_mass_golden(cuda, tag):
    """correct_mass / correct_mass3d / correct_mass27 against the reference's
    outputs (solver.py:420, solver3d.py:287, d3q27.py:729).  The reference
    sums in the field dtype, the kernel in float64 and rounds once: the bound
    is the rounding of the sum (1e-6 relative in float32, 1e-14 in float64)."""
    from tensorlbm_b200 import d3q27, solver, solver3d

    g = golden("mass")
    tol = 1e-6 if tag == "f32" else 1e-14
    for q, fn in ((9, solver.correct_mass), (19, solver3d.correct_mass3d), (27, d3q27.correct_mass27)):
        ref = g[f"m{q}_{tag}"]
        got = N(fn(T(g[f"f{q}_{tag}"], cuda), float(g[f"t{q}_{tag}"])))
        assert got.dtype == ref.dtype and rel_err(got, ref) <= tol, (q, rel_err(got, ref))
        assert rel_err(got, O.correct_mass(g[f"f{q}_{tag}"], float(g[f"t{q}_{tag}"]))) <= tol
    assert same(N(solver3d.correct_mass3d(torch.zeros((19, 2, 3, 4), device=cuda), 5.0)), g["zero_out"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_moving_wall_bounce_back(cuda, tag):
    """Ladd moving wall (rotating_cylinder.py:140, propeller_benchmark.py:221),
    bit for bit against the reference on a rotating disc and rotor."""
    from tensorlbm_b200 import propeller_benchmark, rotating_cylinder

    g = golden("moving_wall")
    disc, rotor = T(g["disc"], cuda), T(g["rotor"], cuda)
    f9, f19 = T(g[f"f9_{tag}"], cuda), T(g[f"f19_{tag}"], cuda)
    ux2, uy2 = rotating_cylinder.rotating_wall_velocity(disc, 30.3, 15.6, 0.004)
    assert same(N(ux2), g["ux2"]) and same(N(uy2), g["uy2"])
    out9 = N(rotating_cylinder.moving_wall_bounce_back(f9, disc, ux2, uy2))
    assert same(out9[:, g["disc"]], g[f"mw9_{tag}"])
    assert same(out9[:, ~g["disc"]], g[f"f9_{tag}"][:, ~g["disc"]])
    ux3, uy3, uz3 = propeller_benchmark.rotating_wall_velocity_3d(rotor, 15.0, 5.6, 3.8, 0.006)
    assert same(N(uy3), g["uy3"]) and same(N(uz3), g["uz3"])
    out19 = N(propeller_benchmark.moving_wall_bounce_back_3d(f19, rotor, ux3, uy3, uz3))
    assert same(out19[:, g["rotor"]], g[f"mw19_{tag}"])
    assert same(out19[:, ~g["rotor"]], g[f"f19_{tag}"][:, ~g["rotor"]])
    with pytest.raises(ValueError):
        rotating_cylinder.moving_wall_bounce_back(f9, disc, ux2, uy2[:-1])


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_collide_trt(cuda, tag):
    """The TRT kernels against the reference's outputs, bit for bit."""
    from tensorlbm_b200 import d3q27, solver, solver3d

    g = golden("collide_trt")
    if tag == "f32":
        assert same(N(solver.collide_trt(T(g["f9"], cuda), 0.6)), g["trt9"])
        assert same(N(solver.collide_trt(T(g["f9"], cuda), 0.57, lambda_trt=0.25)), g["trt9_lam"])
    for q, fn in ((19, solver3d.collide_trt3d), (27, d3q27.collide_trt27)):
        f = T(g[f"f{q}_{tag}"], cuda)
        assert same(N(fn(f, 0.6)), g[f"trt{q}_{tag}"])
        assert same(N(fn(f, 0.57, lambda_trt=0.25)), g[f"trt{q}_lam_{tag}"])


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_collide_rlbm(cuda, tag):
    """The regularised-BGK kernels against the reference's outputs, bit for bit."""
    from tensorlbm_b200 import d3q27, solver, solver3d

    g = golden("collide_rlbm")
    for q, fn in ((9, solver.collide_rlbm), (19, solver3d.collide_rlbm3d), (27, d3q27.collide_rlbm27)):
        f, fr = T(g[f"f{q}_{tag}"], cuda), T(g[f"fr{q}_{tag}"], cuda)
        assert same(N(fn(f, 0.6)), g[f"rlbm{q}_{tag}"])
        assert same(N(fn(f, 0.5046)), g[f"rlbm{q}_low_{tag}"])
        assert same(N(fn(fr, 0.53)), g[f"rlbmr{q}_{tag}"])


def test_trt_sphere_channel_vs_oracle(cuda):
    """The fused step with TRT (pull, Zou/He, bounce-back, drag) against the
    oracle's collide -> stream -> boundaries chain: bit-exact."""
    from tensorlbm_b200 import LBMSolver, boundaries3d

    nz, ny, nx = 8, 10, 20
    obst = boundaries3d.sphere_mask(nx, ny, nz, 7.0, 5.0, 4.0, 2.2, cuda)
    o = obst.cpu().numpy()
    ux = np.full((nz, ny, nx), 0.04, np.float32)
    ux[o] = 0.0
    z = np.zeros_like(ux)
    f0 = O.equilibrium(19, np.ones_like(ux), ux, z, z)
    s = LBMSolver("D3Q19", (nz, ny, nx), 0.56, "trt", device=cuda, obstacle_mask=obst, u_in=0.04, rho_out=1.0,
                  track_force=True, lambda_trt=0.2)
    s.load(T(f0, cuda)).step(6)
    ref, forces = f0, []
    for _ in range(6):
        ref, fo = O.channel_step(ref, 0.56, 0.04, 1.0, None, o, "trt", lambda_trt=0.2)
        forces.append(fo)
    assert same(N(s.f), ref)
    assert np.max(np.abs(N(s.force_history()) - np.array(forces))) < 1e-6 * np.max(np.abs(np.array(forces)))


def test_rlbm_cavity_2d_vs_oracle(cuda):
    """The fused D2Q9 step with the regularised BGK in the verified Re 1000
    cavity's scheme (three half-way walls from the pre-collision state, Zou/He
    lid) against the oracle's collide -> where -> stream -> lid chain at a
    low-viscosity tau: bit-exact."""
    from tensorlbm_b200 import LBMSolver

    n, tau, u_lid = 48, 0.5144, 0.06
    wall = np.zeros((n, n), bool)
    wall[0, :] = wall[:, 0] = wall[:, -1] = True
    z = np.zeros((n, n), np.float32)
    f0 = O.equilibrium(9, np.ones_like(z), z, z)
    s = LBMSolver("D2Q9", (n, n), tau, "rlbm", device=cuda, wall_mask=T(wall, cuda), wall_mode="halfway",
                  u_lid=u_lid)
    s.load(T(f0, cuda)).step(40)
    ref = f0
    for _ in range(40):
        ref = O.cavity_step(ref, tau, wall, u_lid, "rlbm", mode="halfway")
    assert same(N(s.f), ref)


@pytest.mark.parametrize("q", [19, 27])
def test_rlbm_sphere_channel_vs_oracle(cuda, q):
    """The fused 3-D step with the regularised BGK (pull, Zou/He, bounce-back,
    drag) against the oracle's chain: bit-exact populations."""
    from tensorlbm_b200 import LBMSolver, boundaries3d

    nz, ny, nx = 8, 10, 20
    obst = boundaries3d.sphere_mask(nx, ny, nz, 7.0, 5.0, 4.0, 2.2, cuda)
    o = obst.cpu().numpy()
    ux = np.full((nz, ny, nx), 0.04, np.float32)
    ux[o] = 0.0
    z = np.zeros_like(ux)
    f0 = O.equilibrium(q, np.ones_like(ux), ux, z, z)
    s = LBMSolver(f"D3Q{q}", (nz, ny, nx), 0.53, "rlbm", device=cuda, obstacle_mask=obst, u_in=0.04, rho_out=1.0,
                  track_force=True)
    s.load(T(f0, cuda)).step(6)
    ref = f0
    for _ in range(6):
        ref, _ = O.channel_step(ref, 0.53, 0.04, 1.0, None, o, "rlbm")
    assert same(N(s.f), ref)


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_far_field_dropins(cuda, tag):
    """far_field_bc_2d / _3d / _27 against the reference's outputs, bit for bit."""
    from tensorlbm_b200 import boundaries, boundaries3d, boundaries_d3q27

    g = golden("far_field")
    ob9, ob3 = T(g["ob9"], cuda), T(g["ob3"], cuda)
    assert same(N(boundaries.far_field_bc_2d(T(g[f"f9_{tag}"], cuda), 0.07, ob9)), g[f"ff9_{tag}"])
    f19 = T(g[f"f19_{tag}"], cuda)
    assert same(N(boundaries3d.far_field_bc_3d(f19, 0.06, ob3)), g[f"ff19_{tag}"])
    cfg_y = {"far_field_faces": ["y-", "y+"], "periodic_faces": ["z-", "z+"]}
    assert same(N(boundaries3d.far_field_bc_3d(f19, 0.06, None, bc_config=cfg_y)), g[f"ff19y_{tag}"])
    assert same(N(boundaries3d.far_field_bc_3d(f19, 0.06, None, uy=0.01, uz=-0.02)), g[f"ff19uv_{tag}"])
    assert same(N(boundaries_d3q27.far_field_bc_27(T(g[f"f27_{tag}"], cuda), 0.05, ob3)), g[f"ff27_{tag}"])


@pytest.mark.parametrize("q,shape,faces", [(9, (12, 32), "y"), (9, (12, 33), "y"), (19, (6, 8, 16), "yz"),
                                           (19, (6, 8, 15), "yz"), (19, (6, 8, 16), "y"), (27, (6, 8, 16), "yz")])
def test_far_field_step_vs_oracle(cuda, q, shape, faces):
    """The fused step with the far field (BGK, obstacle with drag, a seeded
    inlet perturbation for part of the run) against the oracle's collide ->
    stream -> force -> far field -> bounce-back chain: bit-exact populations
    on the far-field pair kernel (even nx) and the one-cell kernel (odd nx)."""
    from tensorlbm_b200 import LBMSolver

    obst = np.zeros(shape, bool)
    if q == 9:
        obst[4:7, 10:13] = True
    else:
        obst[2:4, 3:5, 6:9] = True
    rng = np.random.default_rng(q + shape[-1])
    u = 0.05
    z = np.zeros(shape, np.float32)
    ux = (u + 0.01 * rng.standard_normal(shape)).astype(np.float32)
    ux[obst] = 0.0
    uy = (0.01 * rng.standard_normal(shape)).astype(np.float32)
    f0 = O.equilibrium(q, np.ones_like(z), ux, uy, None if q == 9 else z)
    lat = {9: "D2Q9", 19: "D3Q19", 27: "D3Q27"}[q]
    s = LBMSolver(lat, shape, 0.58, "bgk", device=cuda, obstacle_mask=T(obst, cuda), u_in=u, far_field=faces,
                  track_force=True)
    s.load(T(f0, cuda))
    ref, forces = f0, []
    for k in range(8):
        du = (0.0, 0.004 * np.sin(0.7 * k), 0.0) if k < 5 else (0.0, 0.0, 0.0)
        s.set_inlet_perturbation(*du).step(1)
        ref, fo = O.far_field_step(ref, 0.58, u, obst, "bgk", z_faces=faces == "yz", inlet_du=du)
        forces.append(fo)
    assert same(N(s.f), ref)
    fh, fr = N(s.force_history()), np.array(forces)
    k = min(fh.shape[1], fr.shape[1])
    assert np.max(np.abs(fh[:, :k] - fr[:, :k])) <= 1e-6 * np.max(np.abs(fr))


def test_far_field_mrt_sponge_vs_oracle(cuda):
    """D2Q9 MRT with a sponge tau field and the far field (the verified
    cylinder's step) against the oracle chain, to the MRT's float32 rounding."""
    from tensorlbm_b200 import LBMSolver, boundaries

    ny, nx, u = 24, 64, 0.05
    obst = np.zeros((ny, nx), bool)
    yy, xx = np.mgrid[0:ny, 0:nx]
    obst[(xx - 16) ** 2 + (yy - 12) ** 2 <= 9] = True
    sigma = N(boundaries.make_sponge_strength(ny, nx, 44, 20, device=cuda))
    tau_field = (0.56 * (1.0 + 10.0 * sigma)).astype(np.float32)
    z = np.zeros((ny, nx), np.float32)
    f0 = O.equilibrium(9, np.ones_like(z), np.where(obst, 0.0, u).astype(np.float32), z)
    s = LBMSolver("D2Q9", (ny, nx), 0.56, "mrt", device=cuda, obstacle_mask=T(obst, cuda), u_in=u, far_field="y",
                  tau_field=T(tau_field, cuda))
    s.load(T(f0, cuda)).step(20)
    ref = f0
    for _ in range(20):
        ref, _ = O.far_field_step(ref, 0.56, u, obst, "mrt", z_faces=False, tau_field=tau_field)
    assert np.max(np.abs(N(s.f) - ref)) <= 2e-6


def test_far_field_d3q27_cumulant_vs_oracle(cuda):
    """The D3Q27 legacy cumulant with the far field on all four lateral planes
    and a drag body (the SUBOFF runners' far_field_bc_27 chain) against the
    oracle, to the cumulant's float32 rounding."""
    from tensorlbm_b200 import LBMSolver

    shape = (8, 10, 24)
    obst = np.zeros(shape, bool)
    obst[3:5, 4:6, 8:11] = True
    z = np.zeros(shape, np.float32)
    ux = np.where(obst, 0.0, 0.05).astype(np.float32)
    f0 = O.equilibrium(27, np.ones_like(z), ux, z, z)
    s = LBMSolver("D3Q27", shape, 0.56, "cumulant", device=cuda, obstacle_mask=T(obst, cuda), u_in=0.05,
                  far_field="yz", track_force=True)
    s.load(T(f0, cuda)).step(10)
    ref = f0
    for _ in range(10):
        ref, _ = O.far_field_step(ref, 0.56, 0.05, obst, "cumulant", z_faces=True)
    assert np.max(np.abs(N(s.f) - ref)) <= 1e-5 * np.max(np.abs(ref))


def test_far_field_rejections(cuda):
    from tensorlbm_b200 import LBMSolver

    with pytest.raises(ValueError):
        LBMSolver("D2Q9", (8, 16), 0.6, "bgk", device=cuda, u_in=0.05, far_field="yz")
    with pytest.raises(ValueError):
        LBMSolver("D3Q19", (4, 8, 16), 0.6, "bgk", device=cuda, u_in=0.05, rho_out=1.0, far_field="y")
    with pytest.raises(NotImplementedError):
        LBMSolver("D3Q19", (4, 8, 16), 0.6, "bgk", device=cuda, u_in=0.05, far_field="y", pattern="aa")


@pytest.mark.parametrize("tag,tol", [("f32", 5 * F32_TOL), ("f64", 1e-12)])
def test_collide_cascaded(cuda, tag, tol):
    """The cascaded kernels against the reference's outputs (fused moment
    transforms: float32 rounding, not bit for bit)."""
    from tensorlbm_b200 import cascaded_collision as cc

    g = golden("collide_cascaded")
    for q, fn, kw in ((19, cc.collide_cascaded_d3q19, dict(s_bulk=1.2, s_3=0.9, s_4=1.3)),
                      (27, cc.collide_cascaded_d3q27, dict(s_bulk=1.2, s_3=0.9, s_4=1.3, s_5=1.1, s_6=0.8))):
        f = T(g[f"f{q}_{tag}"], cuda)
        assert rel_err(N(fn(f, 0.6)), g[f"c{q}_{tag}"]) < tol
        assert rel_err(N(fn(f, 0.57, **kw)), g[f"c{q}r_{tag}"]) < tol
    with pytest.raises(ValueError):
        cc.collide_cascaded_d3q19(T(g["f19_f32"], cuda), 0.5)


@pytest.mark.parametrize("q", [19, 27])
def test_cascaded_sphere_channel_vs_oracle(cuda, q):
    """The fused step with the cascaded collision against the oracle's chain."""
    from tensorlbm_b200 import LBMSolver, boundaries3d

    nz, ny, nx = 8, 10, 20
    obst = boundaries3d.sphere_mask(nx, ny, nz, 7.0, 5.0, 4.0, 2.2, cuda)
    o = obst.cpu().numpy()
    ux = np.full((nz, ny, nx), 0.04, np.float32)
    ux[o] = 0.0
    z = np.zeros_like(ux)
    f0 = O.equilibrium(q, np.ones_like(ux), ux, z, z)
    s = LBMSolver(q, (nz, ny, nx), 0.56, "cascaded", device=cuda, obstacle_mask=obst, u_in=0.04, rho_out=1.0,
                  omega_b=1.1, omega_odd=0.95)
    s.load(T(f0, cuda)).step(6)
    ref = f0
    for _ in range(6):
        ref, _ = O.channel_step(ref, 0.56, 0.04, 1.0, None, o, "cascaded", s_bulk=1.1, s_3=0.95)
    assert rel_err(N(s.f), ref) < 1e-5
