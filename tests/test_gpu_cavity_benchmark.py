"""TensorLBM's verified benchmarks (benchmarks/verified/*) run on the fused
kernel, against the values each benchmark recorded in the reference's own
result files: the 3-D lid-driven cavity at Re 1000 (golden cavity3d_full),
the 2-D cavity at Re 100 (cavity2d_re100) and Re 1000 (cavity2d_re1000, the
regularised BGK), the free-stream cylinder at Re 100 (cylinder2d_small,
cylinder2d_re100), the Hagen-Poiseuille pipe (pipe3d), the shear wave and the
2-D Taylor-Green vortex (tgv2d)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [64, 96])
def test_cavity_3d_full_matches_reference_benchmark(cuda, n):
    """D3Q19 TRT, five half-way walls, Zou/He lid, 100 000 steps: the
    centre-plane centre lines, u_min and the mass drift."""
    from tensorlbm_b200.lid_driven_cavity import cavity_3d_full

    from tests.conftest import golden

    g = golden("cavity3d_full")
    r = cavity_3d_full(n, re=float(g[f"n{n}_re"]), u_lid=float(g[f"n{n}_u_lid"]), steps=int(g[f"n{n}_n_steps_run"]),
                       device=cuda)
    assert r["finite"]
    assert r["tau"] == pytest.approx(float(g[f"n{n}_tau"]), rel=1e-12)
    # the steady centre lines (u / u_lid; the reference stored 6 decimals, and
    # its run used torch's CUDA operators): measured within 8e-6
    assert np.max(np.abs(np.asarray(r["u_centerline_mid"]) - g[f"n{n}_u_centerline_mid"])) <= 5e-5
    assert np.max(np.abs(np.asarray(r["v_centerline_mid"]) - g[f"n{n}_v_centerline_mid"])) <= 5e-5
    assert r["u_min_3d_mid"] == pytest.approx(float(g[f"n{n}_u_min_3d_mid"]), abs=5e-5)
    # the Zou/He lid does not conserve mass; the drift it accumulates over the
    # run agrees to rounding (measured 0.14 % at 64^3, 0.7 % at 96^3)
    assert r["mass_drift"] == pytest.approx(float(g[f"n{n}_mass_drift"]), rel=2e-2)


@pytest.mark.parametrize("n", [128, 192])
def test_cavity_2d_re100_matches_reference_benchmark(cuda, n):
    """TensorLBM's verified 2-D cavity at Re 100 (D2Q9 MRT, three half-way
    walls, Zou/He lid, 100 000 steps) against the point values the reference
    benchmark recorded (golden cavity2d_re100).  The MRT agrees with the
    reference's BLAS products to float32 rounding, not bitwise, and a float32
    steady state is fixed only to that noise: measured within 6e-5 of u_lid."""
    from tensorlbm_b200.lid_driven_cavity import cavity_2d

    from tests.conftest import golden

    g = golden("cavity2d_re100")
    r = cavity_2d(n, re=float(g[f"n{n}_re"]), u_lid=float(g[f"n{n}_u_lid"]), steps=int(g[f"n{n}_steps"]), device=cuda)
    assert r["finite"]
    assert r["tau"] == pytest.approx(float(g[f"n{n}_tau"]), abs=1e-12)
    for key in ("u_mid", "u_bot", "v_mid"):
        assert r[key] == pytest.approx(float(g[f"n{n}_{key}"]), abs=2e-4), key


@pytest.mark.parametrize("n", [192, 256])
def test_cavity_2d_re1000_rlbm_matches_reference_benchmark(cuda, n):
    """TensorLBM's verified 2-D cavity at Re 1000 (D2Q9 regularised BGK at
    tau 0.535 / 0.546, three half-way walls, Zou/He lid, 200 000 steps)
    against the point values and the primary vortex centre the reference
    benchmark recorded (golden cavity2d_re1000).  The collision is bit-exact
    against the reference's CPU operators; its recorded run used torch's CUDA
    operators, whose sums round differently.  Measured: within 1e-5 of u_lid,
    vortex centre identical."""
    from tensorlbm_b200.lid_driven_cavity import cavity_2d

    from tests.conftest import golden

    g = golden("cavity2d_re1000")
    r = cavity_2d(n, re=float(g[f"n{n}_re"]), u_lid=float(g[f"n{n}_u_lid"]), steps=int(g[f"n{n}_steps"]),
                  device=cuda, chunk=1000, collision="rlbm")
    assert r["finite"]
    assert r["tau"] == pytest.approx(float(g[f"n{n}_tau"]), abs=1e-12)
    for key in ("u_mid", "u_bot", "v_mid"):
        assert r[key] == pytest.approx(float(g[f"n{n}_{key}"]), abs=5e-5), key
    assert r["primary_vortex"] == pytest.approx(g[f"n{n}_primary_vortex"].tolist(), abs=2.0 / (n - 1))


def test_cylinder_2d_small_matches_reference_run(cuda):
    """The verified cylinder's chain (D2Q9 MRT with the sponge tau field, far
    field, seeded wake, drag every step) against the benchmark's own run.py
    run eagerly on the CPU at D = 8 for 3000 steps (golden cylinder2d_small):
    the per-step drag and lift coefficients over the whole run, and Cd and St
    of the analysis window (the reference's own series through the
    benchmark's formulas, unrounded), agree to the MRT's float32 rounding
    (its BLAS products against the fused collision): measured 5.7e-4 per step
    in C_d (0.04 %; the series carries step-to-step grid noise of that size),
    4.4e-5 relative in Cd and 6e-5 in St."""
    from tensorlbm_b200.verified import cylinder_2d, lift_strouhal

    from tests.conftest import golden

    g = golden("cylinder2d_small")
    steps = int(g["steps"])
    r = cylinder_2d(8, steps=steps, device=cuda, return_series=True)
    assert r["finite"] and r["seed_steps"] == int(g["seed_steps"])
    w0 = steps // 2
    assert np.max(np.abs(r["cd_series"][w0:] - g["cd_series"][w0:])) <= 1.5e-3
    assert np.max(np.abs(r["cl_series"][w0:] - g["cl_series"][w0:])) <= 1.5e-3
    assert np.max(np.abs(r["cd_series"] - g["cd_series"])) <= 1e-5 * np.max(np.abs(g["cd_series"]))
    assert r["cd"] == pytest.approx(float(g["cd_series"][w0:].mean()), rel=2e-4)
    assert float(g["cd"]) == pytest.approx(float(g["cd_series"][w0:].mean()), abs=5e-5)  # its rounded report
    assert r["st"] == pytest.approx(lift_strouhal(g["cl_series"][w0:], 8, 0.05), rel=2e-4)


@pytest.mark.parametrize("d", [48, 64])
def test_cylinder_2d_re100_benchmark_criteria(cuda, d):
    """The verified cylinder at D = 48 / 64 (60 000 / 90 000 steps) meets the
    benchmark's own acceptance test: Cd within 3 % of Braza's 1.35 and St
    within 3 % of 0.1645 (run.py:58-59; README).  The values recorded in its
    result.json (golden cylinder2d_re100) came from an earlier script
    (README: /tmp/b5_sponge.py), not from the committed run.py whose chain
    this runner follows; they are reported beside ours, not asserted."""
    from tensorlbm_b200.verified import cylinder_2d

    from tests.conftest import golden

    g = golden("cylinder2d_re100")
    r = cylinder_2d(d, steps=int(g[f"d{d}_steps"]), device=cuda)
    assert r["finite"]
    assert abs(r["cd"] / 1.35 - 1.0) <= 0.03
    assert abs(r["st"] / 0.1645 - 1.0) <= 0.03


@pytest.mark.parametrize("r", [20, 40])
def test_pipe_3d_matches_reference_benchmark(cuda, r):
    """TensorLBM's verified Hagen-Poiseuille pipe (D3Q19 BGK, Zou/He velocity
    inlet and pressure outlet, full-way swap at the staircase wall, 20 000 /
    23 600 steps plus a 400-step average) against the profile, centre velocity,
    flow rate, inlet density and mass drift the reference benchmark recorded
    (golden pipe3d).  Measured: profile within 1.8e-5 relative, inlet density
    within 4e-7."""
    from tensorlbm_b200.verified import pipe_3d

    from tests.conftest import golden

    g = golden("pipe3d")
    res = pipe_3d(r, tau=float(g[f"r{r}_tau"]), u_in=float(g[f"r{r}_u_in"]), steps=int(g[f"r{r}_n_steps"]),
                  L_over_R=int(g[f"r{r}_L_over_R"]), device=cuda)
    assert res["finite"]
    prof, ref = np.asarray(res["u_profile"]), g[f"r{r}_u_profile"]
    assert prof.shape == ref.shape
    assert np.max(np.abs(prof - ref) / np.abs(ref)) <= 1e-4
    assert res["u_center"] == pytest.approx(float(g[f"r{r}_u_center"]), rel=1e-4)
    assert res["Q"] == pytest.approx(float(g[f"r{r}_Q"]), rel=1e-4)
    assert res["rho_in_measured"] == pytest.approx(float(g[f"r{r}_rho_in_measured"]), abs=1e-5)
    assert res["mass_drift_pct"] == pytest.approx(float(g[f"r{r}_mass_drift_pct"]), rel=2e-2)


def test_taylor_green_2d_matches_reference_benchmark(cuda):
    """TensorLBM's verified decaying 2-D Taylor-Green vortex (N = 128, Re 100,
    D2Q9 BGK float32, 4900 steps) against the histories and fits the
    benchmark recorded (golden tgv2d, its CPU run): the step is bit-exact, so
    the energies agree to the order of the GPU's mean (measured 1.4e-7), max|u|
    exactly, the decay rates to 1e-8 and the mass drift to 1e-10."""
    from tensorlbm_b200.verified import taylor_green_2d

    from tests.conftest import golden

    g = golden("tgv2d")
    r = taylor_green_2d(int(g["n"]), float(g["re"]), float(g["u0"]), int(g["steps"]), int(g["record_every"]),
                        device=cuda)
    assert r["finite"]
    assert np.array_equal(np.asarray(r["times"]), g["steps_recorded"])
    np.testing.assert_allclose(r["energies"], g["energy"], rtol=1e-6)
    np.testing.assert_allclose(r["umaxs"], g["umax"], rtol=1e-7)
    assert r["gamma_e_sim"] == pytest.approx(float(g["gamma_e_sim"]), rel=1e-6)
    assert r["gamma_vel_sim"] == pytest.approx(float(g["gamma_vel_sim"]), rel=1e-6)
    assert r["mass_drift_rel"] == pytest.approx(float(g["mass_drift_rel"]), abs=1e-9)


@pytest.mark.parametrize("h", [64, 128])
def test_shear_wave_matches_reference_benchmark(cuda, h):
    """TensorLBM's verified decaying shear wave (D2Q9 BGK float32, periodic,
    tau 0.8) against TensorLBM's own eager run of the benchmark (golden
    shear_wave; it reproduces the histories the benchmark recorded exactly):
    the energy and max|u| histories to the order of the GPU's mean/max
    reductions, and the fitted decay rates."""
    from tensorlbm_b200.verified import shear_wave

    from tests.conftest import golden

    g = golden("shear_wave")
    r = shear_wave(h, tau=float(g[f"h{h}_tau"]), u0=float(g[f"h{h}_u0"]), steps=int(g[f"h{h}_steps"]),
                   record_every=int(g[f"h{h}_record_every"]), device=cuda)
    assert r["finite"]
    assert np.array_equal(np.asarray(r["times"]), g[f"h{h}_record_steps"])
    np.testing.assert_array_equal(g[f"h{h}_energy"], g[f"h{h}_energy_compiled"])
    np.testing.assert_allclose(r["energies"], g[f"h{h}_energy"], rtol=1e-6)
    np.testing.assert_allclose(r["umaxs"], g[f"h{h}_umax"], rtol=1e-6)
    assert r["gamma_e_sim"] == pytest.approx(float(g[f"h{h}_gamma_e_sim"]), rel=1e-6)
    assert r["gamma_vel_sim"] == pytest.approx(float(g[f"h{h}_gamma_vel_sim"]), rel=1e-6)
