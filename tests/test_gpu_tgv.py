"""Shifted half-precision storage on the decaying Taylor-Green vortex (D3Q27
cumulant), small grid: every storage format against the FP64 run."""

from __future__ import annotations

import math

import pytest

pytestmark = pytest.mark.gpu


def test_tgv_precision_small(cuda):
    from tensorlbm_b200 import tgv

    res = tgv.run(n=32, re=200.0, t_end=1.0, checkpoints=(0.5, 1.0), samples_per_tc=4, device=cuda,
                  log=lambda *_: None)
    runs = res["runs"]
    for st in ("f64", "f32", "f16", "bf16"):
        assert runs[st]["finite"], st
    # FP32 storage tracks FP64 to float32 rounding; the shifted halves to their mantissa
    assert runs["f32"]["velocity_l2_vs_f64"]["1.0"] < 1e-5
    assert runs["f16"]["velocity_l2_vs_f64"]["1.0"] < 5e-3
    assert runs["bf16"]["velocity_l2_vs_f64"]["1.0"] < 5e-2
    assert abs(runs["f64"]["mass_drift_end"]) < 1e-12
    assert abs(runs["f32"]["mass_drift_end"]) < 1e-5
    # kinetic energy decays
    k = runs["f64"]["history"]["kinetic_energy"]
    assert k[-1] < k[0] and all(math.isfinite(v) for v in k)


@pytest.mark.parametrize("n", [64, 96])
def test_laminar_decay_matches_reference_benchmark(cuda, n):
    """TensorLBM's verified laminar Taylor-Green decay (D3Q19 BGK, Re 24,
    float32, 2000 steps) on the fused kernel against the energy history and the
    fitted decay rate that the reference benchmark recorded (golden
    tgv_laminar, from benchmarks/verified/taylor_green_3d).  The reference ran
    torch's CUDA operators, so agreement is to float32 rounding, not bitwise."""
    import numpy as np

    from tensorlbm_b200 import tgv

    from tests.conftest import golden

    g = golden("tgv_laminar")
    res = tgv.laminar_decay(n, re=float(g[f"n{n}_re"]), u0=float(g[f"n{n}_u0"]), steps=int(g[f"n{n}_steps"]),
                            record_every=int(g[f"n{n}_record_every"]), device=cuda)
    assert res["tau"] == pytest.approx(float(g[f"n{n}_tau"]), rel=1e-12)
    assert np.array_equal(np.asarray(res["times"]), g[f"n{n}_record_steps"])
    # below about 1e-4 E0 the float32 rounding of u (~1e-8) dominates E, and
    # CPU-exact and CUDA torch arithmetic part ways: compare the clean window
    e_ref = g[f"n{n}_energy"]
    clean = e_ref >= 1e-4 * e_ref[0]
    np.testing.assert_allclose(np.asarray(res["energies"])[clean], e_ref[clean], rtol=1e-5)
    t = np.asarray(res["times"], dtype=np.float64)
    sel = clean & (t > 0)

    def rate(e):
        return -np.polyfit(t[sel], np.log(np.asarray(e, dtype=np.float64)[sel]), 1)[0]

    assert rate(res["energies"]) == pytest.approx(rate(e_ref), rel=1e-5)
    # the fit over every recorded step, as the benchmark reports it
    assert res["gamma_e_sim"] == pytest.approx(float(g[f"n{n}_gamma_e_sim"]), rel=2e-4)
    assert res["r2"] > 0.99999
