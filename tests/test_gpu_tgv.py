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
