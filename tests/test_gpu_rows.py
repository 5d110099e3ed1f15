"""Row-staged step kernel (whole x-rows copied into shared memory by bulk
asynchronous copies) against the two-cells-per-thread kernel: the same
stored state bit for bit after many steps, the same drag to float64
summation order, across lattices, storages, boundaries and row lengths."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import lbm as O

pytestmark = pytest.mark.gpu


def T(a, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _run(cuda, q, coll, storage, shape, steps, rows, extra):
    from tensorlbm_b200 import LBMSolver, _lib

    prev = _lib.set_row_staging(rows)
    try:
        rng = np.random.default_rng(7)
        obst = np.zeros(shape, bool)
        nz, ny, nx = shape
        obst[:, ny // 2 - 1:ny // 2 + 2, nx // 3:nx // 3 + 3] = True
        kw = dict(obstacle_mask=T(obst, cuda), track_force=True)
        if extra.get("zou_he", True):
            kw.update(u_in=0.04, rho_out=1.0)
        if extra.get("halfway"):
            wall = np.zeros(shape, bool)
            wall[:, 0, :] = True
            kw.update(wall_mask=T(wall, cuda), wall_mode="halfway")
        if extra.get("tau_field"):
            kw["tau_field"] = T((0.55 + 0.2 * rng.random(shape)).astype(np.float32), cuda)
        ux = (0.04 + 0.01 * rng.standard_normal(shape)).astype(np.float32)
        ux[obst] = 0
        us = [ux] + [(0.01 * rng.standard_normal(shape)).astype(np.float32) for _ in range(2)]
        f0 = O.equilibrium(q, np.ones(shape, np.float32), *us)
        s = LBMSolver(q, shape, 0.6, coll, device=cuda, storage=storage, **kw).load(T(f0, cuda)).step(steps)
        return s.state.clone(), s.force_history().clone(), s.nonfinite_seen()
    finally:
        _lib.set_row_staging(prev)


CASES = [
    (19, "bgk", "f32", (6, 10, 128), {}),
    (19, "bgk", "f16", (6, 10, 128), {"halfway": True}),
    (19, "bgk", "bf16", (4, 8, 64), {}),
    (19, "mrt", "f32", (5, 12, 256), {"tau_field": True}),
    (19, "mrt", "f16", (6, 10, 128), {"halfway": True}),
    (19, "mrt", "bf16", (3, 6, 512), {}),
    (27, "cumulant", "f32", (6, 10, 128), {}),
    (27, "cumulant", "f16", (4, 9, 192), {"halfway": True}),
    (19, "bgk", "f16", (1, 3, 64), {"zou_he": False}),   # fewer rows than CTAs
]


@pytest.mark.parametrize("q,coll,storage,shape,extra", CASES)
def test_rows_kernel_equals_pair_kernel(cuda, q, coll, storage, shape, extra):
    a, fa, bad_a = _run(cuda, q, coll, storage, shape, 25, True, extra)
    b, fb, bad_b = _run(cuda, q, coll, storage, shape, 25, False, extra)
    assert not bad_a and not bad_b
    assert a.dtype == b.dtype and a.shape == b.shape
    assert bool((a.view(-1).view(dtype=_int_view(a)) == b.view(-1).view(dtype=_int_view(b))).all())
    # the drag: the same per-warp partial sums, added in another order
    scale = float(fb.abs().max())
    assert float((fa - fb).abs().max()) <= 1e-12 * max(scale, 1e-300)


def _int_view(t):
    import torch

    return {2: torch.int16, 4: torch.int32, 8: torch.int64}[t.element_size()]


def test_rows_switch_reports_previous_setting(cuda):
    from tensorlbm_b200 import _lib

    prev = _lib.set_row_staging(False)
    try:
        assert _lib.set_row_staging(True) is False
        assert _lib.set_row_staging(True) is True
    finally:
        _lib.set_row_staging(prev)
