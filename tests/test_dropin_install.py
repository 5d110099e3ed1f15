"""install() against the unmodified TensorLBM package (baseline/_ref), on the
CPU: which bindings it replaces and that uninstall() restores them.  No kernel
runs here; tests/test_gpu_dropin_reference.py runs TensorLBM's own runners on
the kernels."""

from __future__ import annotations

import pytest

from baseline import reference

pytestmark = pytest.mark.skipif(not reference.available(), reason="TensorLBM is not installed in baseline/_ref")


def test_install_rebinds_names_bound_at_import_and_uninstall_restores():
    import tensorlbm_b200 as tb

    tl = reference.import_reference()
    import tensorlbm.d3q27 as d27
    import tensorlbm.d3q27_sphere_flow as runner27
    import tensorlbm.solver3d as s3
    import tensorlbm.sphere_flow as runner19

    originals = (d27.collide_bgk27, runner27.collide_bgk27, runner19.collide_bgk3d, runner19.correct_mass3d,
                 runner27.compute_obstacle_forces_27)
    assert runner27.collide_bgk27 is d27.collide_bgk27          # bound at import time
    try:
        patched = tb.install(tl)
        assert "d3q27.collide_bgk27" in patched and "solver3d.collide_bgk3d" in patched
        from tensorlbm_b200 import d3q27 as our27
        from tensorlbm_b200 import obstacles as our_obst
        from tensorlbm_b200 import solver3d as our3

        # the defining modules and the runners' import-time bindings
        assert d27.collide_bgk27 is our27.collide_bgk27
        assert runner27.collide_bgk27 is our27.collide_bgk27
        assert runner27.stream27 is our27.stream27
        assert runner27.compute_obstacle_forces_27 is our_obst.compute_obstacle_forces_27
        assert runner19.collide_bgk3d is our3.collide_bgk3d
        assert runner19.correct_mass3d is our3.correct_mass3d
        assert s3.stream3d is our3.stream3d
        # a module (re-)imported after install() takes the kernels from the patched modules
        import importlib

        late = importlib.reload(runner19)
        assert late.stream3d is our3.stream3d and late.collide_bgk3d is our3.collide_bgk3d
        # names that are not replaced stay the reference's own
        assert runner27.make_channel_wall_mask_27.__module__ == "tensorlbm.boundaries_d3q27"
    finally:
        restored = tb.uninstall()
    assert restored > 0
    assert (d27.collide_bgk27, runner27.collide_bgk27, runner19.collide_bgk3d, runner19.correct_mass3d,
            runner27.compute_obstacle_forces_27) == originals
    assert tb.uninstall() == 0
