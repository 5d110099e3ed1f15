"""tensorlbm_b200 - the TensorLBM lattice-Boltzmann time step on NVIDIA B200 (sm_100a).

Drop-in replacements for TensorLBM's lattice operators and step drivers, each
running hand-written CUDA kernels from ``libtlbm.so`` through its C ABI
(``include/tlbm.h``) on the caller's torch tensors.  Module names follow
TensorLBM (``d3q19``, ``solver3d``, ``boundaries3d``, ...); :func:`install`
patches them into an imported ``tensorlbm`` package.

Inputs must be CUDA tensors; there is no CPU path.
"""

from __future__ import annotations

from . import _lib, lattice  # noqa: F401
from .solvers import FusedSolver3D, LBMSolver, StepConfig, make_step  # noqa: F401

__version__ = "0.1.0"

# (tensorlbm module, attribute) -> (our module, attribute)
_PATCHES = {
    "d2q9": ["equilibrium", "macroscopic"],
    "d3q19": ["equilibrium3d", "macroscopic3d", "equilibrium3d_low_memory", "macroscopic3d_low_memory"],
    "d3q27": ["equilibrium27", "macroscopic27", "collide_bgk27", "collide_mrt27", "collide_trt27", "collide_rlbm27", "stream27",
              "stream27_roll", "correct_mass27"],
    "solver": ["collide_bgk", "collide_bgk_fused", "collide_mrt", "collide_trt", "collide_rlbm", "stream", "correct_mass"],
    "solver3d": ["collide_bgk3d", "collide_mrt3d", "collide_trt3d", "collide_rlbm3d", "collide_mrt3d_low_memory", "stream3d",
                 "stream3d_roll",
                 "correct_mass3d"],
    "cumulant": ["collide_cumulant_d3q27", "collide_cumulant_geier_d3q27", "collide_cumulant_d3q19"],
    "turbulence": ["collide_smagorinsky_bgk", "collide_smagorinsky_bgk3d", "collide_smagorinsky_bgk27"],
    "boundaries": ["cylinder_mask", "bounce_back_cells", "zou_he_inlet_velocity", "zou_he_outlet_pressure",
                   "compute_obstacle_forces", "far_field_bc_2d", "make_sponge_strength"],
    "boundaries3d": ["sphere_mask", "bounce_back_cells_3d", "zou_he_inlet_velocity_3d",
                     "zou_he_outlet_pressure_3d", "zou_he_moving_lid_3d", "far_field_bc_3d"],
    "boundaries_d3q27": ["bounce_back_cells_27", "zou_he_inlet_velocity_27", "zou_he_outlet_pressure_27",
                         "far_field_bc_27"],
    "lid_driven_cavity": ["zou_he_moving_lid"],
    "obstacles": ["compute_obstacle_forces_3d", "compute_obstacle_forces_27"],
    "boundary_registry": ["derive_missing_mask"],
    "rotating_cylinder": ["moving_wall_bounce_back"],
    "propeller_benchmark": ["moving_wall_bounce_back_3d"],
    "bfl_common": ["compute_q_sphere_common", "bfl_bounce_back_common"],
    "interpolated_bc_common": ["compute_q_sphere_27"],
    "bfl_d3q19": ["bouzidi_bounce_back_d3q19"],
    "triton_fused": ["triton_fused", "triton_collide", "triton_stream", "TritonFusedSolver3D", "is_available"],
    "cascaded_collision": ["collide_cascaded_d3q19", "collide_cascaded_d3q27"],
    "triton_fused_distributed": ["DistributedTritonFusedSolver3D", "crossing_face_indices", "init_distributed",
                                 "rank", "world_size", "distributed_is_available"],
    "momentum_exchange": ["momentum_exchange_standard", "momentum_exchange_galilean",
                          "momentum_exchange_background_subtracted", "momentum_exchange_bfl"],
}


# (module name, attribute) -> the object install() replaced there
_ORIGINALS: dict = {}


def install(package=None) -> list[str]:
    """Replace TensorLBM's hot-path functions with these kernels in a live import.

    ``package`` defaults to ``import tensorlbm``.  Each name of ``_PATCHES`` is
    replaced in its defining module.  Then every loaded module of the package
    is searched for globals that *are* one of the replaced objects (an identity
    check) and those are rebound too: runners that bound a name at import time
    (``from .d3q27 import collide_bgk27`` in ``d3q27_sphere_flow.py``, or
    ``from .solver3d import collide_bgk3d`` in ``sphere_flow.py``) then call the
    kernels as well.  Modules imported later pick the new names up from the
    patched defining modules.  Returns the patched ``module.name`` entries.
    Every replaced function requires CUDA tensors afterwards; :func:`uninstall`
    puts the originals back."""
    import importlib
    import sys

    if package is None:
        package = importlib.import_module("tensorlbm")
    prefix = package.__name__
    swap = {}        # id(original) -> (original, replacement)
    patched = []
    for mod_name, names in _PATCHES.items():
        ours = importlib.import_module(f"{__name__}.{mod_name}")
        try:
            theirs = importlib.import_module(f"{prefix}.{mod_name}")
        except ImportError:
            continue
        for name in names:
            if not hasattr(theirs, name):
                continue
            orig, repl = getattr(theirs, name), getattr(ours, name)
            if orig is not repl:
                swap[id(orig)] = (orig, repl)
            patched.append(f"{mod_name}.{name}")
    for mname, mod in list(sys.modules.items()):
        if mod is None or not (mname == prefix or mname.startswith(prefix + ".")):
            continue
        for attr, val in list(vars(mod).items()):
            hit = swap.get(id(val))
            if hit is not None and hit[0] is val:
                _ORIGINALS.setdefault((mname, attr), val)
                setattr(mod, attr, hit[1])
    return patched


def uninstall() -> int:
    """Undo :func:`install`: every rebound global gets its original object
    back.  Returns the number of bindings restored."""
    import sys

    n = 0
    for (mname, attr), val in list(_ORIGINALS.items()):
        mod = sys.modules.get(mname)
        if mod is not None:
            setattr(mod, attr, val)
            n += 1
    _ORIGINALS.clear()
    return n
