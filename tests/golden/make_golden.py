"""Generate golden vectors from the unmodified TensorLBM reference.

Run from the repository root in a checkout that has the reference source:

    python tests/golden/make_golden.py [--reference /path/to/TensorLBM/src]

It imports TensorLBM's torch operators on the CPU (a stub ``matplotlib``
package is put on sys.path first, because TensorLBM's package ``__init__``
imports matplotlib for plotting and matplotlib is not installed here), runs
each hot-path function on small seeded inputs and writes the inputs and
outputs to ``tests/golden/*.npz``.  The tests load these files; nothing at
test time needs the reference.
"""

from __future__ import annotations

import argparse
import pathlib
import sys
import tempfile
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent

_STUB = '''
import sys, types, importlib.abc, importlib.machinery
class _Dummy:
    def __getattr__(self, name): return _Dummy()
    def __call__(self, *a, **k): return _Dummy()
    def __iter__(self): return iter(())
def use(*a, **k): pass
class _Finder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, name, path, target=None):
        if name.startswith("matplotlib.") or name.startswith("mpl_toolkits"):
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None
    def create_module(self, spec):
        m = types.ModuleType(spec.name); m.__path__ = []
        m.__getattr__ = lambda n: _Dummy(); return m
    def exec_module(self, module): pass
sys.meta_path.insert(0, _Finder())
def __getattr__(name): return _Dummy()
'''


def import_reference(src: str):
    stub_dir = pathlib.Path(tempfile.mkdtemp(prefix="tlbm_stub_"))
    (stub_dir / "matplotlib").mkdir()
    (stub_dir / "matplotlib" / "__init__.py").write_text(_STUB)
    sys.path[:0] = [str(stub_dir), src]
    import tensorlbm  # noqa: F401

    return tensorlbm


def near_eq_field(torch, q, spatial, dtype, seed, amp=0.05, noise=0.01):
    """Random rho ~ 1 +- amp, |u| ~ amp, plus a non-equilibrium perturbation."""
    from tensorlbm.d2q9 import equilibrium
    from tensorlbm.d3q19 import equilibrium3d
    from tensorlbm.d3q27 import equilibrium27

    g = torch.Generator().manual_seed(seed)
    rho = 1.0 + amp * (2 * torch.rand(spatial, generator=g, dtype=torch.float64) - 1)
    u = [amp * (2 * torch.rand(spatial, generator=g, dtype=torch.float64) - 1) for _ in range(3)]
    rho, u = rho.to(dtype), [v.to(dtype) for v in u]
    if q == 9:
        feq = equilibrium(rho, u[0], u[1])
    elif q == 19:
        feq = equilibrium3d(rho, *u)
    else:
        feq = equilibrium27(rho, *u)
    pert = noise * (2 * torch.rand(feq.shape, generator=g, dtype=torch.float64) - 1).to(dtype)
    return rho, u, feq * (1 + pert)


def moving_wall(torch) -> None:
    """Ladd moving-wall bounce-back (rotating_cylinder.py / propeller_benchmark.py)
    on a rotating disc / rotor-like cylinder, float32 and float64."""
    from tensorlbm.propeller_benchmark import moving_wall_bounce_back_3d, rotating_wall_velocity_3d
    from tensorlbm.rotating_cylinder import moving_wall_bounce_back, rotating_wall_velocity

    out = {}
    sp2, sp3 = (32, 64), (8, 12, 32)
    for dt, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        _, _, f9 = near_eq_field(torch, 9, sp2, dt, 51)
        _, _, f19 = near_eq_field(torch, 19, sp3, dt, 52)
        yy, xx = torch.meshgrid(torch.arange(sp2[0]), torch.arange(sp2[1]), indexing="ij")
        disc = (xx - 30.3) ** 2 + (yy - 15.6) ** 2 <= 9.5 ** 2
        ux2, uy2 = rotating_wall_velocity(disc, 30.3, 15.6, 0.004)
        zz, yy3, xx3 = torch.meshgrid(torch.arange(sp3[0]), torch.arange(sp3[1]), torch.arange(sp3[2]), indexing="ij")
        rotor = ((yy3 - 5.6) ** 2 + (zz - 3.8) ** 2 <= 3.2 ** 2) & (xx3 >= 9) & (xx3 < 21)
        ux3, uy3, uz3 = rotating_wall_velocity_3d(rotor, 15.0, 5.6, 3.8, 0.006)
        out.update({f"f9_{tag}": f9, f"f19_{tag}": f19,
                    # outputs on the masked cells only; the others must equal the input
                    f"mw9_{tag}": moving_wall_bounce_back(f9, disc, ux2, uy2)[:, disc],
                    f"mw19_{tag}": moving_wall_bounce_back_3d(f19, rotor, ux3, uy3, uz3)[:, rotor]})
        out.update({"disc": disc, "rotor": rotor, "ux2": ux2, "uy2": uy2, "ux3": ux3, "uy3": uy3, "uz3": uz3})
    arrays = {k: (v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else np.asarray(v)) for k, v in out.items()}
    np.savez_compressed(HERE / "moving_wall.npz", **arrays)
    print("wrote moving_wall.npz")


def checkpoints(torch) -> None:
    """Checkpoint files written by TensorLBM itself (checkpoint.py): a
    format-1 pair directory and a format-2 solver-state file, to pin the
    readers of tensorlbm_b200.checkpoint to the reference's own output."""
    import shutil
    import types

    from tensorlbm.checkpoint import eager_state_dict, save_checkpoint, save_solver_checkpoint

    out = HERE / "checkpoint_ref"
    if out.exists():
        shutil.rmtree(out)
    g = torch.Generator().manual_seed(20261203)
    f = torch.rand((19, 2, 3, 4), generator=g, dtype=torch.float32)
    save_checkpoint(f, 123, out / "pair", extra={"case": "golden", "tau": 0.6})
    solver = types.SimpleNamespace(tau=0.55, nz=2, ny=3, nx=4, Q=19, lattice="D3Q19",
                                   mask=torch.rand((2, 3, 4), generator=g) > 0.7)
    torch.manual_seed(7)
    state = eager_state_dict(solver, f * 2.0, step=77, extra={"note": "golden"})
    save_solver_checkpoint(out / "solver_v2.pt", state, metadata={"run": "golden"})
    np.savez_compressed(out / "expected.npz", f=f.numpy(), f2=(f * 2.0).numpy(), mask=solver.mask.numpy(),
                        rng_after_seed7=torch.rand(4, generator=torch.Generator().manual_seed(7)).numpy())
    print(f"wrote {out}")


def rlbm(torch) -> None:
    """Regularised BGK collisions (solver.py:338, solver3d.py:342, d3q27.py:481)
    on seeded near-equilibrium fields, and on the same fields with a seeded
    perturbation of 5 % that puts weight in the higher-order (ghost) moments."""
    from tensorlbm.d3q27 import collide_rlbm27
    from tensorlbm.solver import collide_rlbm
    from tensorlbm.solver3d import collide_rlbm3d

    out = {}
    fns = {9: collide_rlbm, 19: collide_rlbm3d, 27: collide_rlbm27}
    shapes = {9: (8, 8), 19: (4, 4, 8), 27: (4, 4, 8)}
    for dt, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        for q, seed in ((9, 13), (19, 23), (27, 33)):
            _, _, f = near_eq_field(torch, q, shapes[q], dt, seed)
            g = torch.Generator().manual_seed(seed + 100)
            fr = f * (1.0 + 0.05 * (2.0 * torch.rand(f.shape, generator=g, dtype=torch.float64) - 1.0)).to(dt)
            out.update({f"f{q}_{tag}": f, f"rlbm{q}_{tag}": fns[q](f, 0.6), f"rlbm{q}_low_{tag}": fns[q](f, 0.5046),
                        f"fr{q}_{tag}": fr, f"rlbmr{q}_{tag}": fns[q](fr, 0.53)})
    arrays = {k: v.detach().cpu().numpy() for k, v in out.items()}
    np.savez_compressed(HERE / "collide_rlbm.npz", **arrays)
    print("wrote collide_rlbm.npz")


def far_field(torch) -> None:
    """Free-stream far field (boundaries.py:199, boundaries3d.py:446 with and
    without a y-only bc_config, boundaries_d3q27.py:63) on seeded fields with a
    small obstacle, float32 and float64, and the sponge strength of
    boundaries.py:388."""
    from tensorlbm.boundaries import far_field_bc_2d, make_sponge_strength
    from tensorlbm.boundaries3d import far_field_bc_3d
    from tensorlbm.boundaries_d3q27 import far_field_bc_27

    out = {}
    for dt, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        _, _, f9 = near_eq_field(torch, 9, (8, 16), dt, 41)
        _, _, f19 = near_eq_field(torch, 19, (4, 6, 8), dt, 43)
        _, _, f27 = near_eq_field(torch, 27, (4, 6, 8), dt, 47)
        ob9 = torch.zeros((8, 16), dtype=torch.bool)
        ob9[3:5, 6:8] = True
        ob3 = torch.zeros((4, 6, 8), dtype=torch.bool)
        ob3[1:3, 2:4, 3:5] = True
        cfg_y = {"far_field_faces": ["y-", "y+"], "periodic_faces": ["z-", "z+"]}
        out.update({f"f9_{tag}": f9, f"ff9_{tag}": far_field_bc_2d(f9, 0.07, ob9),
                    f"f19_{tag}": f19, f"ff19_{tag}": far_field_bc_3d(f19, 0.06, ob3),
                    f"ff19y_{tag}": far_field_bc_3d(f19, 0.06, None, bc_config=cfg_y),
                    f"ff19uv_{tag}": far_field_bc_3d(f19, 0.06, None, uy=0.01, uz=-0.02),
                    f"f27_{tag}": f27, f"ff27_{tag}": far_field_bc_27(f27, 0.05, ob3)})
    out.update(ob9=ob9, ob3=ob3, sponge=make_sponge_strength(8, 40, 25, 10, power=2.0))
    arrays = {k: v.detach().cpu().numpy() for k, v in out.items()}
    np.savez_compressed(HERE / "far_field.npz", **arrays)
    print("wrote far_field.npz")


def trt(torch) -> None:
    """TRT collisions (solver.py:440, solver3d.py:303, d3q27.py:438) on the
    seeded near-equilibrium fields of the other collision fixtures."""
    from tensorlbm.d3q27 import collide_trt27
    from tensorlbm.solver import collide_trt
    from tensorlbm.solver3d import collide_trt3d

    out = {}
    _, _, f9 = near_eq_field(torch, 9, (8, 8), torch.float32, 11)
    out.update(f9=f9, trt9=collide_trt(f9, 0.6), trt9_lam=collide_trt(f9, 0.57, lambda_trt=0.25))
    for dt, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        _, _, f19 = near_eq_field(torch, 19, (4, 4, 8), dt, 21)
        _, _, f27 = near_eq_field(torch, 27, (4, 4, 8), dt, 31)
        out.update({f"f19_{tag}": f19, f"trt19_{tag}": collide_trt3d(f19, 0.6),
                    f"trt19_lam_{tag}": collide_trt3d(f19, 0.57, lambda_trt=0.25),
                    f"f27_{tag}": f27, f"trt27_{tag}": collide_trt27(f27, 0.6),
                    f"trt27_lam_{tag}": collide_trt27(f27, 0.57, lambda_trt=0.25)})
    arrays = {k: v.detach().cpu().numpy() for k, v in out.items()}
    np.savez_compressed(HERE / "collide_trt.npz", **arrays)
    print("wrote collide_trt.npz")


def bfl(torch) -> None:
    """Bouzidi (BFL) interpolated bounce-back: the sphere link fields
    (bfl_common.py:384, interpolated_bc_common.py:136), the link update
    (bfl_common.py:106) with its force ledger (bfl_d3q19.py:195), and a short
    chain composed in bfl_step's order (bfl_common.py:882): BGK collide ->
    solid cells back to pre-collision -> bounce_back_cells_3d -> stream3d ->
    BFL on the links (with force)."""
    from tensorlbm.bfl_common import bfl_bounce_back_common, compute_q_sphere_common
    from tensorlbm.bfl_d3q19 import bouzidi_bounce_back_d3q19
    from tensorlbm.boundaries3d import bounce_back_cells_3d
    from tensorlbm.d3q19 import equilibrium3d
    from tensorlbm.interpolated_bc_common import compute_q_sphere_27
    from tensorlbm.solver3d import collide_bgk3d, stream3d

    out = {}
    cpu = torch.device("cpu")
    m19, q19 = compute_q_sphere_common(16, 14, 12, 7.3, 6.6, 5.8, 3.7, cpu, lattice="D3Q19")
    m27, q27 = compute_q_sphere_27(12, 11, 10, 5.4, 5.1, 4.7, 2.9, cpu)
    m27c, q27c = compute_q_sphere_common(12, 11, 10, 5.4, 5.1, 4.7, 2.9, cpu, lattice="D3Q27")
    assert torch.equal(m27, m27c) and torch.equal(q27, q27c)
    out.update(m19=m19, q19=q19, m27=m27, q27=q27)
    for q, m, qf, sp, seed in ((19, m19, q19, (12, 14, 16), 61), (27, m27, q27, (10, 11, 12), 62)):
        _, _, fa = near_eq_field(torch, q, sp, torch.float32, seed)
        _, _, fb = near_eq_field(torch, q, sp, torch.float32, seed + 100)
        out[f"f{q}"], out[f"fprev{q}"] = fa, fb
        out[f"bfl{q}"] = bfl_bounce_back_common(fa, fb, m, qf, lattice=f"D3Q{q}")
    f19_force, force = bouzidi_bounce_back_d3q19(out["f19"], out["fprev19"], m19, q19, return_force=True)
    assert torch.equal(f19_force, out["bfl19"])
    out["force19"] = torch.stack(list(force))

    # chain: periodic 24 x 16 x 16 box, sphere r = 3.6 at (9.3, 7.6, 8.2), BGK tau 0.56
    nz, ny, nx = 16, 16, 24
    mask, qfield = compute_q_sphere_common(nx, ny, nz, 9.3, 7.6, 8.2, 3.6, cpu, lattice="D3Q19")
    zz, yy, xx = torch.meshgrid(*(torch.arange(n, dtype=torch.float64) for n in (nz, ny, nx)), indexing="ij")
    solid = ((xx - 9.3) ** 2 + (yy - 7.6) ** 2 + (zz - 8.2) ** 2) <= 3.6 ** 2
    ux = torch.full((nz, ny, nx), 0.03, dtype=torch.float32)
    ux[solid] = 0.0
    zero = torch.zeros_like(ux)
    f = equilibrium3d(torch.ones_like(ux), ux, zero, zero)
    out.update(chain_f0=f.clone(), chain_mask=mask, chain_q=qfield, chain_solid=solid)
    tau, forces = 0.56, []
    for _ in range(8):
        f_post = collide_bgk3d(f, tau)
        g = torch.where(solid.unsqueeze(0), f, f_post)            # no dynamics in the solid
        g = bounce_back_cells_3d(g, solid)
        f, fo = bouzidi_bounce_back_d3q19(stream3d(g), g, mask, qfield, return_force=True)
        forces.append(torch.stack(list(fo)))
    out.update(chain_f=f, chain_forces=torch.stack(forces), chain_tau=torch.tensor(tau))
    arrays = {k: v.detach().cpu().numpy() for k, v in out.items()}
    np.savez_compressed(HERE / "bfl.npz", **arrays)
    print(f"wrote bfl.npz ({(HERE / 'bfl.npz').stat().st_size / 1024:.0f} KB); links per grid "
          f"{int(m19.sum())}, {int(m27.sum())}, chain {int(mask.sum())}")


def cascaded(torch) -> None:
    """Cascaded central-moment collisions (cascaded_collision.py:445, :512)."""
    from tensorlbm.cascaded_collision import collide_cascaded_d3q19, collide_cascaded_d3q27

    out = {}
    for dt, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        _, _, f19 = near_eq_field(torch, 19, (4, 4, 8), dt, 71)
        _, _, f27 = near_eq_field(torch, 27, (4, 4, 8), dt, 72)
        out.update({f"f19_{tag}": f19, f"c19_{tag}": collide_cascaded_d3q19(f19, 0.6),
                    f"c19r_{tag}": collide_cascaded_d3q19(f19, 0.57, s_bulk=1.2, s_3=0.9, s_4=1.3),
                    f"f27_{tag}": f27, f"c27_{tag}": collide_cascaded_d3q27(f27, 0.6),
                    f"c27r_{tag}": collide_cascaded_d3q27(f27, 0.57, s_bulk=1.2, s_3=0.9, s_4=1.3, s_5=1.1, s_6=0.8)})
    np.savez_compressed(HERE / "collide_cascaded.npz", **{k: v.numpy() for k, v in out.items()})
    print("wrote collide_cascaded.npz")


def mem(torch) -> None:
    """Link-wise momentum-exchange drag variants (momentum_exchange.py:75, :138,
    :206, :285) on a seeded field: a sphere plus a wall plane at x = nx - 1
    (links that cross the periodic x face), the near-wall mask restricted to
    z < nz - 3 so that the uniform-stream background does not cancel, scalar and
    per-direction wall fractions with zeros (the 1e-6 clamp)."""
    from tensorlbm import momentum_exchange as me

    nz, ny, nx = 12, 14, 16
    zz, yy, xx = torch.meshgrid(*(torch.arange(n, dtype=torch.float64) for n in (nz, ny, nx)), indexing="ij")
    solid = ((xx - 6.3) ** 2 + (yy - 7.1) ** 2 + (zz - 5.6) ** 2) <= 3.4 ** 2
    solid[:, :, nx - 1] = True
    any_solid = torch.zeros_like(solid)
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                any_solid |= torch.roll(solid, (dz, dy, dx), dims=(0, 1, 2))
    near = any_solid & ~solid
    near[nz - 3:] = False
    g = torch.Generator().manual_seed(81)
    q_scalar = torch.rand((nz, ny, nx), generator=g)
    q_scalar[q_scalar < 0.05] = 0.0
    q_dir = torch.rand((19, nz, ny, nx), generator=g)
    q_dir[q_dir < 0.05] = 0.0
    out = dict(solid=solid, near=near, q_scalar=q_scalar, q_dir=q_dir)
    for dt, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        _, _, f = near_eq_field(torch, 19, (nz, ny, nx), dt, 82)
        out[f"f_{tag}"] = f
        out[f"standard_{tag}"] = torch.tensor(me.momentum_exchange_standard(f, solid, near), dtype=torch.float64)
        out[f"galilean_{tag}"] = torch.tensor(me.momentum_exchange_galilean(f, solid, near, 0.6), dtype=torch.float64)
        out[f"background_{tag}"] = torch.tensor(
            me.momentum_exchange_background_subtracted(f, solid, near, rho0=1.02, u0=(0.05, 0.01, -0.02)),
            dtype=torch.float64)
        out[f"bfl_scalar_{tag}"] = torch.tensor(me.momentum_exchange_bfl(f, solid, near, q_scalar), dtype=torch.float64)
        out[f"bfl_dir_{tag}"] = torch.tensor(me.momentum_exchange_bfl(f, solid, near, q_dir), dtype=torch.float64)
    np.savez_compressed(HERE / "mem.npz", **{k: v.numpy() for k, v in out.items()})
    print(f"wrote mem.npz; links {int(near.sum())} near cells")


def links_c2(torch) -> None:
    """The solid mask and link list of the 512x256x256 sphere channel at full
    size: sphere_mask(512, 256, 256, 128, 128, 128, 16) (boundaries3d.py:29),
    derive_missing_mask with periodic y/z and a closed x (boundary_registry.py:488),
    then torch.nonzero, for D3Q19 and D3Q27.  The (n, 4) (q, z, y, x) list is
    stored as flat row-major indices, delta-encoded (the first entry, then the
    differences, all positive because nonzero is ordered), next to the SHA-256
    of the int64 nonzero output, so a test can check every entry and the exact
    bytes torch returned."""
    import hashlib

    from tensorlbm import boundaries3d as b3
    from tensorlbm.boundary_registry import derive_missing_mask

    cpu = torch.device("cpu")
    nz, ny, nx = 256, 256, 512
    solid = b3.sphere_mask(nx, ny, nz, 128, 128, 128, 16, cpu)
    out = {"shape": np.array([nz, ny, nx])}
    for lat in ("D3Q19", "D3Q27"):
        miss = derive_missing_mask((nz, ny, nx), solid_mask=solid, periodic={"y": True, "z": True, "x": False},
                                   lattice=lat)
        links = torch.nonzero(miss)
        q = miss.shape[0]
        del miss
        dims = torch.tensor([nz * ny * nx, ny * nx, nx, 1], dtype=torch.int64)
        flat = (links * dims).sum(dim=1).numpy()
        assert np.all(np.diff(flat) > 0)
        delta = np.diff(flat, prepend=np.int64(0))
        assert delta.max() < 2**32
        tag = lat[2:].lower()
        out[f"count_{tag}"] = np.int64(links.shape[0])
        out[f"q_{tag}"] = np.int64(q)
        out[f"delta_{tag}"] = delta.astype(np.uint32)
        out[f"sha256_{tag}"] = np.frombuffer(hashlib.sha256(links.contiguous().numpy().tobytes()).digest(),
                                             dtype=np.uint8)
        print(f"  {lat}: {links.shape[0]} links")
    np.savez_compressed(HERE / "links_c2.npz", **out)
    print(f"wrote links_c2.npz ({(HERE / 'links_c2.npz').stat().st_size / 1024:.0f} KB)")


def mass(torch) -> None:
    """Global mass correction f * (target / f.sum()) (solver.py:420,
    solver3d.py:287, d3q27.py:729) on seeded near-equilibrium fields, float32
    and float64, plus the all-zero field that the 1e-30 guard returns as is."""
    from tensorlbm.d3q27 import correct_mass27
    from tensorlbm.solver import correct_mass
    from tensorlbm.solver3d import correct_mass3d

    out = {}
    for dt, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        _, _, f9 = near_eq_field(torch, 9, (16, 32), dt, 91)
        _, _, f19 = near_eq_field(torch, 19, (4, 6, 16), dt, 92)
        _, _, f27 = near_eq_field(torch, 27, (4, 6, 16), dt, 93)
        t9, t19, t27 = 0.97 * float(f9.double().sum()), 1.013 * float(f19.double().sum()), 1001.5
        out.update({f"f9_{tag}": f9, f"t9_{tag}": t9, f"m9_{tag}": correct_mass(f9, t9),
                    f"f19_{tag}": f19, f"t19_{tag}": t19, f"m19_{tag}": correct_mass3d(f19, t19),
                    f"f27_{tag}": f27, f"t27_{tag}": t27, f"m27_{tag}": correct_mass27(f27, t27)})
    zero = torch.zeros((19, 2, 3, 4))
    out["zero_out"] = correct_mass3d(zero, 5.0)
    arrays = {k: (v.numpy() if isinstance(v, torch.Tensor) else np.asarray(v)) for k, v in out.items()}
    np.savez_compressed(HERE / "mass.npz", **arrays)
    print("wrote mass.npz")


def c4_divergence(torch, max_steps: int = 5_000, nx_max: int = 160) -> None:
    """The smallest design points of the batched-form scan (nx <= 160, ny = nx/4,
    cylinder D = ny/8; the seeded design of tensorlbm_b200.batch.uniform_scan
    with seed 20261203), run through TensorLBM's own D2Q9 cylinder chain
    (cylinder_flow.py:854-899, zou_he outlet mode): collide_bgk -> stream ->
    compute_obstacle_forces -> zou_he_inlet_velocity -> zou_he_outlet_pressure ->
    bounce_back_cells(wall) -> bounce_back_cells(cylinder), for up to
    max_steps steps.  Records the first step whose populations are not all
    finite (-1 if none), and for two nx = 128 points the last finite state at
    or before step 200."""
    from tensorlbm import boundaries as b2
    from tensorlbm.d2q9 import equilibrium
    from tensorlbm.solver import collide_bgk, stream

    g = torch.Generator().manual_seed(20261203)
    n = 512
    nxs = torch.randint(128 // 8, 1024 // 8 + 1, (n,), generator=g) * 8
    res = 40.0 + 260.0 * torch.rand(n, generator=g, dtype=torch.float64)
    pick = [i for i in range(n) if int(nxs[i]) <= nx_max]
    cpu = torch.device("cpu")
    out = {"domains": np.array(pick), "max_steps": max_steps}
    for i in pick:
        nx = int(nxs[i])
        ny = nx // 4
        d = ny / 8.0
        re = float(res[i])
        tau = 3.0 * 0.05 * d / re + 0.5
        obst = b2.cylinder_mask(nx, ny, ny / 2.0, ny / 2.0, d / 2.0, cpu)
        wall = b2.make_channel_wall_mask(ny, nx, obst, cpu)
        ux = torch.full((ny, nx), 0.05)
        ux[obst] = 0.0
        f = equilibrium(torch.ones((ny, nx)), ux, torch.zeros((ny, nx)))
        nan_step, check, check_step = -1, f.clone(), 0
        t0 = time.time()
        for step in range(1, max_steps + 1):
            f = collide_bgk(f, tau)
            f = stream(f)
            b2.compute_obstacle_forces(f, obst)
            f = b2.zou_he_inlet_velocity(f, 0.05)
            f = b2.zou_he_outlet_pressure(f, rho_out=1.0)
            f = b2.bounce_back_cells(f, wall)
            f = b2.bounce_back_cells(f, obst)
            if not bool(torch.isfinite(f).all()):
                nan_step = step
                break
            if step <= 200:
                check, check_step = f.clone(), step
        out[f"re_{i}"] = re
        out[f"tau_{i}"] = tau
        out[f"nan_step_{i}"] = nan_step
        if i in (118, 364):   # the last finite state at or before step 200
            out[f"check_{i}"] = check.numpy()
            out[f"check_step_{i}"] = check_step
        print(f"  domain {i}: nx {nx} Re {re:.1f} tau {tau:.5f} -> non-finite at step {nan_step} "
              f"({time.time() - t0:.0f} s)")
    np.savez_compressed(HERE / "c4_divergence.npz", **out)
    print("wrote c4_divergence.npz")


def cavity_case(torch) -> None:
    """TensorLBM's registered lid-driven cavity case (cases/cavity.py:25-110),
    stepped with the case's own chain (CaseBase.make_step, cases/base.py:270-289:
    collide -> pre-streaming half-way walls from the pre-collision state ->
    stream -> Zou/He lid) from case.initial_f(), for three scan points: BGK at
    resolution 32 (Re 100), MRT at 24 (Re 150) and MRT on (6, 20, 40) (Re 200).
    Stores the mid-plane z = nz // 2 of the final populations, the float64 sum
    of every direction, the case's tau and the point's parameters."""
    from tensorlbm.cases import get_case

    points = {"bgk32": dict(resolution=32, re=100.0, collision="bgk", steps=300),
              "mrt24": dict(resolution=24, re=150.0, collision="mrt", steps=300),
              "mrt6x20x40": dict(resolution=(6, 20, 40), re=200.0, collision="mrt", steps=300)}
    out = {}
    for tag, pt in points.items():
        case = get_case("cavity", resolution=pt["resolution"], re=pt["re"], collision=pt["collision"],
                        device="cpu")
        step = case.make_step()
        f = case.initial_f()
        for _ in range(pt["steps"]):
            f = step(f)
        nz = f.shape[1]
        out[f"{tag}_shape"] = np.array(f.shape[1:])
        out[f"{tag}_tau"] = case.units.tau
        out[f"{tag}_re"] = pt["re"]
        out[f"{tag}_u_lid"] = case.u_lid
        out[f"{tag}_steps"] = pt["steps"]
        out[f"{tag}_mid"] = f[:, nz // 2].numpy()
        out[f"{tag}_qsum"] = f.double().sum(dim=(1, 2, 3)).numpy()
        print(f"  cavity {tag}: grid {tuple(f.shape[1:])}, tau {case.units.tau:.5f}, finite {bool(torch.isfinite(f).all())}")
    np.savez_compressed(HERE / "cavity_case.npz", **out)
    print(f"wrote cavity_case.npz ({(HERE / 'cavity_case.npz').stat().st_size / 1024:.0f} KB)")


def tgv_laminar(src: str) -> None:
    """TensorLBM's verified laminar Taylor-Green decay
    (benchmarks/verified/taylor_green_3d: run.py, result.json and the
    energy_history_N*.csv files it wrote, D3Q19 BGK float32 at Re 24 on
    N = 64, 96, 128): the recorded steps, energies E = <|u|^2>/2 and the
    fitted gamma_E of each grid, copied from the reference's own outputs."""
    import json

    bench = pathlib.Path(src).parent / "benchmarks" / "verified" / "taylor_green_3d"
    res = json.loads((bench / "result.json").read_text())
    out = {}
    for case in res["cases"]:
        n = int(case["n"])
        rows = np.loadtxt(bench / f"energy_history_N{n}.csv", delimiter=",", skiprows=1)
        out[f"n{n}_record_steps"] = rows[:, 0].astype(np.int64)
        out[f"n{n}_energy"] = rows[:, 1]
        for key in ("re", "u0", "tau", "steps", "record_every", "gamma_e_sim", "gamma_e_theory", "r2"):
            out[f"n{n}_{key}"] = np.asarray(case[key])
    np.savez_compressed(HERE / "tgv_laminar.npz", **out)
    print(f"wrote tgv_laminar.npz ({len(res['cases'])} grids)")


def cavity3d_full(src: str) -> None:
    """TensorLBM's verified 3-D lid-driven cavity at Re 1000
    (benchmarks/verified/cavity_3d_full: run.py and the case_643.json /
    case_963.json it wrote, D3Q19 TRT, five half-way walls, Zou/He lid,
    100 000 steps): the centre-plane centre lines, u_min and the mass drift of
    each grid, copied from the reference's own outputs."""
    import json

    bench = pathlib.Path(src).parent / "benchmarks" / "verified" / "cavity_3d_full"
    out = {}
    for tag in ("643", "963"):
        case = json.loads((bench / f"case_{tag}.json").read_text())
        n = int(case["nx"])
        for key in ("u_centerline_mid", "v_centerline_mid"):
            out[f"n{n}_{key}"] = np.asarray(case[key], dtype=np.float64)
        for key in ("re", "u_lid", "tau", "n_steps_run", "u_min_3d_mid", "mass_drift", "last_resid"):
            out[f"n{n}_{key}"] = np.asarray(case[key])
    np.savez_compressed(HERE / "cavity3d_full.npz", **out)
    print(f"wrote cavity3d_full.npz ({sorted(out)})")


def cavity2d(src: str, re: int) -> None:
    """TensorLBM's verified 2-D lid-driven cavity (benchmarks/verified/cavity/
    re100 and re1000: run.py and the result.json it wrote; three half-way
    walls, Zou/He lid; Re 100: D2Q9 MRT, 128^2 and 192^2, 100 000 steps;
    Re 1000: D2Q9 regularised BGK, 192^2 and 256^2, 200 000 steps): the point
    values u(0.5, 0.5), u(0.5, 0.0625), v(0.5, 0.5) of each grid (and the
    primary vortex centre where recorded), copied from the reference's own
    outputs."""
    import json

    res = json.loads((pathlib.Path(src).parent / "benchmarks" / "verified" / "cavity" / f"re{re}" /
                      "result.json").read_text())
    out = {}
    for key, case in res["grids"].items():
        n = int(case["nx"])
        for k in ("re", "u_lid", "tau", "steps", "u_mid", "u_bot", "v_mid", "last_resid", "primary_vortex"):
            if k in case:
                out[f"n{n}_{k}"] = np.asarray(case[k])
    np.savez_compressed(HERE / f"cavity2d_re{re}.npz", **out)
    print(f"wrote cavity2d_re{re}.npz ({sorted(out)})")


def cylinder2d(src: str) -> None:
    """TensorLBM's verified free-stream cylinder at Re 100
    (benchmarks/verified/cylinder/re100: run.py and the result.json it wrote;
    D2Q9 MRT with a sponge tau field, far field, seeded wake, D = 48 and 64,
    60 000 / 90 000 steps): the drag coefficient and Strouhal number of each
    grid, copied from the reference's own outputs."""
    import json

    res = json.loads((pathlib.Path(src).parent / "benchmarks" / "verified" / "cylinder" / "re100" /
                      "result.json").read_text())
    out = {}
    for case in res["grids"].values():
        d = int(case["D"])
        for k in ("steps", "cd", "st"):
            out[f"d{d}_{k}"] = np.asarray(case[k])
    np.savez_compressed(HERE / "cylinder2d_re100.npz", **out)
    print(f"wrote cylinder2d_re100.npz ({sorted(out)})")


def cylinder2d_small(src: str) -> None:
    """The verified cylinder's own run.py (benchmarks/verified/cylinder/re100,
    run_case, eager torch on the CPU) at D = 8 (320 x 320) for 3000 steps:
    its per-step drag and lift coefficient series, Cd and St."""
    import importlib.util
    import tempfile

    import torch

    torch.set_num_threads(8)
    path = pathlib.Path(src).parent / "benchmarks" / "verified" / "cylinder" / "re100" / "run.py"
    spec = importlib.util.spec_from_file_location("cylinder_re100_run", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    with tempfile.TemporaryDirectory() as tmp:
        series = pathlib.Path(tmp) / "series.npz"
        res = mod.run_case(8, 100.0, 0.05, 3000, torch.device("cpu"), compile_mode=None, warmup_frac=0.5,
                           series_path=str(series))
        s = np.load(series)
        out = {"cd_series": s["cd"], "cl_series": s["cl"], "cd": np.asarray(res["cd"]),
               "st": np.asarray(res["st"] if res["st"] is not None else np.nan), "steps": np.asarray(3000),
               "seed_steps": np.asarray(res["seed"]["steps"])}
    np.savez_compressed(HERE / "cylinder2d_small.npz", **out)
    print(f"wrote cylinder2d_small.npz (Cd {float(res['cd'])}, St {res['st']})")


def tgv2d(src: str) -> None:
    """TensorLBM's verified decaying 2-D Taylor-Green vortex
    (benchmarks/verified/taylor_green_2d: run.py and the energy_history.csv /
    result.json it wrote; N = 128, Re 100, D2Q9 BGK float32 on the CPU, 4900
    steps): the recorded energy and max|u| histories, decay rates and mass drift."""
    import json

    bench = pathlib.Path(src).parent / "benchmarks" / "verified" / "taylor_green_2d"
    hist = np.loadtxt(bench / "energy_history.csv", delimiter=",", skiprows=1)
    res = json.loads((bench / "result.json").read_text())
    out = {"steps_recorded": hist[:, 0].astype(np.int64), "energy": hist[:, 1], "umax": hist[:, 2]}
    for k in ("n", "re", "u0", "steps", "record_every", "gamma_e_sim", "gamma_vel_sim", "mass_drift_rel"):
        out[k] = np.asarray(res[k])
    np.savez_compressed(HERE / "tgv2d.npz", **out)
    print(f"wrote tgv2d.npz ({sorted(out)})")


def pipe3d(src: str) -> None:
    """TensorLBM's verified Hagen-Poiseuille pipe (benchmarks/verified/
    poiseuille_3d_pipe: run.py and the case_R20.json / case_R40.json it wrote,
    D3Q19 BGK, Zou/He velocity inlet and pressure outlet, full-way swap at the
    staircase pipe wall): the radial profile, centre velocity, flow rate,
    inlet density and mass drift of each radius, copied from the reference's
    own outputs."""
    import json

    bench = pathlib.Path(src).parent / "benchmarks" / "verified" / "poiseuille_3d_pipe"
    out = {}
    for r in (20, 40):
        case = json.loads((bench / f"case_R{r}.json").read_text())
        out[f"r{r}_u_profile"] = np.asarray(case["u_profile"], dtype=np.float64)
        for k in ("tau", "u_in", "n_steps", "u_center", "Q", "rho_in_measured", "mass_drift_pct", "L_over_R"):
            out[f"r{r}_{k}"] = np.asarray(case[k])
    np.savez_compressed(HERE / "pipe3d.npz", **out)
    print(f"wrote pipe3d.npz ({sorted(out)})")


def shear_wave(src: str, torch) -> None:
    """TensorLBM's verified decaying shear wave (benchmarks/verified/
    shear_wave_decay, D2Q9 BGK float32, tau 0.8, H = 64 and 128).  Two sets per
    grid: the case's parameters with the energies, largest |u| and decay rates
    the benchmark recorded (case_H*.json, energy_history_H*.csv; its step ran
    through torch.compile), and the same run of TensorLBM's eager operators
    here (collide_bgk(stream(f)), the benchmark's initial field and sampling,
    run.py:59-100), whose arithmetic the fused kernel reproduces."""
    import json
    import math

    from tensorlbm.d2q9 import equilibrium, macroscopic
    from tensorlbm.solver import collide_bgk, stream

    bench = pathlib.Path(src).parent / "benchmarks" / "verified" / "shear_wave_decay"
    out = {}
    for h in (64, 128):
        case = json.loads((bench / f"case_H{h}.json").read_text())
        rows = np.loadtxt(bench / f"energy_history_H{h}.csv", delimiter=",", skiprows=1)
        out[f"h{h}_record_steps"] = rows[:, 0].astype(np.int64)
        out[f"h{h}_energy_compiled"] = rows[:, 1]
        out[f"h{h}_umax_compiled"] = rows[:, 2]
        for k in ("tau", "u0", "steps", "record_every", "gamma_e_sim", "gamma_vel_sim"):
            out[f"h{h}_{k}"] = np.asarray(case[k])
        tau, u0, steps, every = float(case["tau"]), float(case["u0"]), int(case["steps"]), int(case["record_every"])
        k = 2.0 * math.pi / float(h)
        y, _ = torch.meshgrid(torch.arange(h, dtype=torch.float32), torch.arange(h, dtype=torch.float32), indexing="ij")
        ux0 = u0 * torch.sin(k * y)
        f = equilibrium(torch.ones_like(ux0), ux0, torch.zeros_like(ux0))
        energies, umaxs = [], []
        for step in range(1, steps + 1):
            f = collide_bgk(stream(f), tau)
            if step % every == 0:
                _, uxm, uym = macroscopic(f)
                energies.append(float((0.5 * (uxm * uxm + uym * uym)).mean().item()))
                umaxs.append(float((uxm * uxm + uym * uym).sqrt().max().item()))
        out[f"h{h}_energy"] = np.asarray(energies)
        out[f"h{h}_umax"] = np.asarray(umaxs)
        print(f"  shear wave H{h}: eager vs compiled energy max rel "
              f"{np.max(np.abs(out[f'h{h}_energy'] - rows[:, 1]) / rows[:, 1]):.2e}")
    np.savez_compressed(HERE / "shear_wave.npz", **out)
    print(f"wrote shear_wave.npz ({sorted(out)})")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference/src")
    ap.add_argument("--skip-long", action="store_true", help="skip the 64^3 x 1000-step cavity run")
    ap.add_argument("--only", default=None, help="write only this group of fixtures (e.g. moving_wall)")
    args = ap.parse_args()
    if args.only == "tgv_laminar":
        tgv_laminar(args.reference)
        return
    if args.only == "cavity3d_full":
        cavity3d_full(args.reference)
        return
    if args.only == "tgv2d":
        tgv2d(args.reference)
        return
    if args.only == "cylinder2d_re100":
        cylinder2d(args.reference)
        return
    if args.only == "cylinder2d_small":
        import_reference(args.reference)
        cylinder2d_small(args.reference)
        return
    if args.only in ("cavity2d_re100", "cavity2d_re1000"):
        cavity2d(args.reference, int(args.only[len("cavity2d_re"):]))
        return
    if args.only == "pipe3d":
        pipe3d(args.reference)
        return
    if args.only == "shear_wave":
        import_reference(args.reference)
        import torch

        torch.set_num_threads(8)
        shear_wave(args.reference, torch)
        return
    import_reference(args.reference)
    import torch

    torch.set_num_threads(8)
    if args.only == "moving_wall":
        moving_wall(torch)
        return
    if args.only == "checkpoints":
        checkpoints(torch)
        return
    if args.only == "trt":
        trt(torch)
        return
    if args.only == "rlbm":
        rlbm(torch)
        return
    if args.only == "far_field":
        far_field(torch)
        return
    if args.only == "bfl":
        bfl(torch)
        return
    if args.only == "cascaded":
        cascaded(torch)
        return
    if args.only == "mem":
        mem(torch)
        return
    if args.only == "links_c2":
        links_c2(torch)
        return
    if args.only == "mass":
        mass(torch)
        return
    if args.only == "c4_divergence":
        c4_divergence(torch)
        return
    if args.only == "cavity_case":
        cavity_case(torch)
        return
    from tensorlbm import boundaries as b2
    from tensorlbm import boundaries3d as b3
    from tensorlbm import boundaries_d3q27 as b27
    from tensorlbm import cumulant, obstacles, turbulence
    from tensorlbm.boundary_registry import derive_missing_mask
    from tensorlbm.d2q9 import equilibrium, macroscopic
    from tensorlbm.d3q19 import equilibrium3d, macroscopic3d
    from tensorlbm.d3q27 import collide_bgk27, collide_mrt27, equilibrium27, macroscopic27, stream27
    from tensorlbm.lid_driven_cavity import zou_he_moving_lid
    from tensorlbm.solver import collide_bgk, collide_mrt, stream
    from tensorlbm.solver3d import collide_bgk3d, collide_mrt3d, stream3d

    def save(name, **arrays):
        out = {k: (v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else np.asarray(v)) for k, v in arrays.items()}
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(f"  {name}.npz  ({(HERE / f'{name}.npz').stat().st_size / 1024:.0f} KB)")

    # inner sizes are multiples of 32, where torch's CPU reduction over the
    # direction axis follows one fixed order for every cell (see oracle.lbm.sum0)
    sp2 = (8, 8)            # (ny, nx)
    sp3 = (4, 4, 8)         # (nz, ny, nx)
    tau = 0.6

    print("moments / equilibrium")
    for dt, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        rho, u, f = near_eq_field(torch, 9, sp2, dt, 1)
        r, ux, uy = macroscopic(f)
        save(f"moments_d2q9_{tag}", f=f, rho_in=rho, ux_in=u[0], uy_in=u[1], feq=equilibrium(rho, u[0], u[1]),
             rho=r, ux=ux, uy=uy)
        for q, eqf, macf in ((19, equilibrium3d, macroscopic3d), (27, equilibrium27, macroscopic27)):
            rho, u, f = near_eq_field(torch, q, sp3, dt, q)
            r, ux, uy, uz = macf(f)
            save(f"moments_d3q{q}_{tag}", f=f, rho_in=rho, ux_in=u[0], uy_in=u[1], uz_in=u[2],
                 feq=eqf(rho, *u), rho=r, ux=ux, uy=uy, uz=uz)

    print("collisions")
    _, _, f9 = near_eq_field(torch, 9, sp2, torch.float32, 11)
    tf = 0.55 + 0.2 * torch.rand(sp2, generator=torch.Generator().manual_seed(5))
    save("collide_d2q9_f32", f=f9, tau=tau, tau_field=tf, bgk=collide_bgk(f9, tau), mrt=collide_mrt(f9, tau),
         mrt_field=collide_mrt(f9, tau, tau_field=tf), smag=turbulence.collide_smagorinsky_bgk(f9, tau, C_s=0.17))
    for dt, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        _, _, f19 = near_eq_field(torch, 19, sp3, dt, 21)
        kw19 = dict(f=f19, tau=tau, bgk=collide_bgk3d(f19, tau),
                    smag=turbulence.collide_smagorinsky_bgk3d(f19, tau, C_s=0.17),
                    cum19=cumulant.collide_cumulant_d3q19(f19, tau, omega_b=1.2, omega_even=0.8),
                    cum19_smag=cumulant.collide_cumulant_d3q19(f19, tau, omega_b=1.2, omega_even=0.8, C_s=0.17))
        if dt == torch.float32:  # the reference MRT matrices are float32 only
            kw19["mrt"] = collide_mrt3d(f19, tau)
            kw19["mrt_custom"] = collide_mrt3d(f19, tau, s_e=1.3, s_eps=1.5, s_q=1.1, s_pi=1.25)
        save(f"collide_d3q19_{tag}", **kw19)
        _, _, f27 = near_eq_field(torch, 27, sp3, dt, 31)
        kw27 = dict(f=f27, tau=tau, bgk=collide_bgk27(f27, tau),
                    smag=turbulence.collide_smagorinsky_bgk27(f27, tau, C_s=0.17),
                    cum=cumulant.collide_cumulant_d3q27(f27, tau, omega_b=1.1, omega_odd=1.2, omega_even=0.9),
                    geier=cumulant.collide_cumulant_geier_d3q27(f27, tau, omega_b=1.1, omega_odd=1.2, omega_even=0.9))
        if dt == torch.float32:
            kw27["mrt"] = collide_mrt27(f27, tau)
        save(f"collide_d3q27_{tag}", **kw27)

    print("streaming (integer canary: every value identifies its source)")
    def canary(q, spatial):
        n = int(np.prod(spatial))
        return torch.arange(q * n, dtype=torch.float32).reshape((q,) + spatial)
    c9 = canary(9, (5, 7))
    c19 = canary(19, (3, 4, 5))
    c27 = canary(27, (3, 4, 5))
    save("stream", f9=c9, s9=stream(c9), f19=c19, s19=stream3d(c19), f27=c27, s27=stream27(c27))

    print("boundaries")
    g = torch.Generator().manual_seed(7)
    m2 = torch.rand(sp2, generator=g) < 0.3
    m3 = torch.rand(sp3, generator=g) < 0.3
    _, _, f19 = near_eq_field(torch, 19, sp3, torch.float32, 41)
    _, _, f27 = near_eq_field(torch, 27, sp3, torch.float32, 42)
    _, _, f9 = near_eq_field(torch, 9, sp2, torch.float32, 43)
    prof = 0.05 + 0.01 * torch.rand(sp2[0], generator=g)
    save("bc_d2q9", f=f9, mask=m2, bb=b2.bounce_back_cells(f9, m2), inlet=b2.zou_he_inlet_velocity(f9, 0.05, 0.01),
         inlet_profile=b2.zou_he_inlet_velocity(f9, prof), profile=prof,
         outlet=b2.zou_he_outlet_pressure(f9, 1.02), lid=zou_he_moving_lid(f9, 0.07),
         force=torch.stack(b2.compute_obstacle_forces(f9, m2)))
    save("bc_d3q19", f=f19, mask=m3, bb=b3.bounce_back_cells_3d(f19, m3),
         inlet=b3.zou_he_inlet_velocity_3d(f19.clone(), 0.04, 0.01, -0.005),
         outlet=b3.zou_he_outlet_pressure_3d(f19.clone(), 0.98), lid=b3.zou_he_moving_lid_3d(f19, 0.05),
         force=torch.stack(obstacles.compute_obstacle_forces_3d(f19, m3)))
    save("bc_d3q27", f=f27, mask=m3, bb=b27.bounce_back_cells_27(f27, m3),
         inlet=b27.zou_he_inlet_velocity_27(f27, 0.04, 0.01, -0.005),
         outlet=b27.zou_he_outlet_pressure_27(f27, 0.98),
         force=torch.stack(obstacles.compute_obstacle_forces_27(f27, m3)))

    print("masks and links")
    cpu = torch.device("cpu")
    sph = b3.sphere_mask(32, 16, 16, 12.0, 8.0, 8.0, 4.5, cpu)
    sph_odd = b3.sphere_mask(40, 24, 20, 17.3, 11.7, 9.1, 6.35, cpu)
    big = b3.sphere_mask(512, 256, 256, 128, 128, 128, 16, cpu)  # sphere of D = 32 in the 512x256x256 channel
    cyl = b2.cylinder_mask(200, 50, 25.0, 25.0, 3.125, cpu)
    cyl_odd = b2.cylinder_mask(97, 31, 20.4, 15.5, 4.7, cpu)
    miss19 = derive_missing_mask((16, 16, 32), solid_mask=sph, periodic={"y": True, "z": True, "x": False},
                                 lattice="D3Q19")
    miss27 = derive_missing_mask((16, 16, 32), solid_mask=sph, periodic=False, lattice="D3Q27")
    links19 = torch.nonzero(miss19)
    save("masks", sphere=sph, sphere_odd=sph_odd, big_index=torch.nonzero(big.reshape(-1))[:, 0].to(torch.int64),
         big_count=big.sum(), cylinder=cyl, cylinder_odd=cyl_odd, missing19=np.packbits(miss19.numpy()),
         missing19_shape=np.array(miss19.shape), missing27=np.packbits(miss27.numpy()),
         missing27_shape=np.array(miss27.shape), links19=links19)

    print("step chains")
    from tensorlbm.d3q19 import OPPOSITE as OPP19

    def cavity_walls(n):
        wall = torch.zeros((n, n, n), dtype=torch.bool)
        wall[:, :, 0] = wall[:, :, -1] = wall[:, 0, :] = wall[0, :, :] = wall[-1, :, :] = True
        return wall

    def cavity_run(n, coll, mode, steps, tau_c, u_lid=0.05, stop_at_nan=False):
        """mode "fullway": collide -> stream -> bounce_back_cells_3d(walls) -> lid.
        mode "halfway": collide -> where(wall, f_pre[opp], f) -> stream -> lid
        (benchmarks/verified/cavity_3d_full/run.py:58 and :95-104)."""
        wall = cavity_walls(n)
        z = torch.zeros((n, n, n))
        f = equilibrium3d(torch.ones((n, n, n)), z, z, z)
        nan_step = -1
        for s in range(1, steps + 1):
            f_pre = f
            f = collide_bgk3d(f, tau_c) if coll == "bgk" else collide_mrt3d(f, tau_c)
            if mode == "halfway":
                f = torch.where(wall.unsqueeze(0), f_pre[OPP19], f)
            f = stream3d(f)
            if mode == "fullway":
                f = b3.bounce_back_cells_3d(f, wall)
            f = b3.zou_he_moving_lid_3d(f, u_lid)
            if nan_step < 0 and not bool(torch.isfinite(f).all()):
                nan_step = s
                if stop_at_nan:
                    break
        return f, wall, nan_step

    # 12^3 cavity, 150 steps: the literal full-way chain diverges (NaN) inside the
    # window for BGK and MRT; the production half-way chain stays finite
    n = 12
    tau_c = 3 * 0.05 * n / 100 + 0.5
    for coll in ("bgk", "mrt"):
        for mode in ("fullway", "halfway"):
            f, wall, nan_step = cavity_run(n, coll, mode, 150, tau_c)
            z = torch.zeros((n, n, n))
            save(f"chain_cavity_d3q19_{coll}_{mode}", f0=equilibrium3d(torch.ones((n, n, n)), z, z, z), f=f,
                 wall=wall, tau=tau_c, u_lid=0.05, steps=150, nan_step=nan_step)
        # finite window of the literal chain, compared element-wise
        f, wall, _ = cavity_run(n, coll, "fullway", 12, tau_c)
        z = torch.zeros((n, n, n))
        save(f"chain_cavity_d3q19_{coll}_fullway_window", f0=equilibrium3d(torch.ones((n, n, n)), z, z, z), f=f,
             wall=wall, tau=tau_c, u_lid=0.05, steps=12)

    # sphere channel: collide -> stream -> force -> ZH in -> ZH out -> BB(wall) -> BB(obstacle)
    nz, ny, nx = 12, 12, 24
    obst = b3.sphere_mask(nx, ny, nz, 8.0, 6.0, 6.0, 2.5, cpu)
    empty = torch.zeros_like(obst)
    u_in = 0.04
    for q, coll in ((19, "mrt"), (19, "bgk"), (27, "cumulant"), (27, "geier"), (27, "bgk")):
        ones, zz = torch.ones((nz, ny, nx)), torch.zeros((nz, ny, nx))
        ux0 = torch.full((nz, ny, nx), u_in)
        ux0[obst] = 0.0
        f = (equilibrium3d if q == 19 else equilibrium27)(ones, ux0, zz, zz)
        f0 = f.clone()
        tau_s = 3 * u_in * 5 / 30 + 0.5
        forces = []
        for _ in range(60):
            if q == 19:
                f = collide_mrt3d(f, tau_s) if coll == "mrt" else collide_bgk3d(f, tau_s)
                f = stream3d(f)
                forces.append(torch.stack(obstacles.compute_obstacle_forces_3d(f, obst)))
                f = b3.apply_zou_he_channel_boundaries_3d(f, u_in, empty, obst)
            else:
                if coll == "cumulant":
                    f = cumulant.collide_cumulant_d3q27(f, tau_s)
                elif coll == "geier":
                    f = cumulant.collide_cumulant_geier_d3q27(f, tau_s)
                else:
                    f = collide_bgk27(f, tau_s)
                f = stream27(f)
                forces.append(torch.stack(obstacles.compute_obstacle_forces_27(f, obst)))
                f = b27.apply_zou_he_channel_boundaries_27(f, u_in, empty, obst)
        save(f"chain_sphere_d3q{q}_{coll}", f0=f0, f=f, obstacle=obst, tau=tau_s, u_in=u_in, steps=60,
             forces=torch.stack(forces))

    # D2Q9 cylinder channel with walls: cylinder_flow.py:854-899 (zou_he outlet mode)
    ny2, nx2 = 16, 64
    obst2 = b2.cylinder_mask(nx2, ny2, 10.0, 8.0, 2.5, cpu)
    wall2 = b2.make_channel_wall_mask(ny2, nx2, obst2, cpu)
    ux0 = torch.full((ny2, nx2), 0.05)
    ux0[obst2] = 0.0
    f = equilibrium(torch.ones((ny2, nx2)), ux0, torch.zeros((ny2, nx2)))
    f0 = f.clone()
    tau2 = 3 * 0.05 * 5 / 20 + 0.5  # Re = u D / nu = 20
    forces = []
    for _ in range(200):
        f = collide_bgk(f, tau2)
        f = stream(f)
        forces.append(torch.stack(b2.compute_obstacle_forces(f, obst2)))
        f = b2.zou_he_inlet_velocity(f, 0.05)
        f = b2.zou_he_outlet_pressure(f, rho_out=1.0)
        f = b2.bounce_back_cells(f, wall2)
        f = b2.bounce_back_cells(f, obst2)
    save("chain_cylinder_d2q9_bgk", f0=f0, f=f, obstacle=obst2, wall=wall2, tau=tau2, u_in=0.05, steps=200,
         forces=torch.stack(forces))

    if not args.skip_long:
        # the 64^3, Re=400, lid 0.05 cavity (tau = 3 u N / Re + 0.5)
        n = 64
        tau_c = 3 * 0.05 * n / 400 + 0.5
        mid = n // 2

        def summary(f):
            rho, ux, uy, uz = macroscopic3d(f)
            return dict(rho_mid=rho[mid], ux_mid=ux[mid], uy_mid=uy[mid], uz_mid=uz[mid],
                        ux_center_line=ux[mid, :, mid], uy_center_line=uy[mid, mid, :],
                        sums=torch.stack([rho.double().sum(), ux.double().sum(), uy.double().sum(),
                                          uz.double().sum(), (ux.double() ** 2 + uy.double() ** 2
                                                              + uz.double() ** 2).sum()]),
                        f_sum_per_q=f.double().sum(dim=(1, 2, 3)))

        # literal BGK full-way chain: 20 finite steps, then the step where it turns NaN
        f, _, _ = cavity_run(n, "bgk", "fullway", 20, tau_c)
        _, _, nan_step = cavity_run(n, "bgk", "fullway", 1000, tau_c, stop_at_nan=True)
        save("chain_cavity64_d3q19_bgk_fullway", tau=tau_c, u_lid=0.05, steps=20, nan_step=nan_step, **summary(f))
        print(f"  64^3 BGK full-way cavity: NaN from step {nan_step}")
        # production half-way walls, MRT, 1000 steps (finite)
        t0 = time.time()
        f, _, nan_step = cavity_run(n, "mrt", "halfway", 1000, tau_c)
        dt = time.time() - t0
        save("chain_cavity64_d3q19_mrt_halfway_1000", tau=tau_c, u_lid=0.05, steps=1000, seconds=dt,
             nan_step=nan_step, **summary(f))
        print(f"  64^3 MRT half-way cavity, 1000 steps: {dt:.1f} s ({n**3 * 1000 / dt / 1e6:.2f} MLUPS)")


if __name__ == "__main__":
    main()
