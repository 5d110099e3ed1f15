"""Lattice-generic wrappers over the C ABI, shared by the reference-named modules.

Each function validates its tensors the way TensorLBM does (``ValueError`` for
shape / dtype, ``NotImplementedError`` for unsupported options), makes the
inputs contiguous, allocates the output with torch (plumbing only) and
enqueues the kernel on the current CUDA stream.
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib

LATTICE_DIM = {9: 2, 19: 3, 27: 3}


def grid_of(f: torch.Tensor, q: int) -> tuple[int, int, int]:
    """(nx, ny, nz) of a population tensor of lattice q."""
    dim = LATTICE_DIM[q]
    if f.ndim != dim + 1 or f.shape[0] != q:
        shape = "(9, ny, nx)" if dim == 2 else f"({q}, nz, ny, nx)"
        raise ValueError(f"f must have shape {shape}, got {tuple(f.shape)}")
    if dim == 2:
        return int(f.shape[2]), int(f.shape[1]), 1
    return int(f.shape[3]), int(f.shape[2]), int(f.shape[1])


def _c(t: torch.Tensor) -> torch.Tensor:
    return t if t.is_contiguous() else t.contiguous()


def _mask_u8(mask: torch.Tensor, spatial: tuple[int, ...]) -> torch.Tensor:
    if tuple(mask.shape) != tuple(spatial):
        raise ValueError(f"mask shape {tuple(mask.shape)} does not match the grid {tuple(spatial)}")
    if mask.dtype == torch.bool:
        return _c(mask).view(torch.uint8)
    if mask.dtype in (torch.uint8, torch.int8):
        return _c(mask.to(torch.uint8))
    return _c(mask != 0).view(torch.uint8)


# ---------------------------------------------------------------------------
# moments
# ---------------------------------------------------------------------------


def equilibrium(q: int, rho, ux, uy, uz=None, out: torch.Tensor | None = None) -> torch.Tensor:
    fields = (rho, ux, uy) if q == 9 else (rho, ux, uy, uz)
    if any(t is None for t in fields):
        raise ValueError("equilibrium needs rho and every velocity component")
    shapes = {tuple(t.shape) for t in fields}
    if len(shapes) != 1:
        names = "rho, ux, and uy" if q == 9 else "rho, ux, uy, and uz"
        raise ValueError(f"{names} shapes must match: " + ", ".join(str(tuple(t.shape)) for t in fields))
    dev = _lib.require_cuda(*fields)
    dtype = rho.dtype
    if any(t.dtype != dtype for t in fields):
        raise ValueError("rho and velocity fields must share one dtype")
    code = _lib.real_dtype(rho)
    fields = [_c(t) for t in fields]
    n = fields[0].numel()
    res = torch.empty((q,) + tuple(rho.shape), dtype=dtype, device=dev)
    if n > 0:
        lib = _lib.load()
        st = lib.tlbm_equilibrium(q, code, n, *[t.data_ptr() for t in fields[:3]],
                                  fields[3].data_ptr() if q != 9 else None, res.data_ptr(), _lib.stream_of(dev))
        _lib.check(st, "equilibrium")
    if out is not None:
        out.copy_(res)
        return out
    return res


def macroscopic(q: int, f: torch.Tensor):
    dev = _lib.require_cuda(f)
    if f.shape[0] != q:
        raise ValueError(f"f must have {q} populations on dim 0, got shape {tuple(f.shape)}")
    code = _lib.real_dtype(f)
    f = _c(f)
    spatial = tuple(f.shape[1:])
    outs = [torch.empty(spatial, dtype=f.dtype, device=dev) for _ in range(3 if q == 9 else 4)]
    n = outs[0].numel()
    if n > 0:
        st = _lib.load().tlbm_macroscopic(q, code, n, f.data_ptr(), *[o.data_ptr() for o in outs[:3]],
                                          outs[3].data_ptr() if q != 9 else None, _lib.stream_of(dev))
        _lib.check(st, "macroscopic")
    return tuple(outs)


# ---------------------------------------------------------------------------
# collisions and streaming
# ---------------------------------------------------------------------------


def make_desc(q: int, grid: tuple[int, int, int], dtype_code: int, collision: int, tau: float, *,
              s_e: float = 0.0, s_eps: float = 0.0, s_q: float = 0.0, s_pi: float | None = None,
              omega_b: float = 1.0, omega_odd: float = 1.0, omega_even: float = 1.0, c_smag: float = 0.0,
              bc: int = 0, u_lid: float = 0.0, u_in=(0.0, 0.0, 0.0), rho_out: float = 1.0,
              lambda_trt: float = 3.0 / 16.0, cm_s5: float | None = None, cm_s6: float | None = None) -> _lib.Desc:
    d = _lib.Desc()
    d.lattice = q
    d.dtype = dtype_code
    d.collision = collision
    d.nx, d.ny, d.nz = grid
    d.bc = bc
    d.tau = float(tau)
    d.s_e, d.s_eps, d.s_q = float(s_e), float(s_eps), float(s_q)
    d.s_pi = -1.0 if s_pi is None else float(s_pi)
    d.omega_b, d.omega_odd, d.omega_even = float(omega_b), float(omega_odd), float(omega_even)
    d.c_smag = float(c_smag)
    d.u_lid = float(u_lid)
    d.u_in[0], d.u_in[1], d.u_in[2] = (float(v) for v in u_in)
    d.rho_out = float(rho_out)
    d.lambda_trt = float(lambda_trt)
    d.cm_s5 = -1.0 if cm_s5 is None else float(cm_s5)
    d.cm_s6 = -1.0 if cm_s6 is None else float(cm_s6)
    return d


def collide(q: int, f: torch.Tensor, collision: int, tau: float, *, tau_field: torch.Tensor | None = None,
            out: torch.Tensor | None = None, **rates) -> torch.Tensor:
    dev = _lib.require_cuda(f, tau_field)
    grid = grid_of(f, q)
    code = _lib.real_dtype(f)
    f = _c(f)
    tf = None
    if tau_field is not None:
        if tuple(tau_field.shape) != tuple(f.shape[1:]):
            raise ValueError(f"tau_field shape {tuple(tau_field.shape)} does not match the grid {tuple(f.shape[1:])}")
        tf = _c(tau_field.to(torch.float32))
    res = torch.empty_like(f) if out is None else out
    if f.numel() > 0:
        d = make_desc(q, grid, code, collision, tau, **rates)
        st = _lib.load().tlbm_collide(ctypes.byref(d), code, f.data_ptr(), res.data_ptr(), None, _lib.ptr(tf),
                                      _lib.stream_of(dev))
        _lib.check(st, "collide")
    return res


def stream(q: int, f: torch.Tensor) -> torch.Tensor:
    dev = _lib.require_cuda(f)
    nx, ny, nz = grid_of(f, q)
    code = _lib.real_dtype(f)
    f = _c(f)
    out = torch.empty_like(f)
    if f.numel() > 0:
        st = _lib.load().tlbm_stream(q, code, nx, ny, nz, f.data_ptr(), out.data_ptr(), _lib.stream_of(dev))
        _lib.check(st, "stream")
    return out


def correct_mass(f: torch.Tensor, target_mass: float) -> torch.Tensor:
    dev = _lib.require_cuda(f)
    code = _lib.real_dtype(f)
    f = _c(f)
    out = torch.empty_like(f)
    scratch = torch.empty(1, dtype=torch.float64, device=dev)
    if f.numel() > 0:
        st = _lib.load().tlbm_correct_mass(code, f.numel(), f.data_ptr(), out.data_ptr(), float(target_mass),
                                           scratch.data_ptr(), _lib.stream_of(dev))
        _lib.check(st, "correct_mass")
    return out


# ---------------------------------------------------------------------------
# boundaries
# ---------------------------------------------------------------------------


def bounce_back(q: int, f: torch.Tensor, mask: torch.Tensor) -> torch.Tensor:
    dev = _lib.require_cuda(f, mask)
    grid_of(f, q)
    code = _lib.real_dtype(f)
    f = _c(f)
    m = _mask_u8(mask, tuple(f.shape[1:]))
    out = torch.empty_like(f)
    n = m.numel()
    if n > 0:
        st = _lib.load().tlbm_bounce_back(q, code, n, f.data_ptr(), m.data_ptr(), out.data_ptr(),
                                          _lib.stream_of(dev))
        _lib.check(st, "bounce_back")
    return out


def moving_wall_bounce_back(q: int, f: torch.Tensor, mask: torch.Tensor, *wall_u: torch.Tensor) -> torch.Tensor:
    """Ladd moving-wall bounce-back (out of place); wall_u = (ux_w, uy_w[, uz_w])."""
    dev = _lib.require_cuda(f, mask, *wall_u)
    grid_of(f, q)
    code = _lib.real_dtype(f)
    dim = 2 if q == 9 else 3
    if len(wall_u) != dim:
        raise ValueError(f"moving_wall_bounce_back on Q={q} needs {dim} wall-velocity fields")
    f = _c(f)
    shape = tuple(f.shape[1:])
    m = _mask_u8(mask, shape)
    for u in wall_u:
        if tuple(u.shape) != shape:
            raise ValueError(f"wall velocity shape {tuple(u.shape)} != grid {shape}")
    uw = torch.stack([u.to(f.dtype) for u in wall_u]).contiguous()
    out = torch.empty_like(f)
    n = m.numel()
    if n > 0:
        st = _lib.load().tlbm_moving_wall_bounce_back(q, code, n, f.data_ptr(), m.data_ptr(), uw.data_ptr(),
                                                      out.data_ptr(), _lib.stream_of(dev))
        _lib.check(st, "moving_wall_bounce_back")
    return out


def zou_he_inlet_(q: int, f: torch.Tensor, u_in, uy_in=0.0, uz_in=0.0) -> torch.Tensor:
    """In place on f (which must be contiguous)."""
    dev = _lib.require_cuda(f)
    nx, ny, nz = grid_of(f, q)
    code = _lib.real_dtype(f)
    if not f.is_contiguous():
        raise ValueError("zou_he inlet works in place and needs a contiguous f")
    prof = [None, None]
    scal = [0.0, 0.0]
    for i, v in enumerate((u_in, uy_in)):
        if isinstance(v, torch.Tensor):
            if q != 9:
                raise NotImplementedError("per-row inlet profiles are a D2Q9 feature")
            t = v.to(device=dev, dtype=f.dtype)
            if t.ndim == 0:
                scal[i] = float(t.item())
                continue
            if t.ndim == 2 and t.shape[1] == 1:
                t = t[:, 0]
            if tuple(t.shape) != (ny,):
                raise ValueError(f"Inlet profile must have shape {(ny,)}, got {tuple(t.shape)}")
            prof[i] = _c(t)
        else:
            scal[i] = float(v)
    if prof[0] is None and prof[1] is not None:
        prof[0] = torch.full((ny,), scal[0], dtype=f.dtype, device=dev)
    st = _lib.load().tlbm_zou_he_inlet(q, code, nx, ny, nz, f.data_ptr(), scal[0], scal[1], float(uz_in),
                                       _lib.ptr(prof[0]), _lib.ptr(prof[1]), _lib.stream_of(dev))
    _lib.check(st, "zou_he_inlet_velocity")
    return f


def zou_he_outlet_(q: int, f: torch.Tensor, rho_out: float = 1.0) -> torch.Tensor:
    dev = _lib.require_cuda(f)
    nx, ny, nz = grid_of(f, q)
    code = _lib.real_dtype(f)
    if not f.is_contiguous():
        raise ValueError("zou_he outlet works in place and needs a contiguous f")
    st = _lib.load().tlbm_zou_he_outlet(q, code, nx, ny, nz, f.data_ptr(), float(rho_out), _lib.stream_of(dev))
    _lib.check(st, "zou_he_outlet_pressure")
    return f


def moving_lid_(q: int, f: torch.Tensor, u_lid: float) -> torch.Tensor:
    dev = _lib.require_cuda(f)
    nx, ny, nz = grid_of(f, q)
    code = _lib.real_dtype(f)
    if not f.is_contiguous():
        raise ValueError("moving lid works in place and needs a contiguous f")
    st = _lib.load().tlbm_moving_lid(q, code, nx, ny, nz, f.data_ptr(), float(u_lid), _lib.stream_of(dev))
    _lib.check(st, "zou_he_moving_lid")
    return f


def far_field_(q: int, f: torch.Tensor, ux: float, uy: float = 0.0, uz: float = 0.0,
               z_faces: bool = True) -> torch.Tensor:
    """Free-stream far field in place: inlet and lateral planes feq(1, u),
    zero-gradient outlet (boundaries.py:199, boundaries3d.py:446, boundaries_d3q27.py:63)."""
    dev = _lib.require_cuda(f)
    nx, ny, nz = grid_of(f, q)
    code = _lib.real_dtype(f)
    if not f.is_contiguous():
        raise ValueError("the far field works in place and needs a contiguous f")
    st = _lib.load().tlbm_far_field(q, code, nx, ny, nz, f.data_ptr(), float(ux), float(uy), float(uz),
                                    int(bool(z_faces)), _lib.stream_of(dev))
    _lib.check(st, "far_field_bc")
    return f


def obstacle_force(q: int, f: torch.Tensor, mask: torch.Tensor) -> torch.Tensor:
    """(3,) float64 tensor 2 * sum_mask sum_q c_q f_q."""
    dev = _lib.require_cuda(f, mask)
    grid_of(f, q)
    code = _lib.real_dtype(f)
    f = _c(f)
    m = _mask_u8(mask, tuple(f.shape[1:]))
    out = torch.zeros(3, dtype=torch.float64, device=dev)
    if m.numel() > 0:
        st = _lib.load().tlbm_obstacle_force(q, code, m.numel(), f.data_ptr(), m.data_ptr(), out.data_ptr(),
                                             _lib.stream_of(dev))
        _lib.check(st, "compute_obstacle_forces")
    return out


def moment_sums(q: int, f: torch.Tensor, storage_code: int | None = None) -> torch.Tensor:
    """(4,) float64: total mass and momentum of a population tensor."""
    dev = _lib.require_cuda(f)
    code = storage_code if storage_code is not None else _lib.real_dtype(f)
    f = _c(f)
    n = f[0].numel()
    out = torch.zeros(4, dtype=torch.float64, device=dev)
    if n > 0:
        st = _lib.load().tlbm_moment_sums(q, code, n, f.data_ptr(), out.data_ptr(), _lib.stream_of(dev))
        _lib.check(st, "moment_sums")
    return out


# ---------------------------------------------------------------------------
# masks and links
# ---------------------------------------------------------------------------


def cuda_device(device) -> torch.device:
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if dev.type != "cuda":
        raise RuntimeError(f"tensorlbm_b200 builds masks on CUDA devices only; got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


def sphere_mask(nx, ny, nz, cx, cy, cz, radius, device) -> torch.Tensor:
    dev = cuda_device(device)
    out = torch.empty((nz, ny, nx), dtype=torch.uint8, device=dev)
    if out.numel() > 0:
        st = _lib.load().tlbm_sphere_mask(nx, ny, nz, float(cx), float(cy), float(cz), float(radius),
                                          out.data_ptr(), _lib.stream_of(dev))
        _lib.check(st, "sphere_mask")
    return out.view(torch.bool)


def cylinder_mask(nx, ny, cx, cy, radius, device) -> torch.Tensor:
    dev = cuda_device(device)
    out = torch.empty((ny, nx), dtype=torch.uint8, device=dev)
    if out.numel() > 0:
        st = _lib.load().tlbm_cylinder_mask(nx, ny, float(cx), float(cy), float(radius), out.data_ptr(),
                                            _lib.stream_of(dev))
        _lib.check(st, "cylinder_mask")
    return out.view(torch.bool)


def build_flags(spatial, device, wall=None, obstacle=None, wall_mode: str = "fullway") -> torch.Tensor:
    """Flag byte per cell.  wall_mode "fullway": walls bounce back after the
    pull (bounce_back_cells*); "halfway": walls are reversed before streaming
    and not collided (cases/base.py pre-boundaries)."""
    if wall_mode not in ("fullway", "halfway"):
        raise ValueError(f"wall_mode must be 'fullway' or 'halfway', got {wall_mode!r}")
    dev = cuda_device(device)
    w = None if wall is None else _mask_u8(wall.to(dev), spatial)
    o = None if obstacle is None else _mask_u8(obstacle.to(dev), spatial)
    flags = torch.empty(spatial, dtype=torch.uint8, device=dev)
    wall_flag = _lib.FLAG_HALFWAY if wall_mode == "halfway" else _lib.FLAG_SOLID
    if flags.numel() > 0:
        st = _lib.load().tlbm_build_flags(flags.numel(), _lib.ptr(w), _lib.ptr(o), wall_flag, flags.data_ptr(),
                                          _lib.stream_of(dev))
        _lib.check(st, "build_flags")
    return flags


def missing_mask(q: int, grid: tuple[int, int, int], solid: torch.Tensor | None, periodic_bits: int,
                 device) -> torch.Tensor:
    dev = cuda_device(device)
    nx, ny, nz = grid
    spatial = (ny, nx) if q == 9 else (nz, ny, nx)
    s = None if solid is None else _mask_u8(solid, spatial)
    out = torch.empty((q,) + spatial, dtype=torch.uint8, device=dev)
    st = _lib.load().tlbm_missing_mask(q, nx, ny, nz, _lib.ptr(s), periodic_bits, out.data_ptr(),
                                       _lib.stream_of(dev))
    _lib.check(st, "derive_missing_mask")
    return out.view(torch.bool)


def link_list(mask: torch.Tensor) -> torch.Tensor:
    """Flat indices (int64, increasing) of the non-zero entries of a byte mask.

    Reads the count back to size the output, the one host synchronisation of
    the mask builder (torch.nonzero synchronises for the same reason)."""
    dev = _lib.require_cuda(mask)
    m = _c(mask).view(torch.uint8).reshape(-1) if mask.dtype == torch.bool else _c(mask.to(torch.uint8)).reshape(-1)
    lib = _lib.load()
    count = m.numel()
    nb = lib.tlbm_link_blocks(count)
    blocks = torch.empty(max(nb, 1), dtype=torch.int64, device=dev)
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    s = _lib.stream_of(dev)
    _lib.check(lib.tlbm_link_count(m.data_ptr(), count, blocks.data_ptr(), total.data_ptr(), s), "link_count")
    n = int(total.item())
    out = torch.empty(n, dtype=torch.int64, device=dev)
    if n > 0:
        _lib.check(lib.tlbm_link_list(m.data_ptr(), count, blocks.data_ptr(), out.data_ptr(), s), "link_list")
    return out
