"""Time-step drivers: the "solvers' step()" of TensorLBM on the fused kernel.

Three entry points, all running the sm_100a kernels through the C ABI:

* :class:`LBMSolver` - stateful, one fused kernel per step (the fast path).
  TensorLBM's runners advance ``S_{n+1} = BC(stream(collide(S_n)))``
  (``cases/base.py:270-289``, ``d3q27_sphere_flow.py:246-256``).  The fused
  kernel pulls, applies the boundaries and collides in one pass, so what it
  stores is the post-collision state ``P_n = collide(S_n)``.  The solver keeps
  the previous buffer, so ``solver.f`` returns the TensorLBM-phase ``S_n``
  with one extra pass (boundaries without collision) whenever it is asked for.
* :func:`make_step` - the functional ``step(f) -> f`` closure of
  ``CaseBase.make_step`` with TensorLBM's phase on both sides: a collision
  pass followed by a pull + boundary pass (two passes per step).
* :class:`FusedSolver3D` - same surface as ``TritonFusedSolver3D``
  (``triton_fused.py:676-865``): periodic D3Q19 BGK, ``step(f)`` returns
  ``collide(stream(f))`` in one of two persistent ping-pong buffers.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import torch

from . import _lib, _ops

COLLISIONS = {
    "none": _lib.COLL_NONE,
    "bgk": _lib.COLL_BGK,
    "mrt": _lib.COLL_MRT,
    "cumulant": _lib.COLL_CUMULANT,
    "cumulant_geier": _lib.COLL_CUMULANT_GEIER,
    "cumulant_d3q19": _lib.COLL_CUMULANT_D3Q19,
    "smagorinsky": _lib.COLL_SMAGORINSKY,
    "trt": _lib.COLL_TRT,
    "cascaded": _lib.COLL_CASCADED,
    "rlbm": _lib.COLL_RLBM,
}
_LATTICES = {"D2Q9": 9, "D3Q19": 19, "D3Q27": 27, 9: 9, 19: 19, 27: 27}
# storage dtype -> (C code, torch dtype of the buffer)
STORAGE = {
    "f32": (_lib.F32, torch.float32),
    "f64": (_lib.F64, torch.float64),
    "f16": (_lib.F16_SHIFTED, torch.float16),
    "bf16": (_lib.BF16_SHIFTED, torch.bfloat16),
}
_TORCH_STORAGE = {torch.float32: "f32", torch.float64: "f64", torch.float16: "f16", torch.bfloat16: "bf16"}

# default relaxation rates per lattice (solver.py:249, solver3d.py:107, d3q27.py:643)
_MRT_DEFAULTS = {9: (1.64, 1.54, 1.7), 19: (1.19, 1.4, 1.2), 27: (1.19, 1.4, 1.2)}


@dataclass
class StepConfig:
    """Everything one fused step needs besides the buffers."""

    lattice: int
    shape: tuple[int, ...]          # (ny, nx) or (nz, ny, nx)
    tau: float
    collision: str = "bgk"
    s_e: float | None = None
    s_eps: float | None = None
    s_q: float | None = None
    s_pi: float | None = None
    omega_b: float = 1.0
    omega_odd: float = 1.0
    omega_even: float = 1.0
    c_smag: float = 0.0
    u_lid: float | None = None       # moving lid at y = ny-1
    u_in: tuple[float, float, float] | float | None = None  # Zou/He inlet at x = 0
    rho_out: float | None = None     # Zou/He outlet at x = nx-1
    force_lin: float = 0.0           # linear body force F = A rho u (BGK / MRT / Smagorinsky, float32)
    lambda_trt: float = 3.0 / 16.0   # TRT magic parameter (solver.py:440)
    cm_s5: float | None = None       # cascaded D3Q27 5th / 6th-order rates (None: omega_even)
    cm_s6: float | None = None
    # free-stream far field at velocity u_in (boundaries.py:199, boundaries3d.py:446,
    # boundaries_d3q27.py:63): None, "y" (inlet, outlet and the y planes) or "yz"
    # (3-D: the z planes too, the reference's default)
    far_field: str | None = None
    inlet_du: tuple[float, float, float] = (0.0, 0.0, 0.0)  # far field: extra velocity of the x = 0 plane
    extra: dict = field(default_factory=dict)

    @property
    def grid(self) -> tuple[int, int, int]:
        if self.lattice == 9:
            ny, nx = self.shape
            return nx, ny, 1
        nz, ny, nx = self.shape
        return nx, ny, nz

    def desc(self, dtype_code: int, collision: str | None = None) -> _lib.Desc:
        q = self.lattice
        d_se, d_seps, d_sq = _MRT_DEFAULTS[q]
        bc = 0
        u_in = (0.0, 0.0, 0.0)
        if self.u_lid is not None:
            bc |= _lib.BC_LID
        if self.u_in is not None:
            u_in = (float(self.u_in), 0.0, 0.0) if isinstance(self.u_in, (int, float)) else tuple(self.u_in)
            if self.far_field is None:
                bc |= _lib.BC_ZH_INLET
        if self.far_field is not None:
            if self.far_field not in ("y", "yz") or (self.far_field == "yz" and q == 9):
                allowed = "'y'" if q == 9 else "'y' or 'yz'"
                raise ValueError(f"far_field must be {allowed}, got {self.far_field!r}")
            if self.u_in is None or self.rho_out is not None:
                raise ValueError("the far field takes u_in (its free-stream velocity) and no Zou/He rho_out")
            bc |= _lib.BC_FAR_FIELD | (_lib.BC_FAR_FIELD_Z if self.far_field == "yz" else 0)
        if self.rho_out is not None:
            bc |= _lib.BC_ZH_OUTLET
        coll = COLLISIONS[collision or self.collision]
        d = _ops.make_desc(
            q, self.grid, dtype_code, coll, self.tau,
            s_e=d_se if self.s_e is None else self.s_e,
            s_eps=d_seps if self.s_eps is None else self.s_eps,
            s_q=d_sq if self.s_q is None else self.s_q,
            s_pi=self.s_pi, omega_b=self.omega_b, omega_odd=self.omega_odd, omega_even=self.omega_even,
            c_smag=self.c_smag, bc=bc, u_lid=self.u_lid or 0.0, u_in=u_in,
            rho_out=1.0 if self.rho_out is None else self.rho_out, lambda_trt=self.lambda_trt,
            cm_s5=self.cm_s5, cm_s6=self.cm_s6,
        )
        d.ff_inlet_du[0], d.ff_inlet_du[1], d.ff_inlet_du[2] = (float(v) for v in self.inlet_du)
        if coll in (_lib.COLL_BGK, _lib.COLL_MRT, _lib.COLL_SMAGORINSKY):
            d.force_lin = float(self.force_lin)
        elif self.force_lin and coll != _lib.COLL_NONE:
            raise NotImplementedError("force_lin is implemented for the bgk, mrt and smagorinsky collisions")
        return d


class LBMSolver:
    """Fused single-GPU LBM time stepper (one kernel pass per step).

    Args:
        lattice: "D2Q9", "D3Q19" or "D3Q27" (or 9 / 19 / 27).
        shape: (ny, nx) or (nz, ny, nx).
        tau: shear relaxation time.
        collision: "bgk", "mrt", "trt" (tau = tau_plus, ``lambda_trt=`` the magic
            parameter), "smagorinsky", "cumulant" (D3Q27 legacy),
            "cumulant_geier" (D3Q27), "cumulant_d3q19", "cascaded" (D3Q19 / D3Q27;
            ``omega_b``, ``omega_odd``, ``omega_even``, ``cm_s5``, ``cm_s6`` are
            s_bulk, s_3, s_4, s_5, s_6).
        storage: "f32", "f64", "f16" or "bf16" (half formats hold the deviation f - w,
            scaled by 2^14 for f16, stochastically rounded).
        wall_mask, obstacle_mask: bool fields; both bounce back, only the
            obstacle enters the momentum-exchange force.
        u_lid, u_in, rho_out: enable the lid / Zou-He inlet / outlet planes.
        far_field: "y" or "yz" (3-D) with u_in: the free-stream far field of
            far_field_bc_2d / far_field_bc_3d / far_field_bc_27 instead of Zou/He;
            ``set_inlet_perturbation`` seeds the inlet plane.
        tau_field: optional per-cell tau (BGK and MRT shear rate).
        track_force: record the float64 force of every step.
        curved_wall: a :class:`tensorlbm_b200.bfl.CurvedWall` (Bouzidi links of a
            curved obstacle, D3Q19 / D3Q27); its force is the BFL ledger.
    """

    def __init__(self, lattice, shape, tau: float, collision: str = "bgk", *, device=None, storage="f32",
                 wall_mask=None, obstacle_mask=None, wall_mode: str = "fullway", tau_field=None,
                 track_force: bool = False, wall_velocity=None, curved_wall=None, pattern: str = "ab", **cfg):
        q = _LATTICES[lattice]
        if isinstance(storage, torch.dtype):
            storage = _TORCH_STORAGE[storage]
        if storage not in STORAGE:
            raise ValueError(f"unknown storage {storage!r}; expected one of {sorted(STORAGE)}")
        if collision not in COLLISIONS:
            raise ValueError(f"unknown collision {collision!r}; expected one of {sorted(COLLISIONS)}")
        shape = tuple(int(s) for s in shape)
        if len(shape) != (2 if q == 9 else 3):
            raise ValueError(f"shape {shape} does not fit lattice D{'2' if q == 9 else '3'}Q{q}")
        self.cfg = StepConfig(q, shape, float(tau), collision, **cfg)
        self.device = _ops.cuda_device(device)
        self.q = q
        self.storage = storage
        self.code, self.buf_dtype = STORAGE[storage]
        self.compute_dtype = torch.float64 if storage == "f64" else torch.float32
        self.flags = None
        if wall_mask is not None or obstacle_mask is not None:
            self.flags = _ops.build_flags(shape, self.device, wall_mask, obstacle_mask, wall_mode)
        self.wall_u = None
        if wall_velocity is not None:
            # the obstacle becomes a Ladd moving wall with this velocity field
            if obstacle_mask is None:
                raise ValueError("wall_velocity needs an obstacle_mask (the moving surface)")
            if len(wall_velocity) != len(shape) or any(tuple(u.shape) != shape for u in wall_velocity):
                raise ValueError(f"wall_velocity must be {len(shape)} fields of shape {shape}")
            moving = _ops._mask_u8(obstacle_mask.to(self.device), shape)
            self.flags.bitwise_or_(moving * _lib.FLAG_MOVING)
            self.wall_u = torch.stack([u.to(device=self.device, dtype=self.compute_dtype)
                                       for u in wall_velocity]).contiguous()
        self.curved = None
        if curved_wall is not None:
            # Bouzidi links: solid cells bounce back full-way (not in the drag),
            # the cells with links take the interpolated update; the drag of
            # the wall is the BFL ledger
            if q == 9:
                raise NotImplementedError("curved walls are built for D3Q19 and D3Q27")
            if curved_wall.q != q or tuple(curved_wall.solid.shape) != shape:
                raise ValueError(f"curved_wall is for Q={curved_wall.q} {tuple(curved_wall.solid.shape)}, "
                                 f"the solver is Q={q} {shape}")
            if self.flags is None:
                self.flags = torch.zeros(shape, dtype=torch.uint8, device=self.device)
            solid = curved_wall.solid.to(self.device)
            self.flags.bitwise_or_(solid.to(torch.uint8) * _lib.FLAG_SOLID)
            self.flags.bitwise_or_(curved_wall.cells.to(self.device).to(torch.uint8) * _lib.FLAG_CURVED)
            self.curved = curved_wall
        self.tau_field = None
        if tau_field is not None:
            if tuple(tau_field.shape) != shape:
                raise ValueError(f"tau_field shape {tuple(tau_field.shape)} != {shape}")
            self.tau_field = tau_field.to(device=self.device, dtype=torch.float32).contiguous()
        self.track_force = track_force
        full = (q,) + shape
        if pattern not in ("ab", "aa"):
            raise ValueError(f"pattern must be 'ab' (two buffers) or 'aa' (one buffer, in place), got {pattern!r}")
        if pattern == "aa" and (self.curved is not None or storage == "f64" or self.wall_u is not None or
                                self.cfg.far_field is not None):
            raise NotImplementedError("the AA pattern supports f32 / f16 / bf16 storage without curved or "
                                      "moving walls or the far field")
        self.pattern = pattern
        # two buffers (index of the current one in _cur), or one AA buffer
        # (its layout in _cur: 0 swapped, 1 natural)
        self._buf = [torch.empty(full, dtype=self.buf_dtype, device=self.device)
                     for _ in range(1 if pattern == "aa" else 2)]
        self._cur = 0
        self.steps_done = 0
        self.step_offset = 0          # steps completed before the last load()/resume()
        self._f0: torch.Tensor | None = None
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.forces: list[torch.Tensor] = []
        self._desc = self._attach(self.cfg.desc(self.code))
        self._desc_none = self._attach(self.cfg.desc(self.code, "none"))
        self._graph = None

    def _attach(self, d: _lib.Desc) -> _lib.Desc:
        """Per-cell tables of the solver on a descriptor (moving-wall velocity, Bouzidi links)."""
        if self.wall_u is not None:
            d.wall_velocity = self.wall_u.data_ptr()
        if self.curved is not None:
            self.curved.attach(d)
        return d

    # -- state -----------------------------------------------------------------

    @property
    def n_cells(self) -> int:
        n = 1
        for s in self.cfg.shape:
            n *= s
        return n

    def _stream(self) -> int:
        return _lib.stream_of(self.device)

    def load(self, f: torch.Tensor) -> "LBMSolver":
        """Set the state to a TensorLBM-phase population field S_0."""
        if tuple(f.shape) != (self.q,) + self.cfg.shape:
            raise ValueError(f"f shape {tuple(f.shape)} != {(self.q,) + self.cfg.shape}")
        f = f.to(device=self.device, dtype=self.compute_dtype).contiguous()
        self._f0 = f.clone()
        lib = _lib.load()
        dc = self.cfg.desc(_lib.F64 if self.storage == "f64" else _lib.F32)
        if self.pattern == "aa":
            da = self._attach(self.cfg.desc(self.code))
            _lib.check(lib.tlbm_aa_load(ctypes.byref(da), f.data_ptr(), self._buf[0].data_ptr(), _lib.ptr(self.flags),
                                        _lib.ptr(self.tau_field), self._stream()), "aa_load")
        elif self.storage in ("f32", "f64"):
            _lib.check(lib.tlbm_collide(ctypes.byref(dc), dc.dtype, f.data_ptr(), self._buf[0].data_ptr(), _lib.ptr(self.flags),
                                        _lib.ptr(self.tau_field), self._stream()), "collide")
        else:
            tmp = torch.empty_like(f)
            _lib.check(lib.tlbm_collide(ctypes.byref(dc), _lib.F32, f.data_ptr(), tmp.data_ptr(), _lib.ptr(self.flags),
                                        _lib.ptr(self.tau_field), self._stream()), "collide")
            conv = self.cfg.desc(_lib.F32, "none")
            _lib.check(lib.tlbm_collide(ctypes.byref(conv), self.code, tmp.data_ptr(), self._buf[0].data_ptr(), None,
                                        None, self._stream()), "convert")
        self._cur = 2 if self.pattern == "aa" else 0   # AA: the loaded layout
        self.steps_done = 0
        self.step_offset = 0
        self.forces = []
        self._graph = None
        return self

    def resume(self, populations: torch.Tensor, *, step: int = 0, stored_state: torch.Tensor | None = None,
               aa_layout: int | None = None) -> "LBMSolver":
        """Continue a run from a checkpoint.

        populations: the TensorLBM-phase field S_n (what ``f`` returned when it
        was saved); step: the completed step count n.  With ``stored_state``
        (this solver's own stored P_n in the same storage format, from
        ``state``) the continuation is bit-exact for every storage format;
        without it the state is rebuilt as collide(S_n), which is exactly P_n
        for float32 / float64 storage and a fresh stochastic rounding of it for
        FP16 / BF16."""
        self.load(populations)
        if stored_state is not None:
            buf = self._buf[0]
            if tuple(stored_state.shape) != tuple(buf.shape) or stored_state.dtype != buf.dtype:
                raise ValueError(f"stored_state {tuple(stored_state.shape)} {stored_state.dtype} does not match "
                                 f"this solver's {tuple(buf.shape)} {buf.dtype} ({self.storage} storage)")
            buf.copy_(stored_state.to(self.device))
            if self.pattern == "aa":
                if aa_layout not in (0, 1, 2):
                    raise ValueError("an AA stored state needs its layout (0 swapped, 1 natural, 2 loaded)")
                self._cur = int(aa_layout)
        self.step_offset = int(step)
        return self

    @property
    def step_index(self) -> int:
        """Completed steps, including those before the last load()/resume()."""
        return self.step_offset + self.steps_done

    def _launch(self, src: torch.Tensor, dst: torch.Tensor, force: torch.Tensor | None) -> None:
        st = _lib.load().tlbm_step(ctypes.byref(self._desc), src.data_ptr(), dst.data_ptr(), _lib.ptr(self.flags),
                                   _lib.ptr(self.tau_field), _lib.ptr(force), self.status.data_ptr(),
                                   self._stream())
        _lib.check(st, "tlbm_step")

    def _launch_parity(self, c: int, force: torch.Tensor | None) -> None:
        """One step from parity c: the current buffer (two buffers) or the layout (AA)."""
        if self.pattern == "aa":
            st = _lib.load().tlbm_step_aa(ctypes.byref(self._desc), self._buf[0].data_ptr(), c, _lib.ptr(self.flags),
                                          _lib.ptr(self.tau_field), _lib.ptr(force), self.status.data_ptr(),
                                          self._stream())
            _lib.check(st, "tlbm_step_aa")
        else:
            self._launch(self._buf[c], self._buf[1 - c], force)

    def step(self, n: int = 1) -> "LBMSolver":
        """Advance n time steps (n fused kernel launches)."""
        if self._f0 is None:
            raise RuntimeError("LBMSolver.step() before load(f)")
        for _ in range(n):
            force = None
            if self.track_force:
                force = torch.zeros(3, dtype=torch.float64, device=self.device)
                self.forces.append(force)
            self._launch_parity(self._cur, force)
            self._cur = self._next_parity(self._cur)
            self.steps_done += 1
        return self

    def _next_parity(self, c: int) -> int:
        if self.pattern == "aa":
            return 1 if c == 0 else 0   # loaded / natural -> swapped, swapped -> natural
        return c ^ 1

    def set_inlet_perturbation(self, dux: float = 0.0, duy: float = 0.0, duz: float = 0.0) -> "LBMSolver":
        """Far field: the x = 0 plane takes feq(1, u_in + (dux, duy, duz)) from the
        next step on, as benchmarks/verified/cylinder seeds its wake (drops the
        captured graph)."""
        if self.cfg.far_field is None:
            raise ValueError("the inlet perturbation belongs to the far field (far_field='y' or 'yz')")
        self.cfg.inlet_du = (float(dux), float(duy), float(duz))
        self._desc = self._attach(self.cfg.desc(self.code))
        self._graph = None
        return self

    def set_force_lin(self, a: float) -> "LBMSolver":
        """Change the linear body force A of F = A rho u (drops the captured graph)."""
        self.cfg.force_lin = float(a)
        self._desc = self._attach(self.cfg.desc(self.code))
        self._graph = None
        return self

    def run(self, n: int, *, graph: bool = True, chunk: int = 50) -> "LBMSolver":
        """Advance n steps, replaying a CUDA graph of `chunk` launches when graph=True.

        Force tracking records one force per step, so it runs eagerly."""
        if not graph or self.track_force or n < chunk:
            return self.step(n)
        if self.pattern == "aa" and self._cur == 2:
            # leave the loaded layout eagerly: the graph then cycles swapped <-> natural
            self.step(1)
            n -= 1
        if self._graph is None or self._graph[1] != chunk or self._graph[2] != self._cur:
            # capture `chunk` (even) steps starting from the current buffer parity
            chunk = chunk + (chunk & 1)
            cur0 = self._cur
            s = torch.cuda.Stream(self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    c = cur0
                    for _ in range(chunk):
                        self._launch_parity(c, None)
                        c = self._next_parity(c)
            torch.cuda.current_stream(self.device).wait_stream(s)
            self._graph = (g, chunk, cur0)
        g, chunk, _ = self._graph
        reps, rest = divmod(n, chunk)
        for _ in range(reps):
            g.replay()
        self.steps_done += reps * chunk
        if rest:
            self.step(rest)
        return self

    @property
    def state(self) -> torch.Tensor:
        """Stored post-collision populations P_n (storage format: (f - w) 2^14 for f16, f - w for bf16);
        for the AA pattern the raw buffer, in the layout ``aa_layout``."""
        return self._buf[0] if self.pattern == "aa" else self._buf[self._cur]

    @property
    def aa_layout(self) -> int | None:
        """AA pattern: 0 swapped (post-collision), 1 natural (streamed, not yet bounded),
        2 loaded (S_0 as loaded); None for two buffers."""
        return self._cur if self.pattern == "aa" else None

    @property
    def f(self) -> torch.Tensor:
        """TensorLBM-phase populations S_n = BC(stream(P_{n-1})) as float32/float64."""
        if self._f0 is None:
            raise RuntimeError("LBMSolver.f before load(f)")
        if self.steps_done == 0:
            return self._f0.clone()
        out = torch.empty((self.q,) + self.cfg.shape, dtype=self.compute_dtype, device=self.device)
        if self.pattern == "aa":
            st = _lib.load().tlbm_aa_populations(ctypes.byref(self._desc), self._buf[0].data_ptr(), self._cur,
                                                 _lib.ptr(self.flags), out.data_ptr(), None, self._stream())
            _lib.check(st, "aa_populations")
            return out
        prev = self._buf[1 - self._cur]
        if self.storage in ("f32", "f64"):
            st = _lib.load().tlbm_step(ctypes.byref(self._desc_none), prev.data_ptr(), out.data_ptr(),
                                       _lib.ptr(self.flags), None, None, None, self._stream())
            _lib.check(st, "tlbm_step(stream+bc)")
        else:
            # boundaries in the storage format, then widen to float32 locally
            tmp = torch.empty_like(prev)
            st = _lib.load().tlbm_step(ctypes.byref(self._desc_none), prev.data_ptr(), tmp.data_ptr(),
                                       _lib.ptr(self.flags), None, None, None, self._stream())
            _lib.check(st, "tlbm_step(stream+bc)")
            conv = self.cfg.desc(self.code, "none")
            _lib.check(_lib.load().tlbm_collide(ctypes.byref(conv), _lib.F32, tmp.data_ptr(), out.data_ptr(), None,
                                                None, self._stream()), "convert")
        return out

    def moment_sums(self) -> torch.Tensor:
        """float64 (mass, jx, jy, jz) of the stored post-collision state."""
        sums = _ops.moment_sums(self.q, self.state, self.code)
        if self.pattern == "aa" and self._cur == 0:
            sums[1:] = -sums[1:]   # swapped layout: slot opp(q) holds population q
        return sums   # AA: of the latest collided state, one collision behind the two-buffer step

    def nonfinite_seen(self) -> bool:
        """True if any step produced a non-finite density (reads one int)."""
        return bool(self.status.item() != 0)

    def force_history(self) -> torch.Tensor:
        """float64 force of every recorded step (row k: step k + 1 since the last load)."""
        if not self.forces:
            return torch.zeros((0, 3), dtype=torch.float64, device=self.device)
        if self.pattern == "aa":
            # AA launch k samples step k - 1: drop the sample of the loaded
            # state and take the latest step's from a readout of the buffer
            last = torch.zeros(3, dtype=torch.float64, device=self.device)
            tmp = torch.empty((self.q,) + self.cfg.shape, dtype=self.compute_dtype, device=self.device)
            st = _lib.load().tlbm_aa_populations(ctypes.byref(self._desc), self._buf[0].data_ptr(), self._cur,
                                                 _lib.ptr(self.flags), tmp.data_ptr(), last.data_ptr(),
                                                 self._stream())
            _lib.check(st, "aa_populations")
            return torch.stack(self.forces[1:] + [last])
        return torch.stack(self.forces)


def make_step(lattice, shape, tau: float, collision: str = "bgk", *, device=None, wall_mask=None,
              obstacle_mask=None, wall_mode: str = "fullway", tau_field=None, dtype=torch.float32, **cfg):
    """Functional ``step(f) -> f`` with TensorLBM's chain collide -> stream -> boundaries.

    Two passes per call: collision (local) then pull + boundaries.  Returns a new
    tensor; the input is not modified.  ``step.last_force`` holds the float64
    momentum-exchange force of the latest call when an obstacle is given."""
    q = _LATTICES[lattice]
    shape = tuple(int(s) for s in shape)
    scfg = StepConfig(q, shape, float(tau), collision, **cfg)
    dev = _ops.cuda_device(device)
    code = _lib.real_dtype(torch.empty(0, dtype=dtype))
    flags = None
    if wall_mask is not None or obstacle_mask is not None:
        flags = _ops.build_flags(shape, dev, wall_mask, obstacle_mask, wall_mode)
    tf = None if tau_field is None else tau_field.to(device=dev, dtype=torch.float32).contiguous()
    d_coll = scfg.desc(code)
    d_bc = scfg.desc(code, "none")
    track = obstacle_mask is not None

    def step(f: torch.Tensor) -> torch.Tensor:
        if tuple(f.shape) != (q,) + shape or f.dtype != dtype:
            raise ValueError(f"step expects {(q,) + shape} {dtype}, got {tuple(f.shape)} {f.dtype}")
        _lib.require_cuda(f)
        f = f.contiguous()
        tmp = torch.empty_like(f)
        out = torch.empty_like(f)
        s = _lib.stream_of(dev)
        lib = _lib.load()
        _lib.check(lib.tlbm_collide(ctypes.byref(d_coll), code, f.data_ptr(), tmp.data_ptr(), _lib.ptr(flags), _lib.ptr(tf), s),
                   "collide")
        force = torch.zeros(3, dtype=torch.float64, device=dev) if track else None
        _lib.check(lib.tlbm_step(ctypes.byref(d_bc), tmp.data_ptr(), out.data_ptr(), _lib.ptr(flags), None,
                                 _lib.ptr(force), None, s), "stream+boundaries")
        step.last_force = force
        return out

    step.last_force = None
    return step


# The TritonFusedSolver3D surface (triton_fused.py:676-960): float32, float16
# and bfloat16 storage, precision-policy names; see tensorlbm_b200.triton_fused.
from .triton_fused import TritonFusedSolver3D as FusedSolver3D  # noqa: E402
