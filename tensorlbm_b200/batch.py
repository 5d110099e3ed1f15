"""Batched runner: many independent small D2Q9 or D3Q19 domains advanced together.

TensorLBM's scan runner advances design points one after the other in worker
processes (``scan_runner.py:697`` ``run_scan_point``, ``:979``
``ScanExecutor``), each running the cylinder-flow chain of
``cylinder_flow.py:854-899``.  :class:`BatchedSolver` packs all the domains
of a scan into one population buffer.  It advances them with one kernel launch
per step, replayed as a CUDA graph, or one persistent cooperative launch for
many steps.  Every domain evolves bit for bit as it would alone.
:func:`autotune` picks the tile shape and the execution mode by timing them on
the actual domain set.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib, _ops


BatchDomain = _lib.BatchDomain
BatchDesc = _lib.BatchDesc


def _fn(name):
    return getattr(_lib.load(), name)


@dataclass
class DomainSpec:
    """One domain: (ny, nx) grid (D2Q9) or (nz, ny, nx) with nz > 1 (D3Q19),
    BGK/MRT relaxation time, Zou/He inlet velocity and outlet density (None
    disables the plane), moving-lid velocity at y = ny - 1 (None: no lid),
    wall and obstacle masks, and how the walls bounce back ("fullway" after
    streaming, or "halfway": pre-streaming, from the pre-collision state)."""

    nx: int
    ny: int
    tau: float
    u_in: float | None = None
    rho_out: float | None = 1.0
    wall_mask: torch.Tensor | None = None
    obstacle_mask: torch.Tensor | None = None
    nz: int = 1
    u_lid: float | None = None
    wall_mode: str = "fullway"

    @property
    def shape(self) -> tuple[int, ...]:
        return (self.ny, self.nx) if self.nz == 1 else (self.nz, self.ny, self.nx)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def bc(self) -> int:
        return ((_lib.BC_ZH_INLET if self.u_in is not None else 0) |
                (_lib.BC_ZH_OUTLET if self.rho_out is not None else 0) |
                (_lib.BC_LID if self.u_lid is not None else 0))


def cavity_point(resolution, re: float = 400.0, *, u_lid: float = 0.06, span: int | None = None,
                 device=None) -> DomainSpec:
    """TensorLBM's lid-driven cavity case (cases/cavity.py:25-110) as one
    D3Q19 domain: resolution n gives (nz, ny, nx) = (span or max(4, n // 4), n, n)
    (or an explicit (nz, ny, nx)); stationary walls x = 0, x = nx - 1, y = 0
    bounce back half-way before streaming from the pre-collision state; the
    Zou/He lid moves at y = ny - 1; z is periodic; tau = 1/2 + nu / (1/3) with
    nu = u_lid nx / Re (cases/base.py:67-75 CaseUnits.from_reference); the
    state starts at rest (rho = 1)."""
    if isinstance(resolution, int):
        if resolution < 8:
            raise ValueError(f"resolution must be >= 8, got {resolution}")
        shape = (span if span is not None else max(4, resolution // 4), resolution, resolution)
    else:
        if len(resolution) != 3:
            raise ValueError("resolution sequence must be (nz, ny, nx)")
        shape = tuple(int(v) for v in resolution)
    nz, ny, nx = shape
    if re <= 0 or u_lid <= 0:
        raise ValueError("re and u_lid must be positive")
    nu = u_lid * float(nx) / re
    tau = 0.5 + nu / (1.0 / 3.0)
    dev = _ops.cuda_device(device)
    wall = torch.zeros(shape, dtype=torch.bool, device=dev)
    wall[:, :, 0] = True
    wall[:, :, -1] = True
    wall[:, 0, :] = True
    return DomainSpec(nx, ny, tau, None, None, wall, None, nz=nz, u_lid=float(u_lid), wall_mode="halfway")


def cylinder_channel(nx: int, re: float, u_in: float = 0.05, device=None) -> DomainSpec:
    """The batched-form case: ny = nx/4, cylinder of diameter D = ny/8 at
    (ny/2, ny/2), channel walls top and bottom, tau = 3 u D / Re + 0.5
    (cylinder_flow.py conventions; masks from cylinder_mask / make_channel_wall_mask)."""
    from . import boundaries

    ny = nx // 4
    d = ny / 8.0
    obst = boundaries.cylinder_mask(nx, ny, ny / 2.0, ny / 2.0, d / 2.0, device)
    wall = boundaries.make_channel_wall_mask(ny, nx, obst, device)
    return DomainSpec(nx, ny, 3.0 * u_in * d / re + 0.5, u_in, 1.0, wall, obst)


class BatchedSolver:
    """Packed multi-domain D2Q9 or D3Q19 solver (float32).

    State phase and API follow :class:`tensorlbm_b200.LBMSolver`: ``load``
    takes TensorLBM-phase fields, ``f(i)`` returns domain i in that phase, and
    ``forces`` holds the float64 momentum-exchange force per domain of every
    recorded step."""

    ALIGN = 32  # elements: every domain block starts on a 128-byte boundary

    def __init__(self, domains: list[DomainSpec], collision: str = "bgk", *, device=None,
                 tile: tuple[int, int] = (64, 4), mode: str = "graph", ctas_per_sm: int = 0,
                 lattice: str = "D2Q9", order: str = "domain", retire: bool = False, cells_per_thread: int = 1):
        if collision not in ("bgk", "mrt"):
            raise ValueError("the batched runner supports 'bgk' and 'mrt'")
        if mode not in ("graph", "launch", "persistent"):
            raise ValueError("mode must be 'graph', 'launch' or 'persistent'")
        if lattice not in ("D2Q9", "D3Q19"):
            raise ValueError("the batched runner supports D2Q9 and D3Q19 domains")
        self.q = 9 if lattice == "D2Q9" else 19
        self.lattice = lattice
        self.device = _ops.cuda_device(device)
        self.domains = list(domains)
        for i, d in enumerate(self.domains):
            if (self.q == 9) != (d.nz == 1):
                raise ValueError(f"domain {i} has nz = {d.nz}: {lattice} domains need "
                                 f"{'nz == 1' if self.q == 9 else 'nz > 1'}")
        self.collision = collision
        self.mode = mode
        n = len(self.domains)
        doms = (BatchDomain * n)()
        f_off, c_off = 0, 0
        self.f_offsets, self.cell_offsets = [], []
        for i, d in enumerate(self.domains):
            cells = d.cells
            doms[i].f_offset, doms[i].cell_offset = f_off, c_off
            doms[i].nx, doms[i].ny, doms[i].nz, doms[i].tau = d.nx, d.ny, d.nz, float(d.tau)
            doms[i].u_in = float(d.u_in or 0.0)
            doms[i].rho_out = float(1.0 if d.rho_out is None else d.rho_out)
            doms[i].u_lid = float(d.u_lid or 0.0)
            doms[i].bc = d.bc
            self.f_offsets.append(f_off)
            self.cell_offsets.append(c_off)
            f_off += -(-self.q * cells // self.ALIGN) * self.ALIGN
            c_off += -(-cells // self.ALIGN) * self.ALIGN
        self.n_cells = sum(d.cells for d in self.domains)
        self._host_domains = doms
        self.domains_dev = torch.frombuffer(bytearray(doms), dtype=torch.uint8).to(self.device)
        self.fa = torch.zeros(f_off, dtype=torch.float32, device=self.device)
        self.fb = torch.zeros_like(self.fa)
        self.flags = torch.zeros(c_off, dtype=torch.uint8, device=self.device)
        for i, d in enumerate(self.domains):
            if d.wall_mask is not None or d.obstacle_mask is not None:
                fl = _ops.build_flags(d.shape, self.device, d.wall_mask, d.obstacle_mask, d.wall_mode)
                self.flags[self.cell_offsets[i]: self.cell_offsets[i] + d.cells] = fl.reshape(-1)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        # retire: a domain that turns non-finite is skipped from then on (a
        # scan marks such a point failed; its cells cost nothing more)
        self.domain_status = torch.zeros(n, dtype=torch.int32, device=self.device) if retire else None
        self.sync = torch.zeros(3, dtype=torch.int32, device=self.device)
        self._pgraphs: dict = {}
        self._pgraph_capture = True   # persistent launches go through CUDA graphs
        self.ctas_per_sm = ctas_per_sm
        self.order = order
        if cells_per_thread not in (1, 2):
            raise ValueError("cells_per_thread must be 1 or 2")
        self.cells_per_thread = cells_per_thread
        self.set_tile(*tile)
        self.steps_done = 0
        self.step_offsets = [0] * n   # steps each domain had completed before the last load()/resume()
        self._cur = 0
        self._graph = None
        self.forces: list[torch.Tensor] = []

    # -- layout -----------------------------------------------------------------

    ORDERS = ("domain", "interleave", "largest_first")

    def set_tile(self, tx: int, ty: int, order: str | None = None, cells_per_thread: int | None = None) -> None:
        """Tile shape (tx x ty cells over the rows of each domain) and the
        order of the tile list, which is the CTA-to-domain mapping: the launch
        gives CTA b tile b, the persistent kernel gives CTA b tiles b, b + G,
        b + 2G ...  "domain": each domain's tiles together, row by row;
        "interleave": round robin over the domains (one tile of each in turn);
        "largest_first": the domains by decreasing size, each contiguous.
        cells_per_thread 2 runs a tile on tx / 2 x ty threads, two cells of a
        row each (the pair update where nx is even)."""
        cpt = cells_per_thread or getattr(self, "cells_per_thread", 1)
        if cpt not in (1, 2):
            raise ValueError("cells_per_thread must be 1 or 2")
        if tx % (32 * cpt) or (tx // cpt) * ty > 256 or ty < 1:
            raise ValueError(f"tile_x must be a multiple of {32 * cpt} and (tile_x / {cpt}) * tile_y <= 256")
        self.cells_per_thread = cpt
        order = order or getattr(self, "order", "domain")
        if order not in self.ORDERS:
            raise ValueError(f"order must be one of {self.ORDERS}")
        self.tile = (tx, ty)
        self.order = order
        per = []
        for i, d in enumerate(self.domains):
            per.append([(i, x0, r0) for r0 in range(0, d.ny * d.nz, ty) for x0 in range(0, d.nx, tx)])
        if order == "interleave":
            tiles = [p[k] for k in range(max(len(p) for p in per)) for p in per if k < len(p)]
        elif order == "largest_first":
            tiles = [t for i in sorted(range(len(per)), key=lambda i: -self.domains[i].cells) for t in per[i]]
        else:
            tiles = [t for p in per for t in p]
        self._tiles_all = torch.tensor(tiles, dtype=torch.int32, device=self.device).reshape(-1, 3)
        self._tiles_live = None       # retired-domain mask the tile list was last compacted for
        self.ntiles = len(tiles)
        self.tiles_dev = self._tiles_all.reshape(-1)
        self._graph = None
        self._pgraphs = {}

    def _compact_tiles(self) -> None:
        """With retire=True: drop the tiles of retired domains from the tile
        list (in the list's order), so that no launch visits them; the list is
        rebuilt on the device from the full one whenever the set of retired
        domains changes (one read of the per-domain status words)."""
        if self.domain_status is None:
            return
        live = self.domain_status == 0
        key = live.cpu()
        if self._tiles_live is not None and torch.equal(key, self._tiles_live):
            return
        tiles = self._tiles_all[live[self._tiles_all[:, 0].long()]]
        self._tiles_live = key
        self.ntiles = int(tiles.shape[0])
        self.tiles_dev = tiles.reshape(-1).contiguous()
        self._graph = None
        self._pgraphs = {}

    def _desc(self) -> BatchDesc:
        b = BatchDesc()
        b.lattice, b.dtype = self.q, _lib.F32
        b.collision = _lib.COLL_BGK if self.collision == "bgk" else _lib.COLL_MRT
        b.ndomains = len(self.domains)
        b.tile_x, b.tile_y = self.tile
        b.ctas_per_sm = self.ctas_per_sm
        b.cells_per_thread = self.cells_per_thread
        b.domain_status = _lib.ptr(self.domain_status)
        return b

    def _view(self, buf: torch.Tensor, i: int) -> torch.Tensor:
        d = self.domains[i]
        o = self.f_offsets[i]
        return buf[o: o + self.q * d.cells].view((self.q,) + d.shape)

    def _flags_view(self, i: int) -> torch.Tensor:
        d = self.domains[i]
        o = self.cell_offsets[i]
        return self.flags[o: o + d.cells].view(d.shape)

    def _single_desc(self, i: int, collision: str):
        from .solvers import COLLISIONS

        d = self.domains[i]
        rates = dict(s_e=1.64, s_eps=1.54, s_q=1.7) if self.q == 9 else dict(s_e=1.19, s_eps=1.4, s_q=1.2)
        return _ops.make_desc(self.q, (d.nx, d.ny, d.nz), _lib.F32, COLLISIONS[collision], d.tau, bc=d.bc,
                              u_in=(float(d.u_in or 0.0), 0.0, 0.0), u_lid=float(d.u_lid or 0.0),
                              rho_out=float(1.0 if d.rho_out is None else d.rho_out), **rates)

    # -- state ----------------------------------------------------------------

    def load(self, fields: list[torch.Tensor]) -> "BatchedSolver":
        """TensorLBM-phase initial populations, one (9, ny, nx) tensor per domain."""
        if len(fields) != len(self.domains):
            raise ValueError(f"{len(fields)} fields for {len(self.domains)} domains")
        lib = _lib.load()
        s = _lib.stream_of(self.device)
        for i, f in enumerate(fields):
            d = self.domains[i]
            if tuple(f.shape) != (self.q,) + d.shape:
                raise ValueError(f"domain {i}: expected {(self.q,) + d.shape}, got {tuple(f.shape)}")
            src = f.to(device=self.device, dtype=torch.float32).contiguous()
            desc = self._single_desc(i, self.collision)
            _lib.check(lib.tlbm_collide(ctypes.byref(desc), _lib.F32, src.data_ptr(), self._view(self.fa, i).data_ptr(),
                                        self._flags_view(i).data_ptr(), None, s), "collide")
        self._cur = 0
        self.steps_done = 0
        self.step_offsets = [0] * len(self.domains)
        self.forces = []
        self._graph = None
        self._pgraphs = {}
        if self.domain_status is not None:
            self.domain_status.zero_()
        self._f0 = [f.to(self.device, torch.float32).clone() for f in fields]
        return self

    def retired_domains(self) -> torch.Tensor:
        """Bool per domain: retired after a non-finite density (retire=True only)."""
        if self.domain_status is None:
            return torch.zeros(len(self.domains), dtype=torch.bool, device=self.device)
        return self.domain_status != 0

    def resume(self, fields: list[torch.Tensor], steps: list[int]) -> "BatchedSolver":
        """Continue from checkpointed TensorLBM-phase fields; ``steps[i]`` is the
        step count domain i had completed.  The state is rebuilt as
        collide(S_n), which is exactly the stored state (float32), so the
        continuation is bit-exact."""
        if len(steps) != len(self.domains):
            raise ValueError(f"{len(steps)} step counts for {len(self.domains)} domains")
        self.load(fields)
        self.step_offsets = [int(k) for k in steps]
        return self

    @property
    def step_counts(self) -> list[int]:
        """Completed steps of each domain (all advance together)."""
        return [k + self.steps_done for k in self.step_offsets]

    def _bufs(self):
        return (self.fa, self.fb) if self._cur == 0 else (self.fb, self.fa)

    def _launch(self, src, dst, forces, slot=None) -> None:
        st = _fn("tlbm_batch_step")(ctypes.byref(self._desc()), self.domains_dev.data_ptr(), self.tiles_dev.data_ptr(),
                                   self.ntiles, src.data_ptr(), dst.data_ptr(), self.flags.data_ptr(),
                                   _lib.ptr(forces), _lib.ptr(slot), self.status.data_ptr(),
                                   _lib.stream_of(self.device))
        _lib.check(st, "tlbm_batch_step")

    def _run_recorded_graph(self, n: int, record_every: int, hist: torch.Tensor) -> int:
        """Graph-replayed steps that record forces: the recording launch finds
        its history slot through a device counter that the graph advances.
        Returns the number of steps done (a multiple of the captured chunk)."""
        k = record_every if record_every % 2 == 0 else 2 * record_every  # even: the parity returns
        reps = n // k
        if reps == 0:
            return 0
        slot = torch.zeros(1, dtype=torch.int32, device=self.device)
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s), torch.cuda.graph(g, stream=s):
            c = self._cur
            for j in range(k):
                src, dst = (self.fa, self.fb) if c == 0 else (self.fb, self.fa)
                if j % record_every == 0:
                    self._launch(src, dst, hist, slot)
                    _lib.check(_fn("tlbm_batch_advance_slot")(slot.data_ptr(), _lib.stream_of(self.device)),
                               "tlbm_batch_advance_slot")
                else:
                    self._launch(src, dst, None)
                c ^= 1
        torch.cuda.current_stream(self.device).wait_stream(s)
        for _ in range(reps):
            g.replay()
        self.steps_done += reps * k
        del g
        return reps * k

    def step(self, n: int = 1, *, record_forces: bool = False) -> "BatchedSolver":
        for _ in range(n):
            src, dst = self._bufs()
            forces = None
            if record_forces:
                forces = torch.zeros((len(self.domains), 3), dtype=torch.float64, device=self.device)
                self.forces.append(forces)
            self._launch(src, dst, forces)
            self._cur ^= 1
            self.steps_done += 1
        return self

    def run(self, n: int, *, record_every: int = 0, chunk: int = 64, max_spins: int = 1 << 24) -> torch.Tensor | None:
        """Advance n steps in the configured mode.  With record_every > 0 returns
        the float64 force history (n // record_every, ndomains, 3)."""
        hist = None
        if record_every > 0:
            hist = torch.zeros((-(-n // record_every), len(self.domains), 3), dtype=torch.float64, device=self.device)
        self._compact_tiles()
        if self.ntiles == 0:   # every domain retired
            self._cur ^= n & 1
            self.steps_done += n
            return hist
        if self.mode == "persistent":
            # one persistent cooperative launch of n steps, captured in a CUDA
            # graph the first time (per n, recording interval and parity) and
            # replayed after that; the forces go to the graph's own history
            key = (n, record_every, self._cur, max_spins)
            entry = self._pgraphs.get(key)
            if entry is None and not self._pgraph_capture:
                a, b = self._bufs()
                st = _fn("tlbm_batch_run")(ctypes.byref(self._desc()), self.domains_dev.data_ptr(),
                                          self.tiles_dev.data_ptr(), self.ntiles, a.data_ptr(), b.data_ptr(),
                                          self.flags.data_ptr(), n, _lib.ptr(hist), record_every,
                                          self.sync.data_ptr(), self.status.data_ptr(), max_spins,
                                          _lib.stream_of(self.device))
                _lib.check(st, "tlbm_batch_run")
                self._cur ^= n & 1
                self.steps_done += n
                return hist
            if entry is None:
                ghist = None if hist is None else torch.zeros_like(hist)
                a, b = self._bufs()
                desc = self._desc()
                s = torch.cuda.Stream(self.device)
                s.wait_stream(torch.cuda.current_stream(self.device))
                g = torch.cuda.CUDAGraph()
                try:
                    with torch.cuda.stream(s), torch.cuda.graph(g, stream=s):
                        if ghist is not None:
                            ghist.zero_()
                        st = _fn("tlbm_batch_run")(ctypes.byref(desc), self.domains_dev.data_ptr(),
                                                  self.tiles_dev.data_ptr(), self.ntiles, a.data_ptr(),
                                                  b.data_ptr(), self.flags.data_ptr(), n, _lib.ptr(ghist),
                                                  record_every, self.sync.data_ptr(), self.status.data_ptr(),
                                                  max_spins, _lib.stream_of(self.device))
                        _lib.check(st, "tlbm_batch_run (capture)")
                except RuntimeError:
                    # a runtime without graph capture of cooperative launches:
                    # launch directly from now on
                    torch.cuda.current_stream(self.device).wait_stream(s)
                    self._pgraph_capture = False
                    return self.run(n, record_every=record_every, chunk=chunk, max_spins=max_spins)
                torch.cuda.current_stream(self.device).wait_stream(s)
                entry = (g, ghist)
                self._pgraphs[key] = entry
            entry[0].replay()
            self._cur ^= n & 1
            self.steps_done += n
            return None if hist is None else entry[1].clone()
        if record_every > 0 and self.mode == "graph":
            done = self._run_recorded_graph(n, record_every, hist)
            for k in range(done, n):
                src, dst = self._bufs()
                self._launch(src, dst, hist[k // record_every] if k % record_every == 0 else None)
                self._cur ^= 1
                self.steps_done += 1
            return hist
        if record_every > 0 or self.mode == "launch" or n < chunk:
            for k in range(n):
                src, dst = self._bufs()
                forces = hist[k // record_every] if record_every > 0 and k % record_every == 0 else None
                self._launch(src, dst, forces)
                self._cur ^= 1
                self.steps_done += 1
            return hist
        chunk += chunk & 1
        if self._graph is None or self._graph[1] != chunk or self._graph[2] != self._cur:
            s = torch.cuda.Stream(self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            g = torch.cuda.CUDAGraph()
            cur0 = self._cur
            with torch.cuda.stream(s), torch.cuda.graph(g, stream=s):
                c = cur0
                for _ in range(chunk):
                    src, dst = (self.fa, self.fb) if c == 0 else (self.fb, self.fa)
                    self._launch(src, dst, None)
                    c ^= 1
            torch.cuda.current_stream(self.device).wait_stream(s)
            self._graph = (g, chunk, cur0)
        g = self._graph[0]
        reps, rest = divmod(n, chunk)
        for _ in range(reps):
            g.replay()
        self.steps_done += reps * chunk
        if rest:
            self.step(rest)
        return hist

    def f(self, i: int) -> torch.Tensor:
        """Domain i in TensorLBM's phase (one extra pull + boundary pass)."""
        if self.steps_done == 0:
            return self._f0[i].clone()
        prev = self.fb if self._cur == 0 else self.fa
        d = self.domains[i]
        out = torch.empty((self.q,) + d.shape, dtype=torch.float32, device=self.device)
        desc = self._single_desc(i, "none")
        st = _lib.load().tlbm_step(ctypes.byref(desc), self._view(prev, i).data_ptr(), out.data_ptr(),
                                   self._flags_view(i).data_ptr(), None, None, None, _lib.stream_of(self.device))
        _lib.check(st, "tlbm_step(stream+bc)")
        return out

    def finite_domains(self) -> torch.Tensor:
        """Bool per domain: every stored population of the current state finite.
        (The status word only says that some domain produced a non-finite value.)"""
        cur = self.fa if self._cur == 0 else self.fb
        return torch.stack([torch.isfinite(self._view(cur, i)).all() for i in range(len(self.domains))])

    def timed_steps(self, n: int) -> float:
        """Seconds for n steps in the current mode (CUDA events, after one warm-up step)."""
        self.run(1)
        cur = torch.cuda.current_stream(self.device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(self.device)
        e0.record(cur)
        self.run(n)
        e1.record(cur)
        torch.cuda.synchronize(self.device)
        return e0.elapsed_time(e1) / 1e3


def autotune(solver: BatchedSolver, steps: int = 20,
             tiles=((32, 8), (64, 4), (128, 2), (256, 1), (32, 4), (64, 2), (128, 1), (128, 4), (256, 2), (512, 1)),
             modes=("graph", "persistent"), orders=BatchedSolver.ORDERS, ctas_per_sm=(0, 2, 4),
             cells_per_thread=(1, 2)) -> dict:
    """Time every candidate on the solver's own domains and keep the fastest:
    tile shape x cells per thread x execution mode x CTA-to-domain mapping
    (the tile order of BatchedSolver.set_tile) and, for the persistent
    kernel, the CTAs per SM (0 = as many as fit).  Shapes a cells-per-thread
    choice does not admit are skipped.  Every trial updates every domain
    (retired ones too).  The state is advanced by the trials; reload it
    afterwards."""
    results = []
    for mode in modes:
        for cpt in cells_per_thread:
            for tx, ty in tiles:
                if tx % (32 * cpt) or (tx // cpt) * ty > 256:
                    continue
                for order in orders:
                    for cps in (ctas_per_sm if mode == "persistent" else (0,)):
                        solver.mode = mode
                        solver.ctas_per_sm = cps
                        solver.set_tile(tx, ty, order, cpt)
                        if solver.domain_status is not None:
                            solver.domain_status.zero_()     # every trial updates every domain
                        try:
                            t = solver.timed_steps(steps)
                        except (RuntimeError, NotImplementedError):
                            continue
                        results.append({"mode": mode, "tile": (tx, ty), "cells_per_thread": cpt, "order": order,
                                        "ctas_per_sm": cps, "seconds": t, "mlups": solver.n_cells * steps / t / 1e6})
    best = max(results, key=lambda r: r["mlups"])
    solver.mode = best["mode"]
    solver.ctas_per_sm = best["ctas_per_sm"]
    solver.set_tile(*best["tile"], best["order"], best["cells_per_thread"])
    return {"best": best, "trials": results}


def uniform_scan(n_domains: int, seed: int, device=None, nx_range=(128, 1024), re_range=(40.0, 300.0),
                 u_in: float = 0.05) -> list[DomainSpec]:
    """Seeded design of the batched-form case: nx ~ U{nx_range} (multiple of 8 so
    that ny = nx/4 and D = ny/8 stay whole), Re ~ U(re_range)."""
    g = torch.Generator().manual_seed(seed)
    nxs = torch.randint(nx_range[0] // 8, nx_range[1] // 8 + 1, (n_domains,), generator=g) * 8
    res = re_range[0] + (re_range[1] - re_range[0]) * torch.rand(n_domains, generator=g, dtype=torch.float64)
    return [cylinder_channel(int(nx), float(re), u_in, device) for nx, re in zip(nxs.tolist(), res.tolist())]


def equilibrium_start(domains: list[DomainSpec], device=None) -> list[torch.Tensor]:
    """Start state of each domain: the equilibrium at rho = 1 with the inlet
    velocity in x and zero velocity in the obstacle (cylinder_flow.py start
    state); domains without an inlet start at rest (the cavity case)."""
    from .d2q9 import equilibrium
    from .d3q19 import equilibrium3d

    out = []
    for d in domains:
        ux = torch.full(d.shape, float(d.u_in or 0.0), device=device)
        if d.obstacle_mask is not None:
            ux[d.obstacle_mask.to(ux.device)] = 0.0
        z = torch.zeros_like(ux)
        out.append(equilibrium(torch.ones_like(ux), ux, z) if d.nz == 1 else
                   equilibrium3d(torch.ones_like(ux), ux, z, z))
    return out


def strouhal(lift: torch.Tensor, length_ref: float, u_ref: float, sample_every: int = 1,
             st_band=(0.05, 0.35)) -> float | None:
    """Dominant shedding frequency of a lift history as St = f D / U: Hann
    window, band-limited FFT peak (the FFT branch of postprocess.py:646)."""
    x = lift.detach().double().cpu()
    x = x - x.mean()
    n = x.numel()
    if n < 32:
        return None
    w = torch.hann_window(n, periodic=False, dtype=torch.float64)
    spec = torch.fft.rfft(x * w).abs()
    freq = torch.fft.rfftfreq(n, d=float(sample_every), dtype=torch.float64)
    st = freq * length_ref / u_ref
    band = (st >= st_band[0]) & (st <= st_band[1])
    if not bool(band.any()):
        return None
    k = int(torch.argmax(torch.where(band, spec, torch.zeros_like(spec))))
    return float(st[k])


__all__ =["DomainSpec", "BatchedSolver", "autotune", "cavity_point", "cylinder_channel", "uniform_scan",
           "equilibrium_start", "strouhal"]


def scan(n_domains: int = 512, steps: int = 50_000, record_every: int = 10, seed: int = 20261203,
         sample: int = 16, device=None, nx_range=(128, 1024), re_range=(40.0, 300.0), log=print) -> dict:
    """The batched scan: every domain of a seeded design advanced together for
    `steps` steps (forces recorded every `record_every`), the Strouhal number of
    every domain that stays finite (lift spectrum of the second half), and a
    sample of the same domains run one after the other as plain fused runs for
    the comparison of St, force histories and throughput."""
    from . import LBMSolver

    dev = _ops.cuda_device(device)
    doms = uniform_scan(n_domains, seed, dev, nx_range, re_range)
    f0 = equilibrium_start(doms, dev)
    b = BatchedSolver(doms, "bgk", device=dev)
    tune = autotune(b, steps=20)
    b.load(f0)
    cur = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(cur)
    hist = b.run(steps, record_every=record_every)
    e1.record(cur)
    torch.cuda.synchronize(dev)
    t_batch = e0.elapsed_time(e1) / 1e3
    finite = b.finite_domains().cpu().tolist()
    half = hist.shape[0] // 2
    st_batch = [strouhal(hist[half:, i, 1], d.ny / 8.0, d.u_in, record_every) if finite[i] else None
                for i, d in enumerate(doms)]
    log(f"batched: {b.n_cells * steps / t_batch / 1e6:.0f} MLUPS, {sum(finite)}/{len(doms)} finite, "
        f"tile {tune['best']['tile']} mode {tune['best']['mode']}")
    # sequential sample: finite domains spread over the design
    idx = [i for i in range(len(doms)) if finite[i]]
    pick = [idx[int(k * (len(idx) - 1) / max(sample - 1, 1))] for k in range(min(sample, len(idx)))]
    seq = []
    t_seq, cells_seq = 0.0, 0
    for i in pick:
        d = doms[i]
        s = LBMSolver("D2Q9", (d.ny, d.nx), d.tau, "bgk", device=dev, wall_mask=d.wall_mask,
                      obstacle_mask=d.obstacle_mask, u_in=d.u_in, rho_out=d.rho_out, track_force=True).load(f0[i])
        torch.cuda.synchronize(dev)
        e0.record(cur)
        s.step(steps)
        e1.record(cur)
        torch.cuda.synchronize(dev)
        t_seq += e0.elapsed_time(e1) / 1e3
        cells_seq += d.nx * d.ny * steps
        fh = s.force_history()[0::record_every]  # the batch records steps 0, r, 2r, ...
        st_s = strouhal(fh[fh.shape[0] // 2:, 1], d.ny / 8.0, d.u_in, record_every)
        dmax = float((fh[: hist.shape[0]] - hist[: fh.shape[0], i]).abs().max())
        scale = float(hist[:, i].abs().max())
        seq.append({"domain": i, "nx": d.nx, "re": d.re if hasattr(d, "re") else None, "tau": d.tau,
                    "st_batched": st_batch[i], "st_sequential": st_s,
                    "force_max_rel_diff": dmax / max(scale, 1e-300)})
        del s
    res = {"domains": len(doms), "steps": steps, "record_every": record_every, "cells": b.n_cells,
           "batched_mlups": b.n_cells * steps / t_batch / 1e6, "batched_seconds": t_batch,
           "sequential_sample_mlups": cells_seq / max(t_seq, 1e-12) / 1e6,
           "finite_domains": int(sum(finite)), "autotune": tune["best"],
           "strouhal": [{"nx": d.nx, "tau": d.tau, "st": st_batch[i]} for i, d in enumerate(doms)],
           "sequential_sample": seq}
    res["speedup_vs_sequential"] = res["batched_mlups"] / max(res["sequential_sample_mlups"], 1e-12)
    return res


def main(argv=None) -> None:
    import argparse
    import json
    import pathlib

    ap = argparse.ArgumentParser(description="batched D2Q9 cylinder scan with Strouhal numbers")
    ap.add_argument("--domains", type=int, default=512)
    ap.add_argument("--steps", type=int, default=50_000)
    ap.add_argument("--record-every", type=int, default=10)
    ap.add_argument("--sample", type=int, default=16)
    ap.add_argument("--out", default="batch_scan_out")
    args = ap.parse_args(argv)
    res = scan(args.domains, args.steps, args.record_every, sample=args.sample, log=lambda s: print(s, flush=True))
    out = pathlib.Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    (out / "scan.json").write_text(json.dumps(res))
    print(json.dumps({k: v for k, v in res.items() if k not in ("strouhal",)}))


if __name__ == "__main__":
    main()
