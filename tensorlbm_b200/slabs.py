"""Z-slab decomposition of the fused step: one slab of ``nz_local`` planes per
rank (or per slab in one process), plus one ghost plane on each side, and a
halo exchange of the populations that cross each face.

The layout and exchange are those of TensorLBM's distributed fused solver
(triton_fused_distributed.py:1-60, :442-555):
- rank r owns global planes ``[r nz_local, (r + 1) nz_local)`` at local
  planes ``1 .. nz_local``;
- plane 0 holds the lower neighbour's top plane and ``nz_local + 1`` the
  upper neighbour's bottom plane, periodic in z;
- a pull step reads the lower ghost only for the directions with c_z = +1
  and the upper ghost only for c_z = -1 (D3Q19 5 of 19, D3Q27 9 of 27), so
  only those lanes cross.

Differences from that design:

- **Owned planes only.** The step kernel updates only the owned planes
  (``tlbm_step_planes``). The ghost planes never take part in a periodic
  wrap, so the owned values equal those of the undivided domain bit for bit,
  with any collision, storage format, obstacle, Zou/He x-planes or drag of
  :class:`~tensorlbm_b200.solvers.LBMSolver`.
- **No staging.** Each crossing lane of a boundary plane is one contiguous
  ``ny * nx`` block (the field is (Q, z, y, x)). It is sent straight from the
  owned plane and received straight into the neighbour's ghost plane: no
  gather or scatter kernels, no staging buffers.
- **Overlap.** A step computes the two boundary planes first, posts the
  exchange of their lanes (NCCL runs it on its own stream), then computes
  the interior planes. The next step's launch waits for the exchange on the
  stream, never on the host.
"""

from __future__ import annotations

import ctypes

import torch
import torch.distributed as dist

from . import _lib
from .lattice import LATTICES
from .solvers import LBMSolver


def crossing_face_indices(cz, sign: int) -> tuple[int, ...]:
    """Directions q with c_z[q] == sign: the lanes a pull step reads from the
    ghost plane below (sign +1) or above (sign -1)
    (triton_fused_distributed.py:115)."""
    if sign not in (+1, -1):
        raise ValueError(f"sign must be +1 or -1, got {sign}")
    return tuple(q for q in range(len(cz)) if int(cz[q]) == sign)


class SlabGeometry:
    """Which planes a slab owns and which lanes cross its faces.

    nz_global planes split into ``world`` slabs of nz_global / world planes;
    the local buffer is (Q, nz_local + 2, ny, nx) with the owned planes at
    1 .. nz_local."""

    def __init__(self, q: int, nz_global: int, ny: int, nx: int, world: int = 1, rank: int = 0):
        if q not in (19, 27):
            raise ValueError(f"z-slabs need a 3-D lattice (19 or 27 directions), got {q}")
        if world < 1 or not 0 <= rank < world:
            raise ValueError(f"rank {rank} outside world of {world}")
        if nz_global % world != 0:
            raise ValueError(f"nz_global={nz_global} must be divisible by world_size={world} "
                             "(slab decomposition along z)")
        self.q, self.nz_global, self.ny, self.nx = q, int(nz_global), int(ny), int(nx)
        self.world, self.rank = int(world), int(rank)
        self.nz_local = self.nz_global // self.world
        self.z_start_global = self.rank * self.nz_local
        self.z_end_global = self.z_start_global + self.nz_local
        self.left_neighbor = (self.rank - 1) % self.world
        self.right_neighbor = (self.rank + 1) % self.world
        cz = [int(c[2]) for c in LATTICES[q].c]
        self.cross_up = crossing_face_indices(cz, +1)     # top plane -> upper neighbour's plane 0
        self.cross_dn = crossing_face_indices(cz, -1)     # bottom plane -> lower neighbour's top ghost
        self.n_cross = len(self.cross_up)

    @property
    def local_shape(self) -> tuple[int, int, int, int]:
        return (self.q, self.nz_local + 2, self.ny, self.nx)

    def owned_slice(self) -> tuple[int, int]:
        return (1, self.nz_local + 1)

    def padded_planes(self) -> torch.Tensor:
        """Global plane index of every local plane (ghosts wrap periodically)."""
        z = torch.arange(self.z_start_global - 1, self.z_end_global + 1)
        return z % self.nz_global

    def local_from_global(self, field: torch.Tensor, dim: int = 0) -> torch.Tensor:
        """The local planes (owned and ghosts) of a global field whose z axis is ``dim``."""
        return field.index_select(dim, self.padded_planes().to(field.device)).contiguous()

    def halo_bytes_per_step(self, itemsize: int) -> int:
        """Bytes this slab sends per step (both faces); it receives as many."""
        return 2 * self.n_cross * self.ny * self.nx * itemsize

    def transfers(self, f: torch.Tensor):
        """(send view, destination rank, recv view, source rank) per crossing
        lane, matched in the same order on every rank."""
        top, bottom = self.nz_local, 1
        out = []
        for q in self.cross_up:
            out.append((f[q, top], self.right_neighbor, f[q, 0], self.left_neighbor))
        for q in self.cross_dn:
            out.append((f[q, bottom], self.left_neighbor, f[q, self.nz_local + 1], self.right_neighbor))
        return out


class LoopbackTransport:
    """One slab, periodic onto itself: the lanes are copied on the stream."""

    def start(self, geom: SlabGeometry, f: torch.Tensor):
        for send, _, recv, _ in geom.transfers(f):
            recv.copy_(send)
        return None

    def wait(self, handle) -> None:
        return None


class ProcessGroupTransport:
    """One slab per rank of a torch.distributed group (NCCL on GPUs, gloo on
    CPU tensors).  Every lane is one isend / irecv of a contiguous plane,
    posted as one batch; tags keep the lanes apart for backends that match by
    tag (NCCL matches a pair's messages in posting order)."""

    def __init__(self, group=None):
        self.group = group

    def start(self, geom: SlabGeometry, f: torch.Tensor):
        ops = []
        for k, (send, dst, recv, src) in enumerate(geom.transfers(f)):
            ops.append(dist.P2POp(dist.isend, send, dst, self.group, tag=2 * k))
            ops.append(dist.P2POp(dist.irecv, recv, src, self.group, tag=2 * k))
        return dist.batch_isend_irecv(ops)

    def wait(self, handle) -> None:
        # NCCL: the current stream waits for the exchange; gloo: the host waits
        for w in handle or ():
            w.wait()


class StagedTransport(ProcessGroupTransport):
    """ProcessGroupTransport with a narrower wire format (e.g. float16): the
    crossing lanes are packed and cast into staging planes (n_cross, ny, nx),
    exchanged, and cast back into the ghost planes on landing
    (triton_fused_distributed.py:333 ``halo_dtype``)."""

    def __init__(self, wire_dtype: torch.dtype, group=None):
        super().__init__(group)
        self.wire_dtype = wire_dtype
        self._stage = None
        self._lanes = None
        self._index = None

    def start(self, geom: SlabGeometry, f: torch.Tensor):
        shape = (geom.n_cross, geom.ny, geom.nx)
        lanes = (tuple(geom.cross_up), tuple(geom.cross_dn))
        if (self._stage is None or self._stage[0].shape != shape or self._stage[0].device != f.device
                or self._lanes != lanes):
            # staging planes and lane indices are built once per geometry and
            # device, so an exchange allocates nothing and copies nothing from the host
            self._stage = [torch.empty(shape, dtype=self.wire_dtype, device=f.device) for _ in range(4)]
            self._lanes = lanes
            self._index = (torch.tensor(lanes[0], dtype=torch.int64, device=f.device),
                           torch.tensor(lanes[1], dtype=torch.int64, device=f.device))
        send_up, send_dn, recv_up, recv_dn = self._stage
        up, dn = self._index
        send_up.copy_(f[:, geom.nz_local].index_select(0, up))
        send_dn.copy_(f[:, 1].index_select(0, dn))
        ops = [dist.P2POp(dist.isend, send_up, geom.right_neighbor, self.group, tag=1),
               dist.P2POp(dist.irecv, recv_up, geom.left_neighbor, self.group, tag=1),
               dist.P2POp(dist.isend, send_dn, geom.left_neighbor, self.group, tag=2),
               dist.P2POp(dist.irecv, recv_dn, geom.right_neighbor, self.group, tag=2)]
        return (dist.batch_isend_irecv(ops), geom, f, up, dn)

    def wait(self, handle) -> None:
        if handle is None:
            return
        works, geom, f, up, dn = handle
        super().wait(works)
        f[:, 0].index_copy_(0, up, self._stage[2].to(f.dtype))
        f[:, geom.nz_local + 1].index_copy_(0, dn, self._stage[3].to(f.dtype))


def exchange_halos(geom: SlabGeometry, f: torch.Tensor, transport=None) -> None:
    """Fill f's two ghost planes (crossing lanes) from the neighbouring slabs."""
    transport = transport or (LoopbackTransport() if geom.world == 1 else ProcessGroupTransport())
    transport.wait(transport.start(geom, f))


def exchange_ring(geoms, fields) -> None:
    """The exchange among slabs held by one process (any devices): every
    slab's crossing lanes into its neighbours' ghost planes."""
    for g, f in zip(geoms, fields):
        for q in g.cross_up:
            fields[g.right_neighbor][q, 0].copy_(f[q, g.nz_local])
        for q in g.cross_dn:
            fields[g.left_neighbor][q, g.nz_local + 1].copy_(f[q, 1])


class SlabSolver(LBMSolver):
    """One z-slab of the fused LBM step with halo exchange.

    Args:
        lattice: "D3Q19" or "D3Q27".
        global_shape: (nz_global, ny, nx) of the whole periodic-in-z domain.
        tau, collision, storage and the keyword options: as for
            :class:`LBMSolver` (obstacle / wall masks, tau_field, u_in /
            rho_out Zou-He x-planes, track_force, ...); masks and tau_field
            are GLOBAL fields, sliced here.
        world, rank: the decomposition (default: the torch.distributed group,
            or one slab).
        transport: how the ghost planes are filled: a ProcessGroupTransport
            (default for world > 1), a LoopbackTransport (world 1), or
            "external" (the caller exchanges, as :class:`MultiSlabSolver`
            does for slabs held by one process).
        overlap: compute the two boundary planes first and exchange them
            while the interior planes are computed.
    """

    def __init__(self, lattice, global_shape, tau: float, collision: str = "bgk", *, device=None, world=None,
                 rank=None, transport=None, overlap: bool = True, wall_mask=None, obstacle_mask=None,
                 tau_field=None, **kw):
        if kw.get("pattern", "ab") != "ab":
            raise NotImplementedError("z-slabs use the two-buffer step")
        for opt in ("curved_wall", "wall_velocity"):
            if kw.get(opt) is not None:
                raise NotImplementedError(f"{opt} is not sliced into z-slabs")
        if world is None:
            world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
        if rank is None:
            rank = dist.get_rank() if dist.is_available() and dist.is_initialized() else 0
        q = {"D3Q19": 19, "D3Q27": 27, 19: 19, 27: 27}.get(lattice)
        if q is None:
            raise ValueError(f"z-slabs need D3Q19 or D3Q27, got {lattice!r}")
        nz_g, ny, nx = (int(s) for s in global_shape)
        self.geom = SlabGeometry(q, nz_g, ny, nx, world, rank)
        local = self.geom.local_shape[1:]
        sl = self.geom.local_from_global
        super().__init__(lattice, local, tau, collision, device=device,
                         wall_mask=None if wall_mask is None else sl(wall_mask),
                         obstacle_mask=None if obstacle_mask is None else sl(obstacle_mask),
                         tau_field=None if tau_field is None else sl(tau_field), **kw)
        if transport is None:
            transport = LoopbackTransport() if world == 1 else ProcessGroupTransport()
        self.transport = transport
        self.overlap = bool(overlap)
        self._pending = None

    # -- exchange --------------------------------------------------------------

    def _exchange(self, f: torch.Tensor) -> None:
        if self.transport == "external":
            return
        self._pending = self.transport.start(self.geom, f)

    def _land(self) -> None:
        if self.transport != "external" and self._pending is not None:
            self.transport.wait(self._pending)
        self._pending = None

    def _planes(self, d, src, dst, force, z0: int, nz: int, status=True) -> None:
        st = _lib.load().tlbm_step_planes(ctypes.byref(d), src.data_ptr(), dst.data_ptr(), _lib.ptr(self.flags),
                                          _lib.ptr(self.tau_field), _lib.ptr(force),
                                          self.status.data_ptr() if status else None, z0, nz, self._stream())
        _lib.check(st, "tlbm_step_planes")

    def _launch(self, src: torch.Tensor, dst: torch.Tensor, force: torch.Tensor | None) -> None:
        n = self.geom.nz_local
        self._land()                                   # src's ghost planes are complete
        if self.overlap and n > 2 and self.transport != "external":
            self._planes(self._desc, src, dst, force, 1, 1)
            self._planes(self._desc, src, dst, force, n, 1)
            self._exchange(dst)
            self._planes(self._desc, src, dst, force, 2, n - 2)
        else:
            self._planes(self._desc, src, dst, force, 1, n)
            self._exchange(dst)

    # -- state -----------------------------------------------------------------

    def load(self, f: torch.Tensor) -> "SlabSolver":
        """Set S_0 from the GLOBAL field (Q, nz_global, ny, nx) (sliced with
        its ghost planes, so no exchange is needed) or from this slab's owned
        planes (Q, nz_local, ny, nx) (ghosts exchanged after the load)."""
        g = self.geom
        if tuple(f.shape) == (g.q, g.nz_global, g.ny, g.nx):
            super().load(g.local_from_global(f, dim=1))
            return self
        if tuple(f.shape) != (g.q, g.nz_local, g.ny, g.nx):
            raise ValueError(f"f shape {tuple(f.shape)} is neither the global {(g.q, g.nz_global, g.ny, g.nx)} "
                             f"nor the owned {(g.q, g.nz_local, g.ny, g.nx)} field")
        padded = torch.zeros(g.local_shape, dtype=f.dtype, device=f.device)
        padded[:, 1:g.nz_local + 1] = f
        super().load(padded)
        self._f0 = padded                               # ghost planes of S_0 are not known here
        if self.transport == "external":
            return self
        self._exchange(self._buf[0])
        self._land()
        return self

    def run(self, n: int, *, graph: bool = False, chunk: int = 50) -> "SlabSolver":
        """n eager steps (the exchange is posted on the host every step)."""
        return self.step(n)

    @property
    def f_local(self) -> torch.Tensor:
        """S_n on the padded local grid (ghost planes unspecified)."""
        self._land()
        if self.steps_done == 0:
            return self._f0.clone()
        out = torch.empty((self.q,) + self.cfg.shape, dtype=self.compute_dtype, device=self.device)
        prev = self._buf[1 - self._cur]
        if self.storage in ("f32", "f64"):
            self._planes(self._desc_none, prev, out, None, 1, self.geom.nz_local, status=False)
            return out
        tmp = torch.empty_like(prev)
        self._planes(self._desc_none, prev, tmp, None, 1, self.geom.nz_local, status=False)
        conv = self.cfg.desc(self.code, "none")
        _lib.check(_lib.load().tlbm_collide(ctypes.byref(conv), _lib.F32, tmp.data_ptr(), out.data_ptr(), None,
                                            None, self._stream()), "convert")
        return out

    @property
    def f(self) -> torch.Tensor:
        """This slab's owned planes of S_n, (Q, nz_local, ny, nx)."""
        return self.f_local[:, 1:self.geom.nz_local + 1].contiguous()

    def moment_sums(self) -> torch.Tensor:
        """float64 (mass, jx, jy, jz) of this slab's owned stored planes."""
        from . import _ops
        owned = self.state[:, 1:self.geom.nz_local + 1].contiguous()
        return _ops.moment_sums(self.q, owned, self.code)

    def synchronize(self) -> None:
        """Land the exchange in flight (a no-op when there is none)."""
        self._land()

    def global_force_history(self) -> torch.Tensor:
        """The float64 force of every recorded step summed over all slabs
        (an all-reduce over the process group; this slab's history alone
        when there is one slab)."""
        h = self.force_history().contiguous()
        if isinstance(self.transport, ProcessGroupTransport) and self.geom.world > 1:
            dist.all_reduce(h, group=self.transport.group)
        return h

    def global_nonfinite_seen(self) -> bool:
        flag = self.status.clone()
        if isinstance(self.transport, ProcessGroupTransport) and self.geom.world > 1:
            dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=self.transport.group)
        return bool(flag.item() != 0)


class MultiSlabSolver:
    """Several z-slabs driven by one process, each on its own device (or all on
    one): TensorLBM's single-process multi-device solver
    (multi_gpu.py:672 ``MultiDeviceSolver3D``) on the slab step.  Every step
    launches each slab, then copies the crossing lanes between them; with
    slabs on different devices the host synchronises the devices around the
    copies."""

    def __init__(self, lattice, global_shape, tau: float, collision: str = "bgk", *, devices=("cuda:0",),
                 n_slabs: int | None = None, **kw):
        devices = [torch.device(d) for d in devices]
        n = int(n_slabs or len(devices))
        self.devices = [devices[k % len(devices)] for k in range(n)]
        self.slabs = [SlabSolver(lattice, global_shape, tau, collision, device=self.devices[k], world=n, rank=k,
                                 transport="external", **kw) for k in range(n)]
        self.geom = [s.geom for s in self.slabs]
        self._multi_device = len(set(self.devices)) > 1

    def _sync(self) -> None:
        if self._multi_device:
            for d in set(self.devices):
                torch.cuda.synchronize(d)

    def load(self, f_global: torch.Tensor) -> "MultiSlabSolver":
        for s in self.slabs:
            s.load(f_global.to(s.device))
        return self

    def step(self, n: int = 1) -> "MultiSlabSolver":
        for _ in range(n):
            for s in self.slabs:
                s.step(1)
            self._sync()
            exchange_ring(self.geom, [s._buf[s._cur] for s in self.slabs])
            self._sync()
        return self

    def gather(self) -> torch.Tensor:
        """S_n of the whole domain on the first slab's device."""
        return torch.cat([s.f.to(self.devices[0]) for s in self.slabs], dim=1)

    def force_history(self) -> torch.Tensor:
        """float64 force per step summed over the slabs."""
        return sum(s.force_history().to(self.devices[0]) for s in self.slabs)

    def nonfinite_seen(self) -> bool:
        return any(s.nonfinite_seen() for s in self.slabs)

    @property
    def n_devices(self) -> int:
        return len(set(self.devices))
