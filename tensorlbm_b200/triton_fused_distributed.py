"""Drop-in for ``tensorlbm.triton_fused_distributed``: the periodic D3Q19 BGK
step on z-slabs across ranks, with the halo exchange of the crossing lanes
(triton_fused_distributed.py:196-680), on this library's fused kernel.

Same surface: ``DistributedTritonFusedSolver3D(nz_global, ny, nx, tau,
device, halo_dtype=)`` with ``allocate``, ``from_global``, ``to_global``,
``step``, ``synchronize`` and the size helpers, ``crossing_face_indices``,
``init_distributed``, ``rank``, ``world_size``, ``distributed_is_available``.

Differences that change results or use:
- The kernel updates only the owned planes. The owned values after any
  number of steps equal the single-domain ``triton_fused`` run bit for bit
  (float32 wire).
- ``from_global`` fills the ghost planes from the neighbouring slabs'
  planes of the global field. The reference pre-fills them with copies of
  the nearest owned plane, so its first step differs at the slab faces.
- ``step`` returns one of two solver-owned buffers and accepts the
  returned one back (no aliasing; the reference needs an external
  ping-pong).
- The float32 exchange sends each crossing lane straight from the buffer
  (no staging). ``halo_dtype=torch.float16`` stages and casts, like the
  reference.
"""

from __future__ import annotations

import ctypes
import os

import torch
import torch.distributed as dist

from . import _lib, _ops
from .slabs import (LoopbackTransport, ProcessGroupTransport, SlabGeometry, StagedTransport,
                    crossing_face_indices)
from .triton_fused import DEFAULT_BLOCK_X, DEFAULT_BLOCK_Y, DEFAULT_NUM_STAGES, DEFAULT_NUM_WARPS

__all__ = [
    "DistributedTritonFusedSolver3D",
    "init_distributed",
    "distributed_is_available",
    "world_size",
    "rank",
    "crossing_face_indices",
]

_Q = 19


def distributed_is_available() -> bool:
    return dist.is_available()


def init_distributed(backend: str | None = None) -> tuple[int, int]:
    """Initialise the default group from RANK / WORLD_SIZE (no group for one
    rank); returns (rank, world_size) (triton_fused_distributed.py:152)."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    r = int(os.environ.get("RANK", "0"))
    w = int(os.environ.get("WORLD_SIZE", "1"))
    if w == 1:
        return r, w
    dist.init_process_group(backend=backend, rank=r, world_size=w)
    if backend == "nccl" and torch.cuda.is_available():
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", r)))
    return r, w


def rank() -> int:
    return dist.get_rank() if dist.is_available() and dist.is_initialized() else 0


def world_size() -> int:
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


class DistributedTritonFusedSolver3D:
    """Periodic D3Q19 BGK step on this rank's z-slab (see the module notes)."""

    def __init__(self, nz_global: int, ny: int, nx: int, tau: float, device="cuda:0", *,
                 block_x: int = DEFAULT_BLOCK_X, block_y: int = DEFAULT_BLOCK_Y, num_warps: int = DEFAULT_NUM_WARPS,
                 num_stages: int = DEFAULT_NUM_STAGES, halo_dtype: torch.dtype = torch.float32, group=None) -> None:
        self._rank, self._world = rank(), world_size()
        self.geom = SlabGeometry(_Q, nz_global, ny, nx, self._world, self._rank)
        self.nz_global, self.nz_local = self.geom.nz_global, self.geom.nz_local
        self.ny, self.nx = self.geom.ny, self.geom.nx
        self.nz_with_halo = self.nz_local + 2
        self.tau = float(tau)
        self.device = _ops.cuda_device(device)
        self.block_x, self.block_y, self.num_warps, self.num_stages = block_x, block_y, num_warps, num_stages
        self.z_start_global, self.z_end_global = self.geom.z_start_global, self.geom.z_end_global
        self.left_neighbor, self.right_neighbor = self.geom.left_neighbor, self.geom.right_neighbor
        self._cross_up, self._cross_dn = self.geom.cross_up, self.geom.cross_dn
        self.n_cross = self.geom.n_cross
        halo_dtype = torch.float32 if halo_dtype is None else halo_dtype
        if halo_dtype.itemsize not in (2, 4):
            raise ValueError(f"halo_dtype must be fp32 or fp16, got {halo_dtype}")
        self._halo_dtype = halo_dtype
        if self._world == 1:
            self._transport = LoopbackTransport()
        elif halo_dtype == torch.float32:
            self._transport = ProcessGroupTransport(group)
        else:
            self._transport = StagedTransport(halo_dtype, group)
        self._bufs: list[torch.Tensor] = []
        self._pending = None
        self._pending_target: torch.Tensor | None = None

    # -- shapes and buffers ------------------------------------------------------

    @property
    def local_shape(self) -> tuple[int, int, int, int]:
        return self.geom.local_shape

    def owned_slice(self) -> tuple[int, int]:
        return self.geom.owned_slice()

    def allocate(self, dtype: torch.dtype = torch.float32) -> torch.Tensor:
        """A new (uninitialised) local buffer with ghost planes."""
        return torch.empty(self.local_shape, dtype=dtype, device=self.device)

    def from_global(self, f_global: torch.Tensor) -> torch.Tensor:
        """This rank's owned planes of the global (19, nz_global, ny, nx) field
        with its ghost planes taken from the neighbouring slabs' planes."""
        if tuple(f_global.shape) != (_Q, self.nz_global, self.ny, self.nx):
            raise ValueError(f"f_global shape {tuple(f_global.shape)} does not match expected "
                             f"({_Q}, {self.nz_global}, {self.ny}, {self.nx})")
        return self.geom.local_from_global(f_global.to(self.device), dim=1)

    def to_global(self, f_local: torch.Tensor, f_global: torch.Tensor | None = None) -> torch.Tensor:
        """Write this rank's owned planes into the global field (other ranks'
        planes are left as they are)."""
        if f_global is None:
            f_global = torch.empty((_Q, self.nz_global, self.ny, self.nx), dtype=f_local.dtype, device=self.device)
        elif tuple(f_global.shape) != (_Q, self.nz_global, self.ny, self.nx):
            raise ValueError(f"f_global shape {tuple(f_global.shape)} does not match expected "
                             f"({_Q}, {self.nz_global}, {self.ny}, {self.nx})")
        f_global[:, self.z_start_global:self.z_end_global].copy_(f_local[:, 1:self.nz_local + 1])
        return f_global

    # -- step --------------------------------------------------------------------

    def _finalize_halo(self) -> None:
        if self._pending is not None:
            self._transport.wait(self._pending)
        self._pending = None
        self._pending_target = None

    def step(self, f_local: torch.Tensor) -> torch.Tensor:
        """One periodic BGK step of the owned planes of ``f_local`` (its ghost
        planes current); returns the new local buffer, whose ghost planes are
        being filled by the exchange (landed by the next step or
        :meth:`synchronize`)."""
        if tuple(f_local.shape) != self.local_shape:
            raise ValueError(f"f_local shape {tuple(f_local.shape)} does not match expected {self.local_shape}")
        code = {torch.float32: _lib.F32, torch.float16: _lib.F16, torch.bfloat16: _lib.BF16}.get(f_local.dtype)
        if code is None:
            raise ValueError(f"Unsupported dtype {f_local.dtype}; use float32, float16, or bfloat16.")
        dev = _lib.require_cuda(f_local)
        self._finalize_halo()                   # lands into the buffer returned last time
        f_local = f_local.contiguous()
        if len(self._bufs) != 2 or self._bufs[0].dtype != f_local.dtype or self._bufs[0].device != dev:
            self._bufs = [torch.empty_like(f_local) for _ in range(2)]
        out = self._bufs[1] if f_local.data_ptr() == self._bufs[0].data_ptr() else self._bufs[0]
        d = _ops.make_desc(_Q, (self.nx, self.ny, self.nz_with_halo), code, _lib.COLL_BGK, self.tau)
        lib = _lib.load()
        stream = _lib.stream_of(dev)
        n = self.nz_local
        # the two boundary planes, then the exchange of their lanes, which
        # runs while the interior planes are computed
        boundary = ((1, 1), (n, 1)) if n > 2 else ((1, n),)
        interior = ((2, n - 2),) if n > 2 else ()

        def launch(z0: int, nz: int) -> None:
            st = lib.tlbm_step_planes(ctypes.byref(d), f_local.data_ptr(), out.data_ptr(), None, None, None, None,
                                      z0, nz, stream)
            _lib.check(st, "DistributedTritonFusedSolver3D.step")

        for z0, nz in boundary:
            launch(z0, nz)
        self._pending = self._transport.start(self.geom, out)
        self._pending_target = out
        for z0, nz in interior:
            launch(z0, nz)
        return out

    def synchronize(self) -> None:
        """Land the exchange in flight (no-op when there is none)."""
        self._finalize_halo()

    # -- sizes -------------------------------------------------------------------

    def grid_size_cells(self) -> int:
        return self.nz_local * self.ny * self.nx

    @property
    def staging_shape(self) -> tuple[int, int, int]:
        return (self.n_cross, self.ny, self.nx)

    def staging_bytes(self) -> int:
        """Persistent staging: none for the float32 wire (lanes go straight
        from the buffer), four (n_cross, ny, nx) planes for a narrower wire."""
        if self._world == 1 or self._halo_dtype == torch.float32:
            return 0
        return 4 * self.n_cross * self.ny * self.nx * self._halo_dtype.itemsize

    def halo_bytes_per_step(self) -> int:
        """Bytes this rank sends per step (it receives as many)."""
        if self._world == 1:
            return 0
        return self.geom.halo_bytes_per_step(self._halo_dtype.itemsize)

    def transient_memory_bytes(self) -> int:
        """The two local buffers of (19, nz_local + 2, ny, nx) float32."""
        return 2 * _Q * self.nz_with_halo * self.ny * self.nx * 4
