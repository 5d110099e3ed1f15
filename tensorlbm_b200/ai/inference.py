"""The fused learned-closure LES step (ai/inference.py:68-92
collide_ai_les_bgk is the 2-D original: tau + 3 nu_t from an MLP, then BGK).

LearnedLESSolver advances a periodic D3Q19 box: each launch of tlbm_les_step
pulls, evaluates the network on the tensor cores, relaxes with tau_eff (the
Smagorinsky tau outside the training range) and adds the linear forcing.  The
stored state is the post-collision population field."""

from __future__ import annotations

import torch

from .. import _lib, _ops
from .model import EddyViscosityMLP3D


class LearnedLESSolver:
    def __init__(self, shape, tau0: float, model: EddyViscosityMLP3D, *, force_lin: float = 0.0,
                 c_s: float = 0.17, device=None, track_tau: bool = False):
        nz, ny, nx = (int(s) for s in shape)
        self.shape = (nz, ny, nx)
        self.tau0 = float(tau0)
        if not self.tau0 > 0.5:
            raise ValueError("tau0 must exceed 0.5")
        self.model = model
        self.force_lin = float(force_lin)
        self.c_s = float(c_s)
        self.device = _ops.cuda_device(device if device is not None else model.device)
        full = (19, nz, ny, nx)
        self._buf = [torch.empty(full, dtype=torch.float32, device=self.device) for _ in range(2)]
        self._cur = 0
        self.steps_done = 0
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.fallback = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.tau = torch.empty((nz, ny, nx), dtype=torch.float32, device=self.device) if track_tau else None
        self._graph = None

    def set_force_lin(self, a: float) -> "LearnedLESSolver":
        """Change the linear body force A (drops the captured graph)."""
        self.force_lin = float(a)
        self._graph = None
        return self

    def load(self, f: torch.Tensor) -> "LearnedLESSolver":
        """Set the post-collision state (19, nz, ny, nx)."""
        if tuple(f.shape) != (19,) + self.shape:
            raise ValueError(f"f shape {tuple(f.shape)} != {(19,) + self.shape}")
        self._buf[0].copy_(f.to(self.device, torch.float32))
        self._cur = 0
        self.steps_done = 0
        self._graph = None
        return self

    def _launch(self, src: torch.Tensor, dst: torch.Tensor) -> None:
        nz, ny, nx = self.shape
        st = _lib.load().tlbm_les_step(nx, ny, nz, self.tau0, self.c_s, self.force_lin, self.model.pack().data_ptr(),
                                       src.data_ptr(), dst.data_ptr(), _lib.ptr(self.tau), self.fallback.data_ptr(),
                                       self.status.data_ptr(), _lib.stream_of(self.device))
        _lib.check(st, "les_step")

    def step(self, n: int = 1) -> "LearnedLESSolver":
        for _ in range(n):
            self._launch(self._buf[self._cur], self._buf[1 - self._cur])
            self._cur ^= 1
            self.steps_done += 1
        return self

    def run(self, n: int, chunk: int = 50) -> "LearnedLESSolver":
        """n steps, replaying a CUDA graph of `chunk` launches (the first launch
        of a solver runs eagerly: it sets the kernel's shared-memory limit)."""
        if self.steps_done == 0 and n > 0:
            self.step(1)
            n -= 1
        while n >= chunk and chunk > 1:
            if self._graph is None or self._graph[1] != self._cur:
                self.model.pack()
                g = torch.cuda.CUDAGraph()
                s = torch.cuda.Stream(self.device)
                s.wait_stream(torch.cuda.current_stream(self.device))
                cur0 = self._cur
                with torch.cuda.stream(s):
                    with torch.cuda.graph(g, stream=s):
                        c = cur0
                        for _ in range(chunk):
                            self._launch(self._buf[c], self._buf[1 - c])
                            c ^= 1
                torch.cuda.current_stream(self.device).wait_stream(s)
                self._graph = (g, cur0)
            self._graph[0].replay()
            self._cur ^= chunk & 1
            self.steps_done += chunk
            n -= chunk
            if chunk & 1:
                self._graph = None
        return self.step(n)

    @property
    def state(self) -> torch.Tensor:
        return self._buf[self._cur]

    def velocity(self) -> torch.Tensor:
        """(3, nz, ny, nx) velocity of the stored state."""
        from ..d3q19 import macroscopic3d

        _, ux, uy, uz = macroscopic3d(self.state)
        return torch.stack([ux, uy, uz])

    def nonfinite_seen(self) -> bool:
        return bool(int(self.status.item()) & 1)
