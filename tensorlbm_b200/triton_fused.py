"""Drop-in for ``tensorlbm.triton_fused`` (triton_fused.py): the periodic D3Q19
pull + BGK step ``collide(stream(f))``, its two halves and the solver class,
on this library's fused CUDA kernel instead of a Triton kernel.

float32 storage is bit-exact with TensorLBM's torch path (``collide_bgk3d``
after ``stream3d``).  float16 / bfloat16 hold f itself, computed in float32 and
rounded to nearest on store, like the reduced-precision storage of the Triton
kernel (triton_fused.py:440-522); for long runs the shifted formats of
``LBMSolver(storage="f16" | "bf16")`` keep far more precision.  The tile
arguments of the Triton launchers are accepted and ignored.
"""

from __future__ import annotations

import ctypes
import time

import torch

from . import _lib, _ops

_Q = 19
DEFAULT_BLOCK_X = 32
DEFAULT_BLOCK_Y = 4
DEFAULT_NUM_WARPS = 4
DEFAULT_NUM_STAGES = 2
_CODES = {torch.float32: _lib.F32, torch.float16: _lib.F16, torch.bfloat16: _lib.BF16}
# TensorLBM precision-policy names (precision.py:72-158) with float32 compute
_POLICY_STORE = {"FP32FP32": torch.float32, "FP32FP16": torch.float16, "FP32BF16": torch.bfloat16}


def is_available() -> bool:
    """True when the CUDA library loads and a CUDA device is visible."""
    try:
        _lib.load()
    except (OSError, RuntimeError):
        return False
    return torch.cuda.is_available()


def _run(f: torch.Tensor, out: torch.Tensor | None, collision: int, tau: float, pull: bool) -> torch.Tensor:
    dev = _lib.require_cuda(f)
    if f.dim() != 4 or f.shape[0] != _Q:
        raise ValueError(f"expected a (19, nz, ny, nx) D3Q19 field, got {tuple(f.shape)}")
    code = _CODES.get(f.dtype)
    if code is None:
        raise ValueError(f"Unsupported dtype {f.dtype}; use float32, float16, or bfloat16.")
    f = f.contiguous()
    if out is None:
        out = torch.empty_like(f)
    elif tuple(out.shape) != tuple(f.shape) or out.dtype != f.dtype or not out.is_contiguous():
        raise ValueError("out must be a contiguous tensor of f's shape and dtype")
    _, nz, ny, nx = f.shape
    if f.numel() == 0:
        return out
    d = _ops.make_desc(_Q, (nx, ny, nz), code, collision, tau)
    lib = _lib.load()
    if pull:
        st = lib.tlbm_step(ctypes.byref(d), f.data_ptr(), out.data_ptr(), None, None, None, None,
                           _lib.stream_of(dev))
    else:
        st = lib.tlbm_collide(ctypes.byref(d), code, f.data_ptr(), out.data_ptr(), None, None, _lib.stream_of(dev))
    _lib.check(st, "triton_fused")
    return out


def triton_collide(f: torch.Tensor, tau: float, *, out: torch.Tensor | None = None, block_x: int = DEFAULT_BLOCK_X,
                   block_y: int = DEFAULT_BLOCK_Y, num_warps: int = DEFAULT_NUM_WARPS,
                   num_stages: int = DEFAULT_NUM_STAGES) -> torch.Tensor:
    """BGK collision only (triton_fused.py:534)."""
    return _run(f, out, _lib.COLL_BGK, tau, False)


def triton_stream(f: torch.Tensor, *, out: torch.Tensor | None = None, block_x: int = DEFAULT_BLOCK_X,
                  block_y: int = DEFAULT_BLOCK_Y, num_warps: int = DEFAULT_NUM_WARPS,
                  num_stages: int = DEFAULT_NUM_STAGES) -> torch.Tensor:
    """Periodic pull streaming, bit-exact with torch.roll (triton_fused.py:576)."""
    return _run(f, out, _lib.COLL_NONE, 1.0, True)


def triton_fused(f: torch.Tensor, tau: float, *, out: torch.Tensor | None = None, block_x: int = DEFAULT_BLOCK_X,
                 block_y: int = DEFAULT_BLOCK_Y, num_warps: int = DEFAULT_NUM_WARPS,
                 num_stages: int = DEFAULT_NUM_STAGES) -> torch.Tensor:
    """Periodic pull + BGK in one kernel: collide(stream(f)) (triton_fused.py:618).
    ``out`` must not alias ``f`` (the pull reads neighbours)."""
    return _run(f, out, _lib.COLL_BGK, tau, True)


class TritonFusedSolver3D:
    """Periodic D3Q19 BGK stepper with the surface of TensorLBM's
    ``TritonFusedSolver3D`` (triton_fused.py:676-960): two persistent
    ping-pong buffers, ``step(f)``, ``run(f, n)``, ``benchmark()``.

    ``dtype`` is the storage dtype (float32 / float16 / bfloat16);
    ``precision`` a TensorLBM precision policy or its name (float32 compute
    tiers only), the alternative way to pick it."""

    _Q = _Q

    def __init__(self, nz: int, ny: int, nx: int, tau: float, device="cuda", dtype: torch.dtype | None = None,
                 precision=None, block_x: int = DEFAULT_BLOCK_X, block_y: int = DEFAULT_BLOCK_Y,
                 num_warps: int = DEFAULT_NUM_WARPS, num_stages: int = DEFAULT_NUM_STAGES, **_unused):
        self.precision_policy = None
        if precision is not None:
            name = getattr(precision, "name", precision)
            if not isinstance(name, str):
                raise TypeError(f"precision must be a policy or its name, got {type(precision).__name__}")
            if name.upper().startswith("FP64"):
                raise NotImplementedError(f"precision {name}: the fused kernel computes in float32")
            store = _POLICY_STORE.get(name.upper())
            if store is None:
                raise ValueError(f"Unknown precision policy {name!r}; valid names: {sorted(_POLICY_STORE)}")
            if dtype is not None and dtype != store:
                raise ValueError(f"dtype={dtype} conflicts with precision={name} (store dtype {store}); pass only one.")
            dtype = store
            self.precision_policy = precision
        dtype = torch.float32 if dtype is None else dtype
        if dtype not in _CODES:
            raise ValueError(f"Unsupported dtype {dtype}; use float32, float16, or bfloat16.")
        self.nz, self.ny, self.nx = int(nz), int(ny), int(nx)
        self.tau = float(tau)
        self.device = _ops.cuda_device(device)
        self.dtype = dtype
        self.block_x, self.block_y, self.num_warps, self.num_stages = block_x, block_y, num_warps, num_stages
        self._desc = _ops.make_desc(_Q, (self.nx, self.ny, self.nz), _CODES[dtype], _lib.COLL_BGK, self.tau)
        self._buf_a: torch.Tensor | None = None
        self._buf_b: torch.Tensor | None = None
        self._report_step = 0

    def step(self, f: torch.Tensor) -> torch.Tensor:
        """One step into the internal buffer that is not ``f``."""
        if f.dtype != self.dtype:
            raise ValueError(f"step() input dtype {f.dtype} does not match the solver's storage dtype {self.dtype}")
        if tuple(f.shape) != (_Q, self.nz, self.ny, self.nx):
            raise ValueError(f"f shape {tuple(f.shape)} != {(_Q, self.nz, self.ny, self.nx)}")
        _lib.require_cuda(f)
        f = f.contiguous()
        if self._buf_a is None or self._buf_a.shape != f.shape or self._buf_a.dtype != f.dtype:
            self._buf_a = torch.empty_like(f)
            self._buf_b = torch.empty_like(f)
        out = self._buf_b if f.data_ptr() == self._buf_a.data_ptr() else self._buf_a
        st = _lib.load().tlbm_step(ctypes.byref(self._desc), f.data_ptr(), out.data_ptr(), None, None, None, None,
                                   _lib.stream_of(self.device))
        _lib.check(st, "TritonFusedSolver3D.step")
        return out

    def run(self, f: torch.Tensor, n_steps: int, *, reporters=None) -> tuple[torch.Tensor, list[dict]]:
        """n_steps steps; returns (f, one empty diagnostics dict per step)."""
        if reporters:
            raise NotImplementedError("reporters are TensorLBM's runner layer; run without them")
        for _ in range(int(n_steps)):
            f = self.step(f)
        self._report_step += int(n_steps)
        return f, [{} for _ in range(int(n_steps))]

    def grid_size_cells(self) -> int:
        return self.nz * self.ny * self.nx

    def transient_memory_bytes(self) -> int:
        """Two population buffers."""
        return 2 * self.grid_size_cells() * _Q * self.dtype.itemsize

    def benchmark(self, n_steps: int = 100, warmup: int = 5) -> float:
        """Seconds per step() call, host-timed like the reference's helper."""
        f = torch.zeros(_Q, self.nz, self.ny, self.nx, dtype=self.dtype, device=self.device)
        f += 1e-3 * torch.randn_like(f)
        for _ in range(warmup):
            f = self.step(f)
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        for _ in range(n_steps):
            f = self.step(f)
        torch.cuda.synchronize(self.device)
        return (time.perf_counter() - t0) / n_steps
