"""The 3-D eddy-viscosity MLP (ai/model.py:40-92 is the 2-D original).

9 invariant features of the non-equilibrium stress -> 64 -> 64 -> 64 (SiLU)
-> 1; nu_t = nu_scale * softplus(y).  Parameters live on the GPU as one flat
float32 vector (the training layout of libtlbm: W1 (64x9), b1, W2, b2, W3, b3,
w4, b4).  ``pack()`` produces the bf16 tensor-core blob used by the fused LES
step; ``forward`` (fp32, CUDA cores) and ``infer`` (tcgen05) return y."""

from __future__ import annotations

import math

import numpy as np
import torch

from .. import _lib, _ops

N_FEATURES = 9
HIDDEN = 64


def param_count() -> int:
    return int(_lib.load().tlbm_mlp_param_count())


class EddyViscosityMLP3D:
    """Parameters, feature statistics and training range of the closure."""

    def __init__(self, device=None, seed: int = 0):
        self.device = _ops.cuda_device(device)
        n = param_count()
        self.theta = torch.from_numpy(_init(seed)).to(self.device)
        if self.theta.numel() != n:
            raise RuntimeError(f"libtlbm expects {n} parameters, the initialiser made {self.theta.numel()}")
        self.mean = torch.zeros(N_FEATURES, dtype=torch.float32, device=self.device)
        self.std = torch.ones(N_FEATURES, dtype=torch.float32, device=self.device)
        self.lo = torch.full((N_FEATURES,), -math.inf, dtype=torch.float32, device=self.device)
        self.hi = torch.full((N_FEATURES,), math.inf, dtype=torch.float32, device=self.device)
        self.nu_scale = 1.0
        self._blob: torch.Tensor | None = None

    # -- statistics -------------------------------------------------------------
    def set_feature_stats(self, x: torch.Tensor, margin: float = 0.05) -> None:
        """Normalisation (mean, std) and the fallback range [lo, hi] (the
        training min / max widened by margin x span, at least 1e-6 relative so
        that a constant feature keeps a band that float32 rounding stays in)."""
        x = x.to(self.device, torch.float32)
        self.mean = x.mean(0).contiguous()
        self.std = x.std(0).clamp_min(1e-6).contiguous()
        lo, hi = x.min(0).values, x.max(0).values
        span = torch.maximum(hi - lo, 1e-6 * torch.maximum(lo.abs(), hi.abs()).clamp_min(1e-12))
        self.lo = (lo - margin * span).contiguous()
        self.hi = (hi + margin * span).contiguous()
        self._blob = None

    @property
    def istd(self) -> torch.Tensor:
        return (1.0 / self.std.clamp_min(1e-6)).contiguous()

    # -- evaluation -------------------------------------------------------------
    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """y of raw features (N, 9), float32 on the CUDA cores."""
        x = _features(x, self.device)
        y = torch.empty(x.shape[0], dtype=torch.float32, device=self.device)
        if x.shape[0]:
            _lib.check(_lib.load().tlbm_mlp_eval(self.theta.data_ptr(), self.mean.data_ptr(), self.istd.data_ptr(),
                                                 x.data_ptr(), x.shape[0], y.data_ptr(),
                                                 _lib.stream_of(self.device)), "mlp_eval")
        return y

    def nu_t(self, x: torch.Tensor) -> torch.Tensor:
        return self.nu_scale * torch.nn.functional.softplus(self.forward(x))

    def pack(self) -> torch.Tensor:
        """The tensor-core inference blob (bf16 swizzled weights + float block)."""
        if self._blob is None:
            nbytes = int(_lib.load().tlbm_mlp_blob_bytes())
            blob = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            _lib.check(_lib.load().tlbm_mlp_pack(self.theta.data_ptr(), self.mean.data_ptr(), self.std.data_ptr(),
                                                 self.lo.data_ptr(), self.hi.data_ptr(), float(self.nu_scale),
                                                 blob.data_ptr(), _lib.stream_of(self.device)), "mlp_pack")
            self._blob = blob
        return self._blob

    def infer(self, x: torch.Tensor) -> torch.Tensor:
        """y of raw features (N, 9) on the tensor cores (bf16 weights and layer
        inputs, fp32 accumulation): the arithmetic of the fused LES step."""
        x = _features(x, self.device)
        y = torch.empty(x.shape[0], dtype=torch.float32, device=self.device)
        status = torch.zeros(1, dtype=torch.int32, device=self.device)
        if x.shape[0]:
            _lib.check(_lib.load().tlbm_mlp_infer(self.pack().data_ptr(), x.data_ptr(), x.shape[0], y.data_ptr(),
                                                  status.data_ptr(), _lib.stream_of(self.device)), "mlp_infer")
        if int(status.item()) & 4:
            raise RuntimeError("tensor-core inference: a bounded wait expired")
        return y

    def invalidate(self) -> None:
        self._blob = None

    # -- persistence ------------------------------------------------------------
    def state_dict(self) -> dict:
        return {"theta": self.theta.cpu().numpy(), "mean": self.mean.cpu().numpy(), "std": self.std.cpu().numpy(),
                "lo": self.lo.cpu().numpy(), "hi": self.hi.cpu().numpy(), "nu_scale": np.float64(self.nu_scale)}

    def load_state_dict(self, d: dict) -> "EddyViscosityMLP3D":
        for k in ("theta", "mean", "std", "lo", "hi"):
            setattr(self, k, torch.as_tensor(np.asarray(d[k], np.float32)).to(self.device).contiguous())
        self.nu_scale = float(d["nu_scale"])
        self._blob = None
        return self

    def save(self, path) -> None:
        np.savez(path, **self.state_dict())

    @classmethod
    def load(cls, path, device=None) -> "EddyViscosityMLP3D":
        with np.load(path) as z:
            return cls(device).load_state_dict(dict(z))


def _features(x: torch.Tensor, device) -> torch.Tensor:
    if x.ndim != 2 or x.shape[1] != N_FEATURES:
        raise ValueError(f"features must have shape (N, {N_FEATURES}), got {tuple(x.shape)}")
    _lib.require_cuda(x)
    return x.to(device, torch.float32).contiguous()


def _init(seed: int) -> np.ndarray:
    """Kaiming-uniform weights for SiLU layers (output layer x0.5), zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for shape, fan_in, scale in (((HIDDEN, N_FEATURES), N_FEATURES, 1.0), ((HIDDEN,), 0, 0.0),
                                 ((HIDDEN, HIDDEN), HIDDEN, 1.0), ((HIDDEN,), 0, 0.0),
                                 ((HIDDEN, HIDDEN), HIDDEN, 1.0), ((HIDDEN,), 0, 0.0),
                                 ((HIDDEN,), HIDDEN, 0.5), ((1,), 0, 0.0)):
        if fan_in == 0:
            parts.append(np.zeros(shape))
        else:
            b = scale * math.sqrt(6.0 / fan_in)
            parts.append(rng.uniform(-b, b, size=shape))
    return np.concatenate([p.reshape(-1) for p in parts]).astype(np.float32)
