"""Training of the 3-D closure with the library's own kernels (the counterpart
of ai/train.py:310 train_eddy_viscosity_model: Adam on a weighted MSE).

One step = tlbm_mlp_grad (forward + backward of every mini-batch row, fp32,
per-block partial gradients) + tlbm_mlp_adam (block-ordered reduction and the
Adam update), so the result is deterministic for a given seed."""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch

from .. import _lib
from .model import EddyViscosityMLP3D


@dataclass
class TrainConfig:
    epochs: int = 20
    batch: int = 8192
    lr: float = 2e-3
    lr_final: float = 2e-4        # cosine decay to this
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8
    seed: int = 0
    val_fraction: float = 0.1


def train_eddy_viscosity_model3d(model: EddyViscosityMLP3D, x: torch.Tensor, target: torch.Tensor,
                                 weight: torch.Tensor | None = None, cfg: TrainConfig | None = None,
                                 set_stats: bool = True) -> dict:
    """Fit nu_t = nu_scale softplus(y(x)) to target by Adam on
    sum w (softplus(y) - t / nu_scale)^2 / batch.

    ``weight`` (default 1) is normalised to mean 1 over the data.  With
    set_stats the feature statistics, fallback range and nu_scale (the
    weighted mean target) are taken from x and target.  Returns the history
    {"train_loss": [...per epoch], "val_loss": [...]}."""
    cfg = cfg or TrainConfig()
    dev = model.device
    lib = _lib.load()
    x = x.to(dev, torch.float32).contiguous()
    n = x.shape[0]
    if target.shape != (n,):
        raise ValueError(f"target must have shape ({n},), got {tuple(target.shape)}")
    t = target.to(dev, torch.float32)
    w = torch.ones(n, dtype=torch.float32, device=dev) if weight is None else weight.to(dev, torch.float32)
    w = (w / w.mean().clamp_min(1e-30)).contiguous()
    if set_stats:
        model.set_feature_stats(x)
        model.nu_scale = float((t * w).sum().abs() / w.sum()) or 1.0
    ts = (t / model.nu_scale).contiguous()
    g = torch.Generator(device="cpu").manual_seed(cfg.seed)
    perm = torch.randperm(n, generator=g).to(dev)
    n_val = int(n * cfg.val_fraction)
    val_idx, train_idx = perm[:n_val].contiguous(), perm[n_val:].contiguous()
    n_train = train_idx.numel()
    m = torch.zeros_like(model.theta)
    v = torch.zeros_like(model.theta)
    blocks_max = int(lib.tlbm_mlp_grad_blocks(max(cfg.batch, 1)))
    partial = torch.empty(blocks_max * (model.theta.numel() + 1), dtype=torch.float32, device=dev)
    loss_buf = torch.zeros(1, dtype=torch.float32, device=dev)
    stream = _lib.stream_of(dev)
    istd = model.istd
    steps_per_epoch = max(1, (n_train + cfg.batch - 1) // cfg.batch)
    total = cfg.epochs * steps_per_epoch
    hist = {"train_loss": [], "val_loss": []}
    step = 0
    for _epoch in range(cfg.epochs):
        order = train_idx[torch.randperm(n_train, generator=g).to(dev)].contiguous()
        ep_loss = torch.zeros(1, dtype=torch.float64, device=dev)
        for b0 in range(0, n_train, cfg.batch):
            idx = order[b0:b0 + cfg.batch]
            cnt = idx.numel()
            step += 1
            lr = cfg.lr_final + 0.5 * (cfg.lr - cfg.lr_final) * (1 + math.cos(math.pi * (step - 1) / max(total, 1)))
            _lib.check(lib.tlbm_mlp_grad(model.theta.data_ptr(), model.mean.data_ptr(), istd.data_ptr(), x.data_ptr(),
                                         ts.data_ptr(), w.data_ptr(), idx.data_ptr(), cnt, partial.data_ptr(), stream),
                       "mlp_grad")
            nb = int(lib.tlbm_mlp_grad_blocks(cnt))
            _lib.check(lib.tlbm_mlp_adam(model.theta.data_ptr(), m.data_ptr(), v.data_ptr(), partial.data_ptr(), nb, lr,
                                         cfg.beta1, cfg.beta2, cfg.eps, step, None, loss_buf.data_ptr(), stream),
                       "mlp_adam")
            ep_loss += loss_buf.double() * cnt
        hist["train_loss"].append(float(ep_loss.item()) / max(n_train, 1))
        hist["val_loss"].append(loss_on(model, x, ts, w, val_idx) if n_val else float("nan"))
    model.invalidate()
    return hist


def loss_on(model: EddyViscosityMLP3D, x: torch.Tensor, ts: torch.Tensor, w: torch.Tensor, idx: torch.Tensor) -> float:
    """Weighted MSE (in nu_scale units) of the current parameters on rows idx (no update)."""
    lib = _lib.load()
    dev = model.device
    cnt = idx.numel()
    nb = int(lib.tlbm_mlp_grad_blocks(cnt))
    partial = torch.empty(nb * (model.theta.numel() + 1), dtype=torch.float32, device=dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    zeros = torch.zeros_like(model.theta)
    stream = _lib.stream_of(dev)
    _lib.check(lib.tlbm_mlp_grad(model.theta.data_ptr(), model.mean.data_ptr(), model.istd.data_ptr(), x.data_ptr(),
                                 ts.data_ptr(), w.data_ptr(), idx.data_ptr(), cnt, partial.data_ptr(), stream),
               "mlp_grad")
    _lib.check(lib.tlbm_mlp_adam(model.theta.data_ptr(), zeros.data_ptr(), zeros.clone().data_ptr(),
                                 partial.data_ptr(), nb, 0.0, 0.9, 0.999, 1e-8, 1, None, loss.data_ptr(), stream),
               "mlp_adam")
    return float(loss.item())
