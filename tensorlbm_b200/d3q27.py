"""D3Q27 lattice: tables and operators (tensorlbm/d3q27.py:32-811)."""

from __future__ import annotations

import torch

from . import _lib, _ops
from . import lattice as _lat
from ._tables import tables

C, W, W_EXACT64, OPPOSITE = tables(_lat.D3Q27)
WEIGHT_PRECISION_SCHEME = "rational_binary64_cast_to_runtime_dtype_v1"


def equilibrium27(rho, ux, uy, uz, device=None, *, out: torch.Tensor | None = None) -> torch.Tensor:
    """tensorlbm/d3q27.py:353."""
    return _ops.equilibrium(27, rho, ux, uy, uz, out=out)


def macroscopic27(f: torch.Tensor, device=None):
    """tensorlbm/d3q27.py:395."""
    return _ops.macroscopic(27, f)


def collide_bgk27(f: torch.Tensor, tau: float) -> torch.Tensor:
    """tensorlbm/d3q27.py:423."""
    return _ops.collide(27, f, _lib.COLL_BGK, tau)


def collide_trt27(f: torch.Tensor, tau_plus: float, lambda_trt: float = 3.0 / 16.0) -> torch.Tensor:
    """Two-relaxation-time collision, bit-exact.  tensorlbm/d3q27.py:438."""
    return _ops.collide(27, f, _lib.COLL_TRT, tau_plus, lambda_trt=lambda_trt)


def collide_rlbm27(f: torch.Tensor, tau: float) -> torch.Tensor:
    """Regularised BGK (Latt & Chopard 2006), bit-exact.  tensorlbm/d3q27.py:481."""
    return _ops.collide(27, f, _lib.COLL_RLBM, tau)


def collide_mrt27(f: torch.Tensor, tau: float, s_e: float = 1.19, s_eps: float = 1.4, s_q: float = 1.2,
                  s_pi: float | None = None) -> torch.Tensor:
    """Gram-Schmidt 27x27 MRT, tensorlbm/d3q27.py:643."""
    return _ops.collide(27, f, _lib.COLL_MRT, tau, s_e=s_e, s_eps=s_eps, s_q=s_q, s_pi=s_pi)


def correct_mass27(f: torch.Tensor, target_mass: float) -> torch.Tensor:
    """tensorlbm/d3q27.py:729."""
    return _ops.correct_mass(f, target_mass)


def stream27_roll(f: torch.Tensor) -> torch.Tensor:
    """Periodic streaming, tensorlbm/d3q27.py:766."""
    return _ops.stream(27, f)


stream27 = stream27_roll

__all__ = ["C", "W", "W_EXACT64", "OPPOSITE", "equilibrium27", "macroscopic27", "collide_bgk27",
           "collide_mrt27", "collide_rlbm27", "collide_trt27", "correct_mass27", "stream27", "stream27_roll"]
