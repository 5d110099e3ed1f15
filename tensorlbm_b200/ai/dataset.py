"""Training data of the 3-D closure from DNS populations (ai/dataset.py and
ai/pipeline.py:93 _coarsen_mean are the 2-D originals).

filtered_moments: block means (factor^3) of rho, u and u_i u_j of a D3Q19
population field; les_samples: the nine Pi-invariant features the coarse LES
will see, the subgrid target nu* = -(tau_sgs_dev : S) / (2 S:S) and the weight
S:S.  Both are kernels of libtlbm."""

from __future__ import annotations

import torch

from .. import _lib, _ops

N_MOMENTS = 10


def filtered_moments(f: torch.Tensor, factor: int, force_lin: float = 0.0) -> torch.Tensor:
    """(10, nz/f, ny/f, nx/f) float32 block means of rho, ux, uy, uz, uxux,
    uyuy, uzuz, uxuy, uxuz, uyuz of a (19, nz, ny, nx) float32 field."""
    dev = _lib.require_cuda(f)
    nx, ny, nz = _ops.grid_of(f, 19)
    if f.dtype != torch.float32:
        raise ValueError("filtered_moments expects float32 populations")
    f = f.contiguous()
    if factor < 1 or nx % factor or ny % factor or nz % factor:
        raise ValueError(f"factor {factor} does not divide the grid {(nz, ny, nx)}")
    out = torch.empty((N_MOMENTS, nz // factor, ny // factor, nx // factor), dtype=torch.float32, device=dev)
    _lib.check(_lib.load().tlbm_les_filter_moments(f.data_ptr(), nx, ny, nz, factor, float(force_lin),
                                                   out.data_ptr(), _lib.stream_of(dev)), "les_filter_moments")
    return out


def les_samples(moments: torch.Tensor, tau0: float, c_s: float = 0.17, nu_hat: torch.Tensor | None = None):
    """(features (N, 9), target (N,), weight (N,)) of one filtered field.

    tau0 is the molecular relaxation time on the filtered grid.  nu_hat (per
    filtered cell) sets the tau_eff with which the LES would have produced the
    stress Pi; None uses the Smagorinsky tau of c_s."""
    dev = _lib.require_cuda(moments, nu_hat)
    if moments.ndim != 4 or moments.shape[0] != N_MOMENTS or moments.dtype != torch.float32:
        raise ValueError("moments must be a (10, nz, ny, nx) float32 tensor")
    _, nz, ny, nx = moments.shape
    n = nx * ny * nz
    mom = moments.contiguous()
    nh = None
    if nu_hat is not None:
        if nu_hat.numel() != n:
            raise ValueError(f"nu_hat must have {n} entries")
        nh = nu_hat.to(dev, torch.float32).contiguous()
    x = torch.empty((n, 9), dtype=torch.float32, device=dev)
    t = torch.empty(n, dtype=torch.float32, device=dev)
    w = torch.empty(n, dtype=torch.float32, device=dev)
    _lib.check(_lib.load().tlbm_les_samples(mom.data_ptr(), nx, ny, nz, float(tau0), float(c_s), _lib.ptr(nh),
                                            x.data_ptr(), t.data_ptr(), w.data_ptr(), _lib.stream_of(dev)),
               "les_samples")
    return x, t, w
