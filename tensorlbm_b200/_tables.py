"""torch views of the lattice tables (C, W, W_EXACT64, OPPOSITE) per lattice."""

from __future__ import annotations

import torch

from . import lattice as _lat


def tables(lat: _lat.Lattice):
    c = torch.tensor(lat.c[:, : lat.dim].tolist(), dtype=torch.int64)
    w = torch.tensor(lat.w64.tolist(), dtype=torch.float32)
    w64 = torch.tensor(lat.w64.tolist(), dtype=torch.float64)
    opp = torch.tensor(lat.opp.tolist(), dtype=torch.int64)
    return c, w, w64, opp
