"""Velocity sets, weights and moment bases of the D2Q9, D3Q19 and D3Q27 lattices.

The direction ORDER of each set is part of the public interface: populations are
stored as ``(Q, nz, ny, nx)`` (2-D: ``(Q, ny, nx)``) and callers index them by
direction number, so the order here is the one TensorLBM uses
(``tensorlbm/d2q9.py:8-26``, ``tensorlbm/d3q19.py:6-67``,
``tensorlbm/d3q27.py:32-84``).  Everything else (weights, opposites, moment
matrices) is derived from the velocity set by the functions below, never typed
by hand, so a sign slip in one table cannot disagree with another.

This module is numpy-only; it feeds both the CUDA code generator
(``csrc/gen_tables.py``) and the torch-facing lattice modules.
"""

from __future__ import annotations

from dataclasses import dataclass
from fractions import Fraction

import numpy as np

# --- velocity sets (order = interface) -------------------------------------

_D2Q9_C = [(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1)]

# rest, 6 faces (+x,-x,+y,-y,+z,-z), then the xy, xz, yz edge pairs
_D3Q19_C = [
    (0, 0, 0),
    (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
    (1, 1, 0), (-1, -1, 0), (1, -1, 0), (-1, 1, 0),
    (1, 0, 1), (-1, 0, -1), (1, 0, -1), (-1, 0, 1),
    (0, 1, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1),
]

# rest, 6 faces, 12 edges (xy, xz, yz blocks, x varying fastest), 8 corners
_D3Q27_C = [
    (0, 0, 0),
    (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
    (1, 1, 0), (-1, 1, 0), (1, -1, 0), (-1, -1, 0),
    (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1),
    (0, 1, 1), (0, -1, 1), (0, 1, -1), (0, -1, -1),
    (1, 1, 1), (-1, 1, 1), (1, -1, 1), (-1, -1, 1),
    (1, 1, -1), (-1, 1, -1), (1, -1, -1), (-1, -1, -1),
]


def _weight(c: tuple[int, ...], q: int) -> Fraction:
    """Standard weights by speed class |c|^2 for the three stencils."""
    n2 = sum(v * v for v in c)
    if q == 9:
        return [Fraction(4, 9), Fraction(1, 9), Fraction(1, 36)][n2]
    if q == 19:
        return [Fraction(1, 3), Fraction(1, 18), Fraction(1, 36)][n2]
    return [Fraction(8, 27), Fraction(2, 27), Fraction(1, 54), Fraction(1, 216)][n2]


@dataclass(frozen=True)
class Lattice:
    name: str
    q: int
    dim: int
    c: np.ndarray  # (Q, 3) int64, third column zero for D2Q9
    w: tuple[Fraction, ...]
    opp: np.ndarray  # (Q,) int64

    @property
    def w64(self) -> np.ndarray:
        return np.array([float(v) for v in self.w], dtype=np.float64)

    @property
    def w32(self) -> np.ndarray:
        return self.w64.astype(np.float32)


def _make(name: str, cs: list[tuple[int, ...]]) -> Lattice:
    q = len(cs)
    dim = len(cs[0])
    c = np.zeros((q, 3), dtype=np.int64)
    c[:, :dim] = np.array(cs, dtype=np.int64)
    w = tuple(_weight(tuple(row), q) for row in cs)
    assert sum(w) == 1
    index = {tuple(row): i for i, row in enumerate(c.tolist())}
    opp = np.array([index[tuple((-c[i]).tolist())] for i in range(q)], dtype=np.int64)
    return Lattice(name, q, dim, c, w, opp)


D2Q9 = _make("D2Q9", _D2Q9_C)
D3Q19 = _make("D3Q19", _D3Q19_C)
D3Q27 = _make("D3Q27", _D3Q27_C)
LATTICES = {9: D2Q9, 19: D3Q19, 27: D3Q27}


# --- MRT moment bases --------------------------------------------------------


def mrt_matrix_d2q9() -> np.ndarray:
    """Lallemand-Luo D2Q9 basis (rho, e, eps, jx, qx, jy, qy, pxx, pxy).

    Same rows as ``tensorlbm/solver.py:24-34``; built here from the velocity
    set so the row polynomials are explicit.
    """
    cx = D2Q9.c[:, 0].astype(np.float64)
    cy = D2Q9.c[:, 1].astype(np.float64)
    c2 = cx**2 + cy**2
    rows = [
        np.ones(9),
        3.0 * c2 - 4.0,
        (9.0 * c2**2 - 21.0 * c2 + 8.0) / 2.0,
        cx,
        (3.0 * c2 - 5.0) * cx,
        cy,
        (3.0 * c2 - 5.0) * cy,
        cx**2 - cy**2,
        cx * cy,
    ]
    return np.array(rows)


def mrt_matrix_d3q19() -> np.ndarray:
    """d'Humieres D3Q19 polynomial basis, rows as in ``tensorlbm/solver3d.py:24-55``."""
    cx, cy, cz = (D3Q19.c[:, k].astype(np.float64) for k in range(3))
    e2 = cx**2 + cy**2 + cz**2
    e4 = e2**2
    rows = [
        np.ones(19),
        19.0 * e2 - 30.0,
        (21.0 * e4 - 53.0 * e2 + 24.0) / 2.0,
        cx,
        cx * e2 * (5.0 * e2 - 9.0) / 2.0,
        cy,
        cy * e2 * (5.0 * e2 - 9.0) / 2.0,
        cz,
        cz * e2 * (5.0 * e2 - 9.0) / 2.0,
        3.0 * cx**2 - e2,
        cx**2 - cy**2,
        cx * cy,
        cx * cz,
        cy * cz,
        (3.0 * e2 - 5.0) * (3.0 * cx**2 - e2) / 2.0,
        (3.0 * e2 - 5.0) * (cx**2 - cy**2) / 2.0,
        cx**2 * cy,
        cx**2 * cz,
        cy**2 * cx,
    ]
    return np.array(rows)


def mrt_matrix_d3q27() -> np.ndarray:
    """D3Q27 basis: Gram-Schmidt over 27 raw monomials.

    The raw row list and the orthogonalisation order follow
    ``tensorlbm/d3q27.py:545-635``; the rows must come out identical because
    the relaxation vector addresses them by index.
    """
    cx, cy, cz = (D3Q27.c[:, k].astype(np.float64) for k in range(3))
    e2 = cx**2 + cy**2 + cz**2
    raw = [
        np.ones(27), cx, cy, cz, e2,
        3.0 * cx**2 - e2, cy**2 - cz**2, cx * cy, cx * cz, cy * cz,
        cx * e2, cy * e2, cz * e2,
        cx**2 * cy, cx**2 * cz, cy**2 * cx, cy**2 * cz, cz**2 * cx, cz**2 * cy,
        e2**2, cx**2 * e2, cy**2 * e2, cz**2 * e2,
        cx**2 * cy**2, cx**2 * cz**2, cy**2 * cz**2, cx * cy * cz,
    ]
    basis: list[np.ndarray] = []
    for row in raw:
        v = row.copy()
        for prev in basis:
            v = v - (np.dot(v, prev) / np.dot(prev, prev)) * prev
        if np.sqrt(np.dot(v, v)) < 1e-14:
            # dependent monomial: take the first unit vector with a component
            # outside the current span instead
            for i in range(27):
                u = np.zeros(27)
                u[i] = 1.0
                for prev in basis:
                    u = u - (np.dot(u, prev) / np.dot(prev, prev)) * prev
                if np.sqrt(np.dot(u, u)) > 1e-10:
                    v = u
                    break
        basis.append(v)
    m = np.array(basis)
    assert np.linalg.matrix_rank(m) == 27
    return m


def mrt_matrices(q: int) -> tuple[np.ndarray, np.ndarray]:
    """(M, M^-1) in float64.  Consumers round both to float32 for fp32 runs."""
    m = {9: mrt_matrix_d2q9, 19: mrt_matrix_d3q19, 27: mrt_matrix_d3q27}[q]()
    return m, np.linalg.inv(m)


# --- D3Q27 raw-moment (monomial) basis for the cumulant operators -------------

# (a, b, c) exponent of cx^a cy^b cz^c for moment index k; order as in
# ``tensorlbm/cumulant.py:321-349``.
CUMULANT_DEGREES: list[tuple[int, int, int]] = [
    (0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1),
    (2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1),
    (2, 1, 0), (2, 0, 1), (1, 2, 0), (0, 2, 1), (1, 0, 2), (0, 1, 2), (1, 1, 1),
    (2, 2, 0), (2, 0, 2), (0, 2, 2), (2, 1, 1), (1, 2, 1), (1, 1, 2),
    (2, 2, 1), (2, 1, 2), (1, 2, 2), (2, 2, 2),
]


def monomial_matrix_d3q27() -> np.ndarray:
    c = D3Q27.c.astype(np.float64)
    m = np.zeros((27, 27))
    for i, (a, b, d) in enumerate(CUMULANT_DEGREES):
        m[i] = c[:, 0] ** a * c[:, 1] ** b * c[:, 2] ** d
    return m


def shift_groups() -> tuple[list[tuple[int, int, int]], ...]:
    """Per axis, the (deg0, deg1, deg2) moment-index triplets of the 1-D binomial shift."""
    out = []
    for axis in range(3):
        others = [a for a in range(3) if a != axis]
        bucket: dict[tuple[int, int], dict[int, int]] = {}
        for k, deg in enumerate(CUMULANT_DEGREES):
            bucket.setdefault((deg[others[0]], deg[others[1]]), {})[deg[axis]] = k
        out.append([(b[0], b[1], b[2]) for key, b in sorted(bucket.items()) if len(b) == 3])
    return tuple(out)
