"""CPU oracle: a numpy restatement of TensorLBM's lattice-Boltzmann time step.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA kernels of
tensorlbm_b200: only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline / reference leg import it.  The product never calls it.

Every function restates the TensorLBM function cited beside it (paths inside
the TensorLBM source tree) in plain numpy, keeping the reference's arithmetic
order and dtype behaviour (float32 fields stay float32; the MRT matrices of
D3Q19/D3Q27 are rounded to float32 like the reference's cached tensors).
Parity of this oracle with TensorLBM itself is pinned by the golden vectors in
tests/golden/ (generated by tests/golden/make_golden.py from the unmodified
reference) and checked by tests/test_oracle_golden.py.

Layout: f has shape (Q, nz, ny, nx) for 3-D lattices and (9, ny, nx) for D2Q9.
"""

from __future__ import annotations

from fractions import Fraction

import numpy as np

# ---------------------------------------------------------------------------
# lattice tables (tensorlbm/d2q9.py:8-26, d3q19.py:6-67, d3q27.py:32-84)
# ---------------------------------------------------------------------------

_C9 = [(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1)]
_C19 = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
        (1, 1, 0), (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 0, 1), (-1, 0, -1), (1, 0, -1), (-1, 0, 1),
        (0, 1, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1)]
_C27 = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
        (1, 1, 0), (-1, 1, 0), (1, -1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1),
        (0, 1, 1), (0, -1, 1), (0, 1, -1), (0, -1, -1),
        (1, 1, 1), (-1, 1, 1), (1, -1, 1), (-1, -1, 1), (1, 1, -1), (-1, 1, -1), (1, -1, -1), (-1, -1, -1)]
C = {9: np.array(_C9, dtype=np.int64), 19: np.array(_C19, dtype=np.int64), 27: np.array(_C27, dtype=np.int64)}
_WFRAC = {
    9: [Fraction(4, 9)] + [Fraction(1, 9)] * 4 + [Fraction(1, 36)] * 4,
    19: [Fraction(1, 3)] + [Fraction(1, 18)] * 6 + [Fraction(1, 36)] * 12,
    27: [Fraction(8, 27)] + [Fraction(2, 27)] * 6 + [Fraction(1, 54)] * 12 + [Fraction(1, 216)] * 8,
}
W64 = {q: np.array([float(v) for v in w]) for q, w in _WFRAC.items()}


def opposite(q: int) -> np.ndarray:
    c = C[q]
    idx = {tuple(r): i for i, r in enumerate(c.tolist())}
    return np.array([idx[tuple((-c[i]).tolist())] for i in range(q)], dtype=np.int64)


def zou_he_partner(q: int) -> np.ndarray:
    """Known population paired with each unknown one in the x-face Zou/He
    conditions.  D3Q19 pairs true opposites (boundaries3d.py:14-19); the D3Q27
    tables pair x-mirrors, e.g. 7 (1,1,0) with 8 (-1,1,0)
    (boundaries_d3q27.py:36-41), and that pairing is what TensorLBM computes."""
    if q != 27:
        return opposite(q)
    c = C[27]
    idx = {tuple(r): i for i, r in enumerate(c.tolist())}
    return np.array([idx[(-int(r[0]), int(r[1]), int(r[2]))] for r in c], dtype=np.int64)


def weights(q: int, dtype) -> np.ndarray:
    """D2Q9 keeps float32 weights for every field dtype (d2q9.py:22-36);
    D3Q19/D3Q27 cast the binary64 weights (d3q19.py:58-80)."""
    if q == 9:
        return W64[9].astype(np.float32).astype(dtype)
    return W64[q].astype(dtype)


def _view(v: np.ndarray, ndim: int) -> np.ndarray:
    return v.reshape((-1,) + (1,) * ndim)


# ---------------------------------------------------------------------------
# moments and equilibrium
# ---------------------------------------------------------------------------


def sum0(a: np.ndarray) -> np.ndarray:
    """Sum over axis 0 in the order torch's CPU reduction uses for a (Q, ...)
    tensor whose inner size is a multiple of its vector block: rows 0..15
    accumulated in order, rows 16.. in order, then the two partial sums added.
    (Measured against torch 2.11 bit for bit; for inner sizes that are not a
    multiple of 32 torch handles the last columns with another order.)"""
    head = np.zeros_like(a[0])
    for r in a[:16]:
        head = head + r
    if a.shape[0] <= 16:
        return head
    tail = np.zeros_like(a[0])
    for r in a[16:]:
        tail = tail + r
    return tail + head


def macroscopic(f: np.ndarray):
    """d2q9.py:61-74, d3q19.py:165-186, d3q27.py:395-420."""
    q = f.shape[0]
    nd = f.ndim - 1
    c = C[q].astype(f.dtype)
    rho = sum0(f)
    rs = np.maximum(rho, f.dtype.type(1e-12))
    ux = sum0(f * _view(c[:, 0], nd)) / rs
    uy = sum0(f * _view(c[:, 1], nd)) / rs
    if q == 9:
        return rho, ux, uy, None
    uz = sum0(f * _view(c[:, 2], nd)) / rs
    return rho, ux, uy, uz


def equilibrium(q: int, rho, ux, uy, uz=None) -> np.ndarray:
    """d2q9.py:39-58, d3q19.py:83-125, d3q27.py:353-392."""
    nd = rho.ndim
    dt = rho.dtype
    c = C[q]
    w = _view(weights(q, dt), nd)
    if q == 9:
        usq = ux * ux + uy * uy
        cu = _view(c[:, 0].astype(dt), nd) * ux + _view(c[:, 1].astype(dt), nd) * uy
    else:
        usq = ux * ux + uy * uy + uz * uz
        cu = (_view(c[:, 0].astype(dt), nd) * ux + _view(c[:, 1].astype(dt), nd) * uy
              + _view(c[:, 2].astype(dt), nd) * uz)
    return w * rho[None] * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq[None])


# ---------------------------------------------------------------------------
# collisions
# ---------------------------------------------------------------------------


def collide_bgk(f: np.ndarray, tau: float) -> np.ndarray:
    """solver.py:67-71, solver3d.py:100-104, d3q27.py:423-437."""
    rho, ux, uy, uz = macroscopic(f)
    feq = equilibrium(f.shape[0], rho, ux, uy, uz)
    return f - (f - feq) / f.dtype.type(tau)


def collide_trt(f: np.ndarray, tau_plus: float, lambda_trt: float = 3.0 / 16.0) -> np.ndarray:
    """solver.py:440-486, solver3d.py:303-336, d3q27.py:438-480: the symmetric
    part relaxes with tau_plus, the antisymmetric part with
    tau_minus = 1/2 + Lambda / (tau_plus - 1/2) (formed in float64, used as a
    scalar of the field's dtype)."""
    q = f.shape[0]
    t = f.dtype.type
    rho, ux, uy, uz = macroscopic(f)
    feq = equilibrium(q, rho, ux, uy, uz)
    tau_minus = 0.5 + lambda_trt / (tau_plus - 0.5)
    opp = opposite(q)
    half = t(0.5)
    f_plus, f_minus = half * (f + f[opp]), half * (f - f[opp])
    e_plus, e_minus = half * (feq + feq[opp]), half * (feq - feq[opp])
    return f - (f_plus - e_plus) / t(tau_plus) - (f_minus - e_minus) / t(tau_minus)


_CASCADED_DEGREES = {
    19: [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1),
         (2, 1, 0), (2, 0, 1), (1, 2, 0), (0, 2, 1), (1, 0, 2), (0, 1, 2), (2, 2, 0), (2, 0, 2), (0, 2, 2)],
    27: [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1),
         (2, 1, 0), (2, 0, 1), (1, 2, 0), (0, 2, 1), (1, 0, 2), (0, 1, 2), (1, 1, 1), (2, 2, 0), (2, 0, 2), (0, 2, 2),
         (2, 1, 1), (1, 2, 1), (1, 1, 2), (2, 2, 1), (2, 1, 2), (1, 2, 2), (2, 2, 2)],
}


def collide_cascaded(f: np.ndarray, tau: float, s_bulk: float = 1.0, s_3: float = 1.0, s_4: float = 1.0,
                     s_5=None, s_6=None) -> np.ndarray:
    """cascaded_collision.py:445-576: raw moments of f_neq by the float64 monomial
    matrix cast to the field's dtype, binomial shift x, y, z over the complete
    (degree 0, 1, 2) triples, per-order relaxation with the trace / deviator
    split at second order (:330-442), unshift z, y, x, inverse matrix."""
    q = f.shape[0]
    dt = f.dtype
    deg = _CASCADED_DEGREES[q]
    c = C[q].astype(np.float64)
    m64 = np.array([c[:, 0] ** a * c[:, 1] ** b * c[:, 2] ** d for a, b, d in deg])
    M, Minv = m64.astype(dt), np.linalg.inv(m64).astype(dt)
    rho, ux, uy, uz = macroscopic(f)
    feq = equilibrium(q, rho, ux, uy, uz)
    sp = f.shape[1:]
    m = (M @ (f - feq).reshape(q, -1)).reshape((q,) + sp)
    groups = []
    for dim in range(3):
        other = [d for d in range(3) if d != dim]
        bucket = {}
        for idx, dg in enumerate(deg):
            bucket.setdefault((dg[other[0]], dg[other[1]]), {})[dg[dim]] = idx
        groups.append([(v[0], v[1], v[2]) for _, v in sorted(bucket.items()) if all(k in v for k in (0, 1, 2))])

    def shift(k, g, u, sign):
        out = k.copy()
        for i0, i1, i2 in g:
            if sign < 0:
                out[i1] = k[i1] - u * k[i0]
                out[i2] = k[i2] - 2.0 * u * k[i1] + u * u * k[i0]
            else:
                out[i1] = k[i1] + u * k[i0]
                out[i2] = k[i2] + 2.0 * u * k[i1] + u * u * k[i0]
        return out

    for g, u in zip(groups, (ux, uy, uz)):
        m = shift(m, g, u, -1)
    k = m.copy()
    tr = m[4] + m[5] + m[6]
    trs = (1.0 - s_bulk) * tr
    om = 1.0 / tau
    for i in (4, 5, 6):
        k[i] = (1.0 - om) * (m[i] - tr / 3.0) + trs / 3.0
    for i in (7, 8, 9):
        k[i] = (1.0 - om) * m[i]
    s5 = s_4 if s_5 is None else s_5
    s6 = s_4 if s_6 is None else s_6
    for i, dg in enumerate(deg):
        order = sum(dg)
        if order >= 3:
            k[i] = (1.0 - {3: s_3, 4: s_4, 5: s5, 6: s6}[order]) * m[i]
    for g, u in zip(groups[::-1], (uz, uy, ux)):
        k = shift(k, g, u, 1)
    return feq + (Minv @ k.reshape(q, -1)).reshape((q,) + sp)


def mrt_matrix(q: int) -> np.ndarray:
    """Moment bases: solver.py:24-34 (D2Q9), solver3d.py:24-55 (D3Q19),
    d3q27.py:545-635 (D3Q27 Gram-Schmidt)."""
    c = C[q].astype(np.float64)
    if q == 9:
        cx, cy = c[:, 0], c[:, 1]
        c2 = cx**2 + cy**2
        return np.array([np.ones(9), 3 * c2 - 4, (9 * c2**2 - 21 * c2 + 8) / 2, cx, (3 * c2 - 5) * cx, cy,
                         (3 * c2 - 5) * cy, cx**2 - cy**2, cx * cy])
    cx, cy, cz = c[:, 0], c[:, 1], c[:, 2]
    e2 = cx**2 + cy**2 + cz**2
    if q == 19:
        return np.array([np.ones(19), 19 * e2 - 30, (21 * e2**2 - 53 * e2 + 24) / 2, cx,
                         cx * e2 * (5 * e2 - 9) / 2, cy, cy * e2 * (5 * e2 - 9) / 2, cz,
                         cz * e2 * (5 * e2 - 9) / 2, 3 * cx**2 - e2, cx**2 - cy**2, cx * cy, cx * cz, cy * cz,
                         (3 * e2 - 5) * (3 * cx**2 - e2) / 2, (3 * e2 - 5) * (cx**2 - cy**2) / 2, cx**2 * cy,
                         cx**2 * cz, cy**2 * cx])
    raw = [np.ones(27), cx, cy, cz, e2, 3 * cx**2 - e2, cy**2 - cz**2, cx * cy, cx * cz, cy * cz,
           cx * e2, cy * e2, cz * e2, cx**2 * cy, cx**2 * cz, cy**2 * cx, cy**2 * cz, cz**2 * cx, cz**2 * cy,
           e2**2, cx**2 * e2, cy**2 * e2, cz**2 * e2, cx**2 * cy**2, cx**2 * cz**2, cy**2 * cz**2,
           cx * cy * cz]
    rows: list[np.ndarray] = []
    for r in raw:
        v = r.copy()
        for p in rows:
            v = v - (v @ p) / (p @ p) * p
        if np.sqrt(v @ v) < 1e-14:
            for i in range(27):
                u = np.zeros(27)
                u[i] = 1.0
                for p in rows:
                    u = u - (u @ p) / (p @ p) * p
                if np.sqrt(u @ u) > 1e-10:
                    v = u
                    break
        rows.append(v)
    return np.array(rows)


def _mrt_rates(q: int, tau: float, s_e, s_eps, s_q, s_pi) -> list[float]:
    s_nu = 1.0 / tau
    if q == 9:
        return [0.0, s_e, s_eps, 0.0, s_q, 0.0, s_q, s_nu, s_nu]
    if s_pi is None:
        s_pi = s_e
    if q == 19:
        return [0.0, s_e, s_eps, 0.0, s_q, 0.0, s_q, 0.0, s_q] + [s_nu] * 5 + [s_pi, s_pi, 1.0, 1.0, 1.0]
    return [0.0] * 4 + [s_e] + [s_nu] * 5 + [s_q] * 9 + [s_eps] + [s_pi] * 7


def collide_mrt(f: np.ndarray, tau: float, s_e=None, s_eps=None, s_q=None, s_pi=None, tau_field=None):
    """m = M f, m* = m - s (m - M feq), f' = M^-1 m* (solver.py:249-331,
    solver3d.py:107-160, d3q27.py:643-727).  D3Q19/D3Q27 matrices are float32
    in the reference whatever the field dtype (solver3d.py:93-97)."""
    q = f.shape[0]
    defaults = {9: (1.64, 1.54, 1.7), 19: (1.19, 1.4, 1.2), 27: (1.19, 1.4, 1.2)}[q]
    s_e = defaults[0] if s_e is None else s_e
    s_eps = defaults[1] if s_eps is None else s_eps
    s_q = defaults[2] if s_q is None else s_q
    m64 = mrt_matrix(q)
    mat_dt = f.dtype if q == 9 else np.float32
    m = m64.astype(mat_dt)
    minv = np.linalg.inv(m64).astype(mat_dt)
    spatial = f.shape[1:]
    ff = f.reshape(q, -1)
    rho, ux, uy, uz = macroscopic(f)
    feq = equilibrium(q, rho, ux, uy, uz).reshape(q, -1)
    mom = m @ ff
    meq = m @ feq
    s = np.array(_mrt_rates(q, tau, s_e, s_eps, s_q, s_pi), dtype=f.dtype)[:, None]
    if tau_field is not None:
        s = np.repeat(s, ff.shape[1], axis=1)
        inv = (1.0 / tau_field.astype(f.dtype)).reshape(-1)
        s[7] = inv
        s[8] = inv
    mstar = mom - s * (mom - meq)
    return (minv @ mstar).reshape((q,) + spatial).astype(f.dtype)


def neq_stress(fneq: np.ndarray):
    q = fneq.shape[0]
    nd = fneq.ndim - 1
    c = C[q].astype(fneq.dtype)
    cx = _view(c[:, 0], nd)
    cy = _view(c[:, 1], nd)
    pxx = sum0(cx * cx * fneq)
    pyy = sum0(cy * cy * fneq)
    pxy = sum0(cx * cy * fneq)
    if q == 9:
        return pxx, pyy, None, pxy, None, None
    cz = _view(c[:, 2], nd)
    return pxx, pyy, sum0(cz * cz * fneq), pxy, sum0(cx * cz * fneq), sum0(cy * cz * fneq)


def smagorinsky_tau(tau: float, pi_norm, rho, c_s: float):
    """turbulence.py:183-208 with the clamps of :77-100."""
    rs = np.maximum(rho, rho.dtype.type(1e-12))
    disc = tau**2 + 18.0 * c_s**2 * pi_norm / rs
    te = 0.5 * (tau + np.sqrt(np.maximum(disc, 0.0)))
    return np.clip(te, 0.5001, max(1.0, tau + 0.5)).astype(rho.dtype)


def collide_smagorinsky(f: np.ndarray, tau: float, c_s: float = 0.1) -> np.ndarray:
    """turbulence.py:216 (D2Q9), :245 (D3Q19), :472 (D3Q27)."""
    q = f.shape[0]
    rho, ux, uy, uz = macroscopic(f)
    fneq = f - equilibrium(q, rho, ux, uy, uz)
    pxx, pyy, pzz, pxy, pxz, pyz = neq_stress(fneq)
    if q == 9:
        rad = pxx**2 + pyy**2 + 2.0 * pxy**2
    else:
        rad = pxx**2 + pyy**2 + pzz**2 + 2.0 * (pxy**2 + pxz**2 + pyz**2)
    pn = np.sqrt(np.maximum(rad, rad.dtype.type(1e-30)))
    te = smagorinsky_tau(tau, pn, rho, c_s)
    return f - fneq / te[None]


def collide_rlbm(f: np.ndarray, tau: float) -> np.ndarray:
    """Regularised BGK (Latt & Chopard 2006): solver.py:338-392 (D2Q9),
    solver3d.py:342-403 (D3Q19), d3q27.py:481-540 (D3Q27).  The second moment
    of f - feq is projected on the Hermite basis H = c c - I/3 and relaxed:
    feq + (1 - 1/tau) * ((9/2 w) * (H_xx Pi_xx + H_yy Pi_yy [+ H_zz Pi_zz]
    + 2 H_xy Pi_xy [+ 2 H_xz Pi_xz + 2 H_yz Pi_yz])), each operation rounded in
    the field's dtype with Python scalars taken at that dtype.  The projection
    takes the float32-rounded weights for every dtype (the default dtype of
    _w_on, d3q19.py:75-80, d3q27.py:345-350); the equilibrium keeps its own."""
    q = f.shape[0]
    nd = f.ndim - 1
    t = f.dtype.type
    rho, ux, uy, uz = macroscopic(f)
    feq = equilibrium(q, rho, ux, uy, uz)
    fneq = f - feq
    pxx, pyy, pzz, pxy, pxz, pyz = neq_stress(fneq)
    c = C[q].astype(f.dtype)
    cx, cy = _view(c[:, 0], nd), _view(c[:, 1], nd)
    cs2 = t(1.0 / 3.0)
    s = (cx * cx - cs2) * pxx + (cy * cy - cs2) * pyy
    if q == 9:
        s = s + (t(2) * (cx * cy)) * pxy
    else:
        cz = _view(c[:, 2], nd)
        s = s + (cz * cz - cs2) * pzz
        s = s + (t(2) * (cx * cy)) * pxy + (t(2) * (cx * cz)) * pxz + (t(2) * (cy * cz)) * pyz
    reg = (t(4.5) * _view(W64[q].astype(np.float32).astype(f.dtype), nd)) * s
    return feq + t(1.0 - 1.0 / tau) * reg


def collide_cumulant_d3q19(f: np.ndarray, tau: float, omega_b=1.0, omega_odd=1.0, omega_even=1.0, c_s=0.0):
    """Hermite-regularised stress relaxation, cumulant.py:1159-1420 (Smagorinsky branch only)."""
    rho, ux, uy, uz = macroscopic(f)
    feq = equilibrium(19, rho, ux, uy, uz)
    fneq = f - feq
    pxx, pyy, pzz, pxy, pxz, pyz = neq_stress(fneq)
    if c_s > 0.0:
        pn = np.sqrt(pxx**2 + pyy**2 + pzz**2 + 2.0 * (pxy**2 + pxz**2 + pyz**2))
        rs = np.maximum(rho, rho.dtype.type(1e-12))
        te = 0.5 * (tau + np.sqrt(tau * tau + 18.0 * c_s * c_s * pn / rs))
        omega = (1.0 / te).astype(f.dtype)
    else:
        omega = 1.0 / tau
    tr = pxx + pyy + pzz
    sxx = pxx - omega * pxx - (omega_b - omega) * tr / 3.0
    syy = pyy - omega * pyy - (omega_b - omega) * tr / 3.0
    szz = pzz - omega * pzz - (omega_b - omega) * tr / 3.0
    sxy = pxy - omega * pxy
    sxz = pxz - omega * pxz
    syz = pyz - omega * pyz
    c = C[19].astype(f.dtype)
    cx, cy, cz = (_view(c[:, k], 3) for k in range(3))
    w = _view(np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=f.dtype), 3)
    cs2 = 1.0 / 3.0
    hxx, hyy, hzz = cx * cx - cs2, cy * cy - cs2, cz * cz - cs2
    reg = 4.5 * w * (hxx * sxx + hyy * syy + hzz * szz + 2.0 * cx * cy * sxy + 2.0 * cx * cz * sxz
                     + 2.0 * cy * cz * syz)
    ho = fneq - 4.5 * w * (hxx * pxx + hyy * pyy + hzz * pzz + 2.0 * cx * cy * pxy + 2.0 * cx * cz * pxz
                           + 2.0 * cy * cz * pyz)
    return (feq + reg + (1.0 - omega_even) * ho).astype(f.dtype)


# D3Q27 cumulant machinery (cumulant.py:321-457, 904-919)
DEGREES = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1),
           (0, 1, 1), (2, 1, 0), (2, 0, 1), (1, 2, 0), (0, 2, 1), (1, 0, 2), (0, 1, 2), (1, 1, 1), (2, 2, 0),
           (2, 0, 2), (0, 2, 2), (2, 1, 1), (1, 2, 1), (1, 1, 2), (2, 2, 1), (2, 1, 2), (1, 2, 2), (2, 2, 2)]


def _shift_groups():
    out = []
    for axis in range(3):
        others = [a for a in range(3) if a != axis]
        bucket: dict = {}
        for k, d in enumerate(DEGREES):
            bucket.setdefault((d[others[0]], d[others[1]]), {})[d[axis]] = k
        out.append([(b[0], b[1], b[2]) for key, b in sorted(bucket.items()) if len(b) == 3])
    return out


_GROUPS = _shift_groups()


def monomial_matrix() -> np.ndarray:
    c = C[27].astype(np.float64)
    return np.array([c[:, 0] ** a * c[:, 1] ** b * c[:, 2] ** d for a, b, d in DEGREES])


def _shift(m, groups, u, sign):
    out = m.copy()
    for i0, i1, i2 in groups:
        out[i1] = m[i1] + sign * u * m[i0]
        out[i2] = m[i2] + sign * 2.0 * u * m[i1] + u * u * m[i0]
    return out


def to_central(m, ux, uy, uz):
    m = _shift(m, _GROUPS[0], ux, -1.0)
    m = _shift(m, _GROUPS[1], uy, -1.0)
    return _shift(m, _GROUPS[2], uz, -1.0)


def to_raw(k, ux, uy, uz):
    k = _shift(k, _GROUPS[2], uz, 1.0)
    k = _shift(k, _GROUPS[1], uy, 1.0)
    return _shift(k, _GROUPS[0], ux, 1.0)


def legacy_forward(k):
    """cumulant.py:470-577"""
    C_ = k.copy()
    k200, k020, k002, k110, k101, k011 = k[4], k[5], k[6], k[7], k[8], k[9]
    C_[17] = k[17] - k200 * k020 - 2.0 * k110 * k110
    C_[18] = k[18] - k200 * k002 - 2.0 * k101 * k101
    C_[19] = k[19] - k020 * k002 - 2.0 * k011 * k011
    C_[20] = k[20] - k200 * k011 - 2.0 * k101 * k110
    C_[21] = k[21] - k020 * k101 - 2.0 * k110 * k011
    C_[22] = k[22] - k002 * k110 - 2.0 * k101 * k011
    C_[23] = k[23] - k200 * k[13] - 2.0 * k110 * k[16]
    C_[24] = k[24] - k200 * k[15] - 2.0 * k101 * k[16]
    C_[25] = k[25] - k020 * k[14] - 2.0 * k011 * k[16]
    C_[26] = (k[26] - k200 * C_[19] - k020 * C_[18] - k002 * C_[17]
              - 2.0 * (k110 * C_[22] + k101 * C_[21] + k011 * C_[20]) + 2.0 * k200 * k020 * k002
              + 4.0 * k110 * k101 * k011 + 2.0 * k110 * k110 * k002 + 2.0 * k101 * k101 * k020
              + 2.0 * k011 * k011 * k200)
    return C_


def legacy_inverse(C_):
    """cumulant.py:580-651"""
    k = C_.copy()
    c200, c020, c002, c110, c101, c011 = C_[4], C_[5], C_[6], C_[7], C_[8], C_[9]
    k[17] = C_[17] + c200 * c020 + 2.0 * c110 * c110
    k[18] = C_[18] + c200 * c002 + 2.0 * c101 * c101
    k[19] = C_[19] + c020 * c002 + 2.0 * c011 * c011
    k[20] = C_[20] + c200 * c011 + 2.0 * c101 * c110
    k[21] = C_[21] + c020 * c101 + 2.0 * c110 * c011
    k[22] = C_[22] + c002 * c110 + 2.0 * c101 * c011
    k[23] = C_[23] + c200 * C_[13] + 2.0 * c110 * C_[16]
    k[24] = C_[24] + c200 * C_[15] + 2.0 * c101 * C_[16]
    k[25] = C_[25] + c020 * C_[14] + 2.0 * c011 * C_[16]
    k[26] = (C_[26] + c200 * C_[19] + c020 * C_[18] + c002 * C_[17]
             + 2.0 * (c110 * C_[22] + c101 * C_[21] + c011 * C_[20]) - 2.0 * c200 * c020 * c002
             - 4.0 * c110 * c101 * c011 - 2.0 * c110 * c110 * c002 - 2.0 * c101 * c101 * c020
             - 2.0 * c011 * c011 * c200)
    return k


def collide_cumulant_d3q27(f: np.ndarray, tau: float, omega_b=1.0, omega_odd=1.0, omega_even=1.0):
    """cumulant.py:935-1047 (C_s = 0)."""
    om = 1.0 / tau
    rho, ux, uy, uz = macroscopic(f)
    feq = equilibrium(27, rho, ux, uy, uz)
    fneq = f - feq
    m64 = monomial_matrix()
    M = m64.astype(f.dtype)
    Minv = np.linalg.inv(m64).astype(f.dtype)
    sp = f.shape[1:]
    m = (M @ fneq.reshape(27, -1)).reshape((27,) + sp)
    Cn = legacy_forward(to_central(m, ux, uy, uz))
    out = Cn.copy()
    tr = Cn[4] + Cn[5] + Cn[6]
    trs = (1.0 - omega_b) * tr
    for i in range(3):
        out[4 + i] = (1.0 - om) * (Cn[4 + i] - tr / 3.0) + trs / 3.0
    for i in (7, 8, 9):
        out[i] = (1.0 - om) * Cn[i]
    out[10:17] = (1.0 - omega_odd) * Cn[10:17]
    out[17:27] = (1.0 - omega_even) * Cn[17:27]
    ms = to_raw(legacy_inverse(out), ux, uy, uz)
    return (feq + (Minv @ ms.reshape(27, -1)).reshape((27,) + sp)).astype(f.dtype)


def geier_forward(k):
    """cumulant.py:674-745"""
    rho = k[0]
    t = k / rho
    c = t.copy()
    c[17] = t[17] - (t[5] * t[4] + 2.0 * t[7] ** 2)
    c[18] = t[18] - (t[6] * t[4] + 2.0 * t[8] ** 2)
    c[19] = t[19] - (t[6] * t[5] + 2.0 * t[9] ** 2)
    c[20] = t[20] - (t[9] * t[4] + 2.0 * t[8] * t[7])
    c[21] = t[21] - (2.0 * t[9] * t[7] + t[5] * t[8])
    c[22] = t[22] - (t[6] * t[7] + 2.0 * t[9] * t[8])
    c[23] = t[23] - (2.0 * t[9] * t[10] + t[5] * t[11] + t[13] * t[4] + 2.0 * t[8] * t[12] + 4.0 * t[7] * t[16])
    c[24] = t[24] - (t[6] * t[10] + 2.0 * t[9] * t[11] + t[15] * t[4] + 4.0 * t[8] * t[16] + 2.0 * t[14] * t[7])
    c[25] = t[25] - (t[6] * t[12] + 4.0 * t[9] * t[16] + 2.0 * t[15] * t[7] + t[5] * t[14] + 2.0 * t[13] * t[8])
    c[26] = t[26] - (-2.0 * t[6] * t[5] * t[4] - 4.0 * t[6] * t[7] ** 2 + t[6] * t[17] - 4.0 * t[9] ** 2 * t[4]
                     - 16.0 * t[9] * t[8] * t[7] + 4.0 * t[9] * t[20] + 2.0 * t[15] * t[10]
                     - 4.0 * t[5] * t[8] ** 2 + t[5] * t[18] + 2.0 * t[13] * t[11] + t[19] * t[4]
                     + 4.0 * t[8] * t[21] + 2.0 * t[14] * t[12] + 4.0 * t[7] * t[22] + 4.0 * t[16] ** 2)
    out = c * rho
    out[0] = rho
    return out


def geier_inverse(c):
    """cumulant.py:748-815"""
    rho = c[0]
    t = c / rho
    k = t.copy()
    k[17] = t[5] * t[4] + 2.0 * t[7] ** 2 + t[17]
    k[18] = t[6] * t[4] + 2.0 * t[8] ** 2 + t[18]
    k[19] = t[6] * t[5] + 2.0 * t[9] ** 2 + t[19]
    k[20] = t[9] * t[4] + 2.0 * t[8] * t[7] + t[20]
    k[21] = 2.0 * t[9] * t[7] + t[5] * t[8] + t[21]
    k[22] = t[6] * t[7] + 2.0 * t[9] * t[8] + t[22]
    k[23] = 2.0 * t[9] * t[10] + t[5] * t[11] + t[13] * t[4] + 2.0 * t[8] * t[12] + 4.0 * t[7] * t[16] + t[23]
    k[24] = t[6] * t[10] + 2.0 * t[9] * t[11] + t[15] * t[4] + 4.0 * t[8] * t[16] + 2.0 * t[14] * t[7] + t[24]
    k[25] = t[6] * t[12] + 4.0 * t[9] * t[16] + 2.0 * t[15] * t[7] + t[5] * t[14] + 2.0 * t[13] * t[8] + t[25]
    k[26] = (t[6] * t[5] * t[4] + 2.0 * t[6] * t[7] ** 2 + t[6] * t[17] + 2.0 * t[9] ** 2 * t[4]
             + 8.0 * t[9] * t[8] * t[7] + 4.0 * t[9] * t[20] + 2.0 * t[15] * t[10] + 2.0 * t[5] * t[8] ** 2
             + t[5] * t[18] + 2.0 * t[13] * t[11] + t[19] * t[4] + 4.0 * t[8] * t[21] + 2.0 * t[14] * t[12]
             + 4.0 * t[7] * t[22] + 4.0 * t[16] ** 2 + t[26])
    out = k * rho
    out[0] = rho
    return out


def collide_cumulant_geier_d3q27(f: np.ndarray, tau: float, omega_b=1.0, omega_odd=1.0, omega_even=1.0):
    """cumulant.py:1050-1156 (C_s = 0)."""
    om = 1.0 / tau
    rho, ux, uy, uz = macroscopic(f)
    feq = equilibrium(27, rho, ux, uy, uz)
    m64 = monomial_matrix()
    M = m64.astype(f.dtype)
    Minv = np.linalg.inv(m64).astype(f.dtype)
    sp = f.shape[1:]
    m = (M @ f.reshape(27, -1)).reshape((27,) + sp)
    meq = (M @ feq.reshape(27, -1)).reshape((27,) + sp)
    Cc = geier_forward(to_central(m, ux, uy, uz))
    Ce = geier_forward(to_central(meq, ux, uy, uz))
    D = Cc - Ce
    out = Cc.copy()
    tr = D[4] + D[5] + D[6]
    for i in range(3):
        out[4 + i] = Cc[4 + i] - (om * (D[4 + i] - tr / 3.0) + omega_b * tr / 3.0)
    for i in (7, 8, 9):
        out[i] = Cc[i] - om * D[i]
    out[10:17] = Cc[10:17] - omega_odd * D[10:17]
    out[17:27] = Cc[17:27] - omega_even * D[17:27]
    ms = to_raw(geier_inverse(out), ux, uy, uz)
    return (Minv @ ms.reshape(27, -1)).reshape((27,) + sp).astype(f.dtype)


COLLIDERS = {
    "bgk": collide_bgk,
    "mrt": collide_mrt,
    "trt": collide_trt,
    "rlbm": collide_rlbm,
    "cascaded": collide_cascaded,
    "smagorinsky": collide_smagorinsky,
    "cumulant_d3q19": collide_cumulant_d3q19,
    "cumulant": collide_cumulant_d3q27,
    "cumulant_geier": collide_cumulant_geier_d3q27,
}


# ---------------------------------------------------------------------------
# streaming and boundaries
# ---------------------------------------------------------------------------


def stream(f: np.ndarray) -> np.ndarray:
    """Periodic pull f'[q, x] = f[q, x - c_q] (solver.py:396, solver3d.py:210, d3q27.py:766)."""
    q = f.shape[0]
    out = np.empty_like(f)
    for i in range(q):
        c = C[q][i]
        if q == 9:
            out[i] = np.roll(f[i], shift=(int(c[1]), int(c[0])), axis=(0, 1))
        else:
            out[i] = np.roll(f[i], shift=(int(c[2]), int(c[1]), int(c[0])), axis=(0, 1, 2))
    return out


def bounce_back(f: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """where(mask, f[opp], f): boundaries.py:39, boundaries3d.py:112, boundaries_d3q27.py:45."""
    return np.where(mask[None], f[opposite(f.shape[0])], f)


# ---------------------------------------------------------------------------
# Bouzidi (BFL) interpolated bounce-back on curved walls
# ---------------------------------------------------------------------------


def sphere_links(q: int, nx: int, ny: int, nz: int, cx: float, cy: float, cz: float, radius: float):
    """Boundary links of a sphere and their wall fractions: bfl_common.py:384-477
    (D3Q19, D3Q27) and interpolated_bc_common.py:136-233 (D3Q27).  Link (x, d):
    x outside the sphere and x + c_d inside (float64 squared distances against
    radius^2); its fraction is the ray-sphere intersection along c_d in float64,
    clamped to [1e-6, 1] and stored as float32 (0.5 off the links)."""
    zz, yy, xx = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(ny, dtype=np.float64),
                             np.arange(nx, dtype=np.float64), indexing="ij")
    r2 = radius ** 2
    mask = np.zeros((q, nz, ny, nx), dtype=bool)
    qf = np.full((q, nz, ny, nx), 0.5, dtype=np.float32)
    for d in range(q):
        dcx, dcy, dcz = (float(v) for v in C[q][d])
        if dcx == 0.0 and dcy == 0.0 and dcz == 0.0:
            continue
        near = ((xx + dcx - cx) ** 2 + (yy + dcy - cy) ** 2 + (zz + dcz - cz) ** 2) <= r2
        fluid = ((xx - cx) ** 2 + (yy - cy) ** 2 + (zz - cz) ** 2) > r2
        link = fluid & near
        if not link.any():
            continue
        dx, dy, dz = xx - cx, yy - cy, zz - cz
        a = dcx ** 2 + dcy ** 2 + dcz ** 2
        b = 2.0 * (dcx * dx + dcy * dy + dcz * dz)
        c = dx ** 2 + dy ** 2 + dz ** 2 - r2
        disc = b ** 2 - 4.0 * a * c
        root = np.sqrt(np.where(link & (disc >= 0.0), disc, 0.0))
        t1 = (-b - root) / (2.0 * a)
        t2 = (-b + root) / (2.0 * a)
        v1 = (t1 > 1e-10) & (t1 <= 1.0 + 1e-10)
        v2 = (t2 > 1e-10) & (t2 <= 1.0 + 1e-10)
        frac = np.where(v1 & v2, np.minimum(t1, t2), np.where(v1, t1, np.where(v2, t2, 0.5)))
        mask[d] = link
        qf[d] = np.where(link, np.clip(frac, 1e-6, 1.0).astype(np.float32), qf[d])
    return mask, qf


def _bfl_values(f_prev: np.ndarray, mask: np.ndarray, qf: np.ndarray):
    """Per link (x, d) the value sent back into x along -c_d (bfl_common.py:169-180):
    q < 1/2: 2q P_d(x) + (1 - 2q) P_d(x - c_d);  q >= 1/2: P_d(x)/(2q) + ((2q - 1)/(2q)) P_opp(x),
    each product and sum rounded in the populations' dtype (q promoted to it)."""
    q = f_prev.shape[0]
    t = f_prev.dtype.type
    qv = qf.astype(f_prev.dtype)
    up = stream(f_prev)                                # P_d(x - c_d)
    lin = (qv < t(0.5)) & mask
    quad = (~lin) & mask
    bc_lin = t(2.0) * qv * f_prev + (t(1.0) - t(2.0) * qv) * up
    sq = np.where(quad, qv, t(1.0))
    inv = t(1.0) / (t(2.0) * sq)
    bc_quad = f_prev * inv + (t(2.0) * sq - t(1.0)) * inv * f_prev[opposite(q)]
    return np.where(lin, bc_lin, bc_quad)


def bfl_bounce_back(f: np.ndarray, f_prev: np.ndarray, mask: np.ndarray, qf: np.ndarray) -> np.ndarray:
    """bfl_common.py:106-190: f_out[opp_d](x) = value of link (x, d); f elsewhere.
    f is post-stream, f_prev the pre-stream populations."""
    opp = opposite(f.shape[0])
    bc = _bfl_values(f_prev, mask, qf)
    return np.where(mask[opp], bc[opp], f)


def bfl_force(f_prev: np.ndarray, mask: np.ndarray, qf: np.ndarray) -> np.ndarray:
    """Force ledger of bfl_d3q19.py:339-377 (stationary wall, laboratory frame):
    sum over links of c_d (P_d(x) + value), the pair sum rounded in the
    populations' dtype, accumulated here in float64."""
    q = f_prev.shape[0]
    bc = _bfl_values(f_prev, mask, qf)
    link_sum = (f_prev + bc).astype(np.float64)
    out = np.zeros(3)
    for d in range(1, q):
        out += C[q][d].astype(np.float64) * link_sum[d][mask[d]].sum()
    return out


def bfl_chain_step(f: np.ndarray, tau: float, solid: np.ndarray, mask: np.ndarray, qf: np.ndarray,
                   collision: str = "bgk", **kw):
    """One step in bfl_step's order (bfl_common.py:882-955) after the collision:
    solid cells keep their pre-collision populations, bounce_back_cells_3d on
    the solid, stream, then the link update.  Returns (f, force)."""
    g = np.where(solid[None], f, COLLIDERS[collision](f, tau, **kw))
    g = bounce_back(g, solid)
    return bfl_bounce_back(stream(g), g, mask, qf), bfl_force(g, mask, qf)


# ---------------------------------------------------------------------------
# Link-wise momentum exchange (MEM drag variants)
# ---------------------------------------------------------------------------

def _roll_to_neighbour(a: np.ndarray, c) -> np.ndarray:
    """a[x + c] with periodic wrap (torch.roll(a, -c) in momentum_exchange.py:53-70)."""
    if a.ndim == 2:
        return np.roll(a, shift=(-int(c[1]), -int(c[0])), axis=(0, 1))
    return np.roll(a, shift=(-int(c[2]), -int(c[1]), -int(c[0])), axis=(0, 1, 2))


def link_momentum_sums(f: np.ndarray, solid: np.ndarray, near: np.ndarray, q_wall=None) -> np.ndarray:
    """Per direction q >= 1 over the fluid->solid links (near[x] and
    solid[x + c_q]): the sum of (f_q(x) + f_opp(x + c_q)), weighted by
    1 / max(q_wall, 1e-6) (float32) when q_wall is given, and the link count.
    Per-link values in f's dtype, the sums in float64 (momentum_exchange.py:75-360
    sums each direction in f's dtype).  Returns 2Q float64."""
    q = f.shape[0]
    opp = opposite(q)
    out = np.zeros(2 * q)
    inv = None
    if q_wall is not None:
        inv = (np.float32(1.0) / np.maximum(q_wall.astype(np.float32), np.float32(1e-6))).astype(np.float32)
    for i in range(1, q):
        link = near & _roll_to_neighbour(solid, C[q][i])
        val = f[i] + _roll_to_neighbour(f[opp[i]], C[q][i])
        if inv is not None:
            w = inv[i] if inv.ndim == f.ndim else inv
            val = val * w.astype(f.dtype)
        out[i] = val[link].astype(np.float64).sum()
        out[q + i] = float(link.sum())
    return out


def mem_force(sums: np.ndarray, variant: str = "standard", tau: float = 1.0, rho0: float = 1.0,
              u0=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Force on the wall from the link sums: standard Ladd sum (momentum_exchange.py:75),
    Galilean factor 1 + 1/(2 tau) (:138), the uniform-stream background
    2 rho0 w_q (1 + 4.5 (c_q.u0)^2 - 1.5 |u0|^2) per link removed (:206, with
    the float32 weights of the reference);
    "bfl" is the standard form of the 1/q-weighted sums (:285)."""
    q = sums.size // 2
    c = C[q].astype(np.float64)
    s = sums[:q].copy()
    if variant == "galilean":
        s = s * (1.0 + 1.0 / (2.0 * tau))
    elif variant == "background":
        u = np.zeros(3)
        u[:len(u0)] = u0
        cu = c @ u[:c.shape[1]]
        w32 = W64[q].astype(np.float32).astype(np.float64)       # W.float() in the reference
        bg = 2.0 * rho0 * w32 * (1.0 + 4.5 * cu * cu - 1.5 * float(u @ u))
        s = s - bg * sums[q:]
    elif variant not in ("standard", "bfl"):
        raise ValueError(f"unknown MEM variant {variant!r}")
    s[0] = 0.0
    return (c * s[:, None]).sum(axis=0)


def moving_wall_bounce_back(f: np.ndarray, mask: np.ndarray, *wall_u: np.ndarray) -> np.ndarray:
    """Ladd moving wall: where(mask, bounce_back(f) + ((2 w_q) rho) (c_q . u_w) 3, f),
    rho = sum0(f), the float32 W tensor cast to f's dtype for both lattices and
    c_q . u_w summed x, y, z in order: rotating_cylinder.py:140-190 (D2Q9),
    propeller_benchmark.py:221-270 (D3Q19)."""
    q = f.shape[0]
    dt = f.dtype
    nd = f.ndim - 1
    rho = sum0(f)
    fbb = bounce_back(f, mask)
    c = C[q].astype(dt)
    w = _view(W64[q].astype(np.float32).astype(dt), nd)
    u = [np.asarray(v).astype(dt) for v in wall_u]
    cu = _view(c[:, 0], nd) * u[0][None] + _view(c[:, 1], nd) * u[1][None]
    if len(u) == 3:
        cu = cu + _view(c[:, 2], nd) * u[2][None]
    corr = dt.type(2.0) * w * rho[None] * cu * dt.type(3.0)
    return np.where(mask[None], fbb + corr, fbb)


def zou_he_inlet(f: np.ndarray, u_in: float, uy_in: float = 0.0, uz_in: float = 0.0) -> np.ndarray:
    """x = 0 velocity inlet: boundaries.py:50 (D2Q9), boundaries3d.py:205, boundaries_d3q27.py:107."""
    q = f.shape[0]
    f = f.copy()
    if q == 9:
        f0, f2, f3, f4, f6, f7 = (f[i][:, 0] for i in (0, 2, 3, 4, 6, 7))
        rho = (f0 + f2 + f4 + 2.0 * (f3 + f6 + f7)) / (1.0 - u_in)
        f[1][:, 0] = f3 + (2.0 / 3.0) * rho * u_in
        f[5][:, 0] = f7 - 0.5 * (f2 - f4) + (1.0 / 6.0) * rho * u_in + 0.5 * rho * uy_in
        f[8][:, 0] = f6 + 0.5 * (f2 - f4) + (1.0 / 6.0) * rho * u_in - 0.5 * rho * uy_in
        return f
    c = C[q]
    zero = [i for i in range(q) if c[i, 0] == 0]
    neg = [i for i in range(q) if c[i, 0] < 0]
    pos = [i for i in range(q) if c[i, 0] > 0]
    opp = zou_he_partner(q)
    s0 = f[zero[0]][:, :, 0].copy()
    for i in zero[1:]:
        s0 = s0 + f[i][:, :, 0]
    sn = f[neg[0]][:, :, 0].copy()
    for i in neg[1:]:
        sn = sn + f[i][:, :, 0]
    rho = (s0 + 2.0 * sn) / (1.0 - u_in)
    r3 = rho[..., None]
    dt = f.dtype
    feq = equilibrium(q, r3, np.full_like(r3, u_in, dtype=dt), np.full_like(r3, uy_in, dtype=dt),
                      np.full_like(r3, uz_in, dtype=dt))
    for k in pos:
        f[k][:, :, 0] = feq[k][:, :, 0] - feq[opp[k]][:, :, 0] + f[opp[k]][:, :, 0]
    return f


def zou_he_outlet(f: np.ndarray, rho_out: float = 1.0) -> np.ndarray:
    """x = nx-1 pressure outlet: boundaries.py:102, boundaries3d.py:269, boundaries_d3q27.py:179."""
    q = f.shape[0]
    f = f.copy()
    if q == 9:
        f1, f2, f4, f5, f8 = (f[i][:, -1] for i in (1, 2, 4, 5, 8))
        ux = -1.0 + (f[0][:, -1] + f2 + f4 + 2.0 * (f1 + f5 + f8)) / rho_out
        f[3][:, -1] = f1 - (2.0 / 3.0) * rho_out * ux
        f[7][:, -1] = f5 + 0.5 * (f2 - f4) - (1.0 / 6.0) * rho_out * ux
        f[6][:, -1] = f8 - 0.5 * (f2 - f4) - (1.0 / 6.0) * rho_out * ux
        return f
    c = C[q]
    zero = [i for i in range(q) if c[i, 0] == 0]
    pos = [i for i in range(q) if c[i, 0] > 0]
    neg = [i for i in range(q) if c[i, 0] < 0]
    opp = zou_he_partner(q)
    s0 = f[zero[0]][:, :, -1].copy()
    for i in zero[1:]:
        s0 = s0 + f[i][:, :, -1]
    sp = f[pos[0]][:, :, -1].copy()
    for i in pos[1:]:
        sp = sp + f[i][:, :, -1]
    ux = -1.0 + (s0 + 2.0 * sp) / rho_out
    r3 = np.full_like(ux, rho_out)[..., None]
    feq = equilibrium(q, r3, ux[..., None], np.zeros_like(r3), np.zeros_like(r3))
    for k in neg:
        f[k][:, :, -1] = feq[k][:, :, 0] - feq[opp[k]][:, :, 0] + f[opp[k]][:, :, -1]
    return f


def moving_lid(f: np.ndarray, u_lid: float) -> np.ndarray:
    """Zou/He lid on the whole y = ny-1 plane: lid_driven_cavity.py:431 (D2Q9),
    boundaries3d.py:324 (D3Q19)."""
    f = f.copy()
    if f.shape[0] == 9:
        f0, f1, f2, f3, f5, f6 = (f[i][-1, :].copy() for i in (0, 1, 2, 3, 5, 6))
        rho = f0 + f1 + 2.0 * f2 + f3 + 2.0 * f5 + 2.0 * f6
        f[4][-1, :] = f2
        f[7][-1, :] = f5 + 0.5 * (f1 - f3) - 0.5 * rho * u_lid
        f[8][-1, :] = f6 - 0.5 * (f1 - f3) + 0.5 * rho * u_lid
        return f
    fl = {i: f[i][:, -1, :].copy() for i in range(19)}
    s0 = fl[0] + fl[1] + fl[2] + fl[5] + fl[6] + fl[11] + fl[12] + fl[13] + fl[14]
    sp = fl[3] + fl[7] + fl[10] + fl[15] + fl[17]
    rho = s0 + 2.0 * sp
    sx0 = fl[1] - fl[2] + fl[11] - fl[12] + fl[13] - fl[14]
    dx = rho * u_lid - (sx0 + (fl[7] - fl[10]))
    sz0 = fl[5] - fl[6] + fl[11] - fl[12] - fl[13] + fl[14]
    f[4][:, -1, :] = fl[3]
    f[8][:, -1, :] = 0.5 * (fl[7] + fl[10]) - 0.5 * dx
    f[9][:, -1, :] = 0.5 * (fl[7] + fl[10]) + 0.5 * dx
    f[16][:, -1, :] = fl[15] + 0.5 * sz0
    f[18][:, -1, :] = fl[17] - 0.5 * sz0
    return f


def obstacle_force(f: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """2 sum_solid sum_q c_q f_q in float64: boundaries.py:162, obstacles.py:91, :197."""
    q = f.shape[0]
    fs = f.astype(np.float64)[:, mask]
    c = C[q].astype(np.float64)
    return np.array([2.0 * (c[:, k] @ fs.sum(axis=1)) for k in range(2 if q == 9 else 3)] + ([0.0] if q == 9 else []))


# ---------------------------------------------------------------------------
# masks
# ---------------------------------------------------------------------------


def sphere_mask(nx, ny, nz, cx, cy, cz, radius) -> np.ndarray:
    """float32 (x-cx)^2+(y-cy)^2+(z-cz)^2 <= r^2, boundaries3d.py:29."""
    zz, yy, xx = np.meshgrid(np.arange(nz, dtype=np.float32), np.arange(ny, dtype=np.float32),
                             np.arange(nx, dtype=np.float32), indexing="ij")
    f32 = np.float32
    d = (xx - f32(cx)) ** 2 + (yy - f32(cy)) ** 2 + (zz - f32(cz)) ** 2
    return d <= f32(radius**2)


def cylinder_mask(nx, ny, cx, cy, radius) -> np.ndarray:
    """boundaries.py:8"""
    yy, xx = np.meshgrid(np.arange(ny, dtype=np.float32), np.arange(nx, dtype=np.float32), indexing="ij")
    f32 = np.float32
    return (xx - f32(cx)) ** 2 + (yy - f32(cy)) ** 2 <= f32(radius**2)


def missing_mask(q: int, shape, solid=None, periodic=(False, False, False)) -> np.ndarray:
    """boundary_registry.py:488-575; shape (nz, ny, nx), periodic (z, y, x)."""
    nz, ny, nx = shape
    blocked = np.zeros(shape, dtype=bool) if solid is None else solid.astype(bool)
    out = np.zeros((q,) + tuple(shape), dtype=bool)
    zi, yi, xi = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    for i in range(q):
        cx, cy, cz = (int(v) for v in C[q][i])
        sz, sy, sx = zi - cz, yi - cy, xi - cx
        oob = np.zeros(shape, dtype=bool)
        for src, n, per in ((sz, nz, periodic[0]), (sy, ny, periodic[1]), (sx, nx, periodic[2])):
            if per:
                src %= n
            else:
                oob |= (src < 0) | (src >= n)
                np.clip(src, 0, n - 1, out=src)
        out[i] = oob | blocked[sz, sy, sx]
    return out


def link_index(missing: np.ndarray) -> np.ndarray:
    """Row-major flat indices of the True entries, the order of torch.nonzero
    that boundary_registry.py:488's callers apply to the missing mask."""
    return np.flatnonzero(missing.reshape(-1)).astype(np.int64)


def correct_mass(f: np.ndarray, target_mass: float) -> np.ndarray:
    """f * (target / sum(f)) in the field dtype, unchanged when |sum| < 1e-30:
    solver.py:420-437, solver3d.py:287-300, d3q27.py:729-745.  The sum is taken
    in float64 and then rounded to the field dtype; torch sums float32 in its own
    blocked order, so for float64 fields the scale can differ from the
    reference's by the rounding of the sum (the golden test allows 1e-14)."""
    t = f.dtype.type
    cur = t(f.sum(dtype=np.float64))
    if abs(cur) < 1e-30:
        return f
    return f * (t(target_mass) / cur)


def cavity_walls_3d(n_z, n_y, n_x) -> np.ndarray:
    """Five no-slip walls of benchmarks/verified/cavity_3d_full/run.py:85-89."""
    wall = np.zeros((n_z, n_y, n_x), dtype=bool)
    wall[:, :, 0] = True
    wall[:, :, -1] = True
    wall[:, 0, :] = True
    wall[0, :, :] = True
    wall[-1, :, :] = True
    return wall


# ---------------------------------------------------------------------------
# time-step chains
# ---------------------------------------------------------------------------


def cavity_step(f: np.ndarray, tau: float, wall: np.ndarray, u_lid: float, collision="bgk", mode="fullway",
                **kw) -> np.ndarray:
    """mode "fullway": collide -> stream -> bounce-back on the walls -> Zou/He lid.
    mode "halfway": collide -> where(wall, f_pre[opp], f) -> stream -> lid
    (benchmarks/verified/cavity_3d_full/run.py:58, :95-104)."""
    fc = COLLIDERS[collision](f, tau, **kw)
    if mode == "halfway":
        fc = np.where(wall[None], f[opposite(f.shape[0])], fc)
    f = stream(fc)
    if mode == "fullway":
        f = bounce_back(f, wall)
    return moving_lid(f, u_lid)


def far_field(f: np.ndarray, ux: float, uy: float = 0.0, uz: float = 0.0, z_faces: bool = True,
              inlet_du=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Free-stream far field: boundaries.py:199-220 (D2Q9), boundaries3d.py:446-538
    (D3Q19), boundaries_d3q27.py:63-104 (D3Q27).  feq(1, u) of the lattice's
    equilibrium on the inlet plane, the outlet plane copied from x = nx-2, then
    feq on the y planes (and the z planes with z_faces, 3-D).  inlet_du, the
    seeding of benchmarks/verified/cylinder (run.py:104-113), overwrites the
    inlet plane afterwards with feq(1, u + inlet_du)."""
    q = f.shape[0]
    dt = f.dtype
    one = np.ones((1,) * (f.ndim - 1), dtype=dt)

    def feq_of(vx, vy, vz):
        return equilibrium(q, one, one * dt.type(vx), one * dt.type(vy), None if q == 9 else one * dt.type(vz))

    e = feq_of(ux, uy, uz)
    out = f.copy()
    out[..., 0] = e[..., 0]
    out[..., -1] = out[..., -2]
    if q == 9:
        out[:, 0, :] = e[:, 0, :]
        out[:, -1, :] = e[:, 0, :]
    else:
        out[:, :, 0, :] = e[:, :, 0, :]
        out[:, :, -1, :] = e[:, :, 0, :]
        if z_faces:
            out[:, 0, :, :] = e[:, 0, :, :]
            out[:, -1, :, :] = e[:, 0, :, :]
    if any(v != 0.0 for v in inlet_du):
        out[..., 0] = feq_of(ux + inlet_du[0], uy + inlet_du[1], uz + inlet_du[2])[..., 0]
    return out


def far_field_step(f, tau, u_in, obstacle, collision="bgk", z_faces=True, inlet_du=(0.0, 0.0, 0.0), **kw):
    """collide -> stream -> force -> far field -> bounce-back(obstacle), the chain
    of benchmarks/verified/cylinder/re100/run.py:97-113 and of the 3-D far-field
    runners (sphere_gridconv_re100_worker.py:150-160)."""
    f = COLLIDERS[collision](f, tau, **kw)
    f = stream(f)
    force = obstacle_force(f, obstacle) if obstacle is not None else None
    f = far_field(f, u_in, z_faces=z_faces, inlet_du=inlet_du)
    if obstacle is not None:
        f = bounce_back(f, obstacle)
    return f, force


def channel_step(f, tau, u_in, rho_out, wall, obstacle, collision="bgk", wall_u=None, **kw):
    """collide -> stream -> force -> Zou/He inlet -> outlet -> bounce-back(wall)
    -> bounce-back(obstacle): d3q27_sphere_flow.py:246-256, cylinder_flow.py:854-899.
    With wall_u (the obstacle's wall velocity, one array per axis) the obstacle
    pass is the Ladd moving wall instead, as rotating_cylinder.py:241-253 orders it."""
    f = COLLIDERS[collision](f, tau, **kw)
    f = stream(f)
    force = obstacle_force(f, obstacle) if obstacle is not None else None
    if u_in is not None:
        f = zou_he_inlet(f, u_in)
    if rho_out is not None:
        f = zou_he_outlet(f, rho_out)
    if wall is not None:
        f = bounce_back(f, wall)
    if obstacle is not None:
        f = bounce_back(f, obstacle) if wall_u is None else moving_wall_bounce_back(f, obstacle, *wall_u)
    return f, force
