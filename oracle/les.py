"""CPU oracle for the learned eddy-viscosity closure and the forced LES step.

TEST INFRASTRUCTURE ONLY.  This module checks the CUDA kernels of
tensorlbm_b200.ai: only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline import it.  The product never calls it.

The closure is new (TensorLBM's closure is 2-D: ai/model.py:40-92 maps three
strain components through a 2x16 tanh MLP to nu_t, ai/inference.py:68-92
applies tau + 3 nu_t).  What it shares with the reference and is restated here:

* Smagorinsky tau_eff (turbulence.py:183-208, the fallback and the comparison) through
  oracle.lbm.smagorinsky_tau, i.e. nu_t = C_s^2 |S|_F in lattice units;
* block-mean coarsening (ai/pipeline.py:93 _coarsen_mean, here in 3-D);
* the energy spectrum of benchmarks/pending/dit_turbulence/run.py:158-177
  (rfftn, norm="ortho", shells round(|k|), weight 2 for 0 < kx < N/2).

The network: 9 features -> 64 -> 64 -> 64 (SiLU) -> 1, nu_t = nu_scale *
softplus(y), tau_eff = tau0 + 3 nu_t.  Parameters are one flat vector in the
order W1 (64x9, row = output), b1, W2 (64x64), b2, W3, b3, w4 (64), b4.
"""

from __future__ import annotations

import numpy as np

from oracle import lbm as O

N_FEAT = 9
HIDDEN = 64
C_SMAG = 0.17
SIZES = [("W1", (HIDDEN, N_FEAT)), ("b1", (HIDDEN,)), ("W2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
         ("W3", (HIDDEN, HIDDEN)), ("b3", (HIDDEN,)), ("w4", (HIDDEN,)), ("b4", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(theta: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = theta[o:o + n].reshape(shape)
        o += n
    return out


def init_params(seed: int) -> np.ndarray:
    """Kaiming-uniform weights for SiLU layers, zero biases (float32)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in SIZES:
        if name.startswith("b"):
            parts.append(np.zeros(shape))
        else:
            fan_in = shape[-1] if len(shape) == 2 else HIDDEN
            bound = np.sqrt(6.0 / fan_in) * (0.5 if name == "w4" else 1.0)
            parts.append(rng.uniform(-bound, bound, size=shape))
    return np.concatenate([p.reshape(-1) for p in parts]).astype(np.float32)


# ---------------------------------------------------------------------------
# network
# ---------------------------------------------------------------------------


def sigmoid(a):
    return 1.0 / (1.0 + np.exp(-a))


def silu(a):
    return a * sigmoid(a)


def dsilu(a):
    s = sigmoid(a)
    return s * (1.0 + a * (1.0 - s))


def softplus(y):
    return np.maximum(y, 0.0) + np.log1p(np.exp(-np.abs(y)))


def forward(theta, z):
    """z: (N, 9) normalised features -> (y, cache).  float64."""
    p = {k: v.astype(np.float64) for k, v in unpack(np.asarray(theta, np.float64)).items()}
    z = np.asarray(z, np.float64)
    a1 = z @ p["W1"].T + p["b1"]
    h1 = silu(a1)
    a2 = h1 @ p["W2"].T + p["b2"]
    h2 = silu(a2)
    a3 = h2 @ p["W3"].T + p["b3"]
    h3 = silu(a3)
    y = h3 @ p["w4"] + p["b4"][0]
    return y, (p, z, a1, h1, a2, h2, a3, h3)


def loss_and_grad(theta, z, target, weight):
    """Weighted MSE of softplus(y) against target (both in units of nu_scale):
    L = sum_i w_i (softplus(y_i) - t_i)^2 / N (the weights are normalised to
    mean 1 over the whole data set beforehand).  Returns (L, dL/dtheta)."""
    y, (p, z, a1, h1, a2, h2, a3, h3) = forward(theta, z)
    t = np.asarray(target, np.float64)
    w = np.asarray(weight, np.float64)
    sw = float(len(w))
    sp = softplus(y)
    r = sp - t
    loss = float((w * r * r).sum() / sw)
    dy = 2.0 * w * r / sw * sigmoid(y)
    g = {"w4": h3.T @ dy, "b4": np.array([dy.sum()])}
    d3 = np.outer(dy, p["w4"]) * dsilu(a3)
    g["W3"], g["b3"] = d3.T @ h2, d3.sum(0)
    d2 = (d3 @ p["W3"]) * dsilu(a2)
    g["W2"], g["b2"] = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ p["W2"]) * dsilu(a1)
    g["W1"], g["b1"] = d1.T @ z, d1.sum(0)
    return loss, np.concatenate([g[name].reshape(-1) for name, _ in SIZES])


def adam(theta, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (Kingma & Ba, bias-corrected), float64; step counts from 1."""
    m = b1 * m + (1.0 - b1) * grad
    v = b2 * v + (1.0 - b2) * grad * grad
    mh = m / (1.0 - b1 ** step)
    vh = v / (1.0 - b2 ** step)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v


def bf16(a):
    """Round float32 values to bfloat16 (nearest even) and back to float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def forward_bf16(theta, z):
    """The inference arithmetic of the tensor-core kernels: bf16 inputs and
    weights with float32 accumulation in every layer (the output layer too);
    between layers h = bf16(0.5 (acc + b)) and SiLU = bf16(h + h bf16(tanh h))."""
    p = unpack(np.asarray(theta, np.float32))
    h = bf16(np.asarray(z, np.float32))
    for wn, bn in (("W1", "b1"), ("W2", "b2"), ("W3", "b3")):
        acc = (h.astype(np.float64) @ bf16(p[wn]).astype(np.float64).T).astype(np.float32)
        hh = bf16(np.float32(0.5) * (acc + p[bn]))
        t = bf16(np.tanh(hh.astype(np.float64)).astype(np.float32))
        h = bf16((hh.astype(np.float64) + hh.astype(np.float64) * t.astype(np.float64)).astype(np.float32))
    y = (h.astype(np.float64) @ bf16(p["w4"]).astype(np.float64)).astype(np.float32)
    return (y + p["b4"][0]).astype(np.float32)


# ---------------------------------------------------------------------------
# features of the non-equilibrium stress
# ---------------------------------------------------------------------------


def features(p6, rho, tau0: float, c_s: float = C_SMAG) -> np.ndarray:
    """Nine rotation- and Galilean-invariant inputs from Pi_neq = (xx, yy, zz, xy, xz, yz),
    the density and the molecular tau (float64):
      0 m = |dev Pi|_F / rho        1 log(m + 1e-12)       2 Lode 3 sqrt(6) det(dev Pi) / |dev Pi|^3
      3 tr Pi / rho                 4 rho - 1              5 tau0
      6 tau_s - tau0 (Smagorinsky)  7 m / tau0             8 sqrt(m)"""
    xx, yy, zz, xy, xz, yz = (np.asarray(c, np.float64) for c in p6)
    rho = np.asarray(rho, np.float64)
    tr = xx + yy + zz
    dxx, dyy, dzz = xx - tr / 3.0, yy - tr / 3.0, zz - tr / 3.0
    n2 = dxx * dxx + dyy * dyy + dzz * dzz + 2.0 * (xy * xy + xz * xz + yz * yz)
    nd = np.sqrt(n2)
    det = (dxx * (dyy * dzz - yz * yz) - xy * (xy * dzz - yz * xz) + xz * (xy * yz - dyy * xz))
    lode = np.where(nd > 1e-20, 3.0 * np.sqrt(6.0) * det / np.maximum(nd, 1e-20) ** 3, 0.0)
    lode = np.clip(lode, -1.0, 1.0)
    m = nd / rho
    full = np.sqrt(np.maximum(xx * xx + yy * yy + zz * zz + 2.0 * (xy * xy + xz * xz + yz * yz), 1e-30))
    disc = np.maximum(tau0 * tau0 + 18.0 * c_s * c_s * full / rho, 0.0)
    tau_s = np.clip(0.5 * (tau0 + np.sqrt(disc)), 0.5001, max(1.0, tau0 + 0.5))
    return np.stack([m, np.log(m + 1e-12), lode, tr / rho, rho - 1.0, np.full_like(m, tau0), tau_s - tau0,
                     m / tau0, np.sqrt(m)], axis=-1)


# ---------------------------------------------------------------------------
# filtered-DNS training samples
# ---------------------------------------------------------------------------


def coarsen(field: np.ndarray, factor: int) -> np.ndarray:
    """Block mean over factor^3 cells of the trailing three axes (ai/pipeline.py:93 in 3-D)."""
    *lead, nz, ny, nx = field.shape
    f = field.reshape(*lead, nz // factor, factor, ny // factor, factor, nx // factor, factor)
    return f.mean(axis=(-5, -3, -1))


def filtered_moments(rho, u, factor: int) -> np.ndarray:
    """(10, ...) block means of rho, u_x, u_y, u_z, u_xu_x, u_yu_y, u_zu_z, u_xu_y, u_xu_z, u_yu_z."""
    ux, uy, uz = (np.asarray(c, np.float64) for c in u)
    ch = [np.asarray(rho, np.float64), ux, uy, uz, ux * ux, uy * uy, uz * uz, ux * uy, ux * uz, uy * uz]
    return np.stack([coarsen(c, factor) for c in ch])


def strain(ub):
    """S_ij = (d_i u_j + d_j u_i) / 2 by periodic central differences, order (xx, yy, zz, xy, xz, yz)."""
    def d(a, axis):  # axis: 0 = x (last array axis), 1 = y, 2 = z
        ax = 2 - axis
        return 0.5 * (np.roll(a, -1, axis=ax) - np.roll(a, 1, axis=ax))
    g = [[d(ub[j], i) for j in range(3)] for i in range(3)]  # g[i][j] = d_i u_j
    return (g[0][0], g[1][1], g[2][2], 0.5 * (g[0][1] + g[1][0]), 0.5 * (g[0][2] + g[2][0]),
            0.5 * (g[1][2] + g[2][1]))


def les_samples(mom: np.ndarray, tau0: float, nu_of=None):
    """Training samples of one filtered field (float64).

    target nu* = -(tau_sgs_dev : S) / (2 S:S); weight = S:S (so that the
    weighted-MSE optimum matches the subgrid dissipation in every feature bin).
    The LES sees Pi_neq = -2 rho c_s^2 tau_eff S = -(2/3) rho tau_eff S; tau_eff
    is tau0 + 3 nu_of(S-features) if given, else the Smagorinsky tau."""
    rho, ux, uy, uz = mom[0], mom[1], mom[2], mom[3]
    t_sgs = (mom[4] - ux * ux, mom[5] - uy * uy, mom[6] - uz * uz, mom[7] - ux * uy, mom[8] - ux * uz,
             mom[9] - uy * uz)
    s = strain((ux, uy, uz))
    ss = s[0] ** 2 + s[1] ** 2 + s[2] ** 2 + 2.0 * (s[3] ** 2 + s[4] ** 2 + s[5] ** 2)
    trt = (t_sgs[0] + t_sgs[1] + t_sgs[2]) / 3.0
    tds = ((t_sgs[0] - trt) * s[0] + (t_sgs[1] - trt) * s[1] + (t_sgs[2] - trt) * s[2]
           + 2.0 * (t_sgs[3] * s[3] + t_sgs[4] * s[4] + t_sgs[5] * s[5]))
    nu_star = -tds / (2.0 * ss + 1e-30)
    if nu_of is None:
        tau_eff = tau0 + 3.0 * C_SMAG ** 2 * np.sqrt(ss)
    else:
        tau_eff = tau0 + 3.0 * nu_of(s, rho)
    p6 = [-(2.0 / 3.0) * rho * tau_eff * c for c in s]
    x = features(p6, rho, tau0)
    return x.reshape(-1, N_FEAT), nu_star.reshape(-1), ss.reshape(-1)


# ---------------------------------------------------------------------------
# forced collisions (exact-difference forcing, linear Lundgren force F = A rho u)
# ---------------------------------------------------------------------------


def forced_bgk(f: np.ndarray, tau_eff, a_lin: float) -> np.ndarray:
    """f - (f - feq(rho, u)) / tau_eff + feq(rho, u + A u) - feq(rho, u), float64."""
    f = np.asarray(f, np.float64)
    rho, ux, uy, uz = O.macroscopic(f)
    feq = O.equilibrium(19, rho, ux, uy, uz)
    out = f - (f - feq) / np.asarray(tau_eff)[None] if np.ndim(tau_eff) else f - (f - feq) / tau_eff
    if a_lin != 0.0:
        k = 1.0 + a_lin
        out = out + O.equilibrium(19, rho, ux * k, uy * k, uz * k) - feq
    return out


def energy_spectrum(u: np.ndarray) -> np.ndarray:
    """E(k), k = 0..kmax, of a periodic (3, n, n, n) field (run.py:158-177 conventions)."""
    n = u.shape[-1]
    uh = np.fft.rfftn(u, axes=(1, 2, 3), norm="ortho")
    kx = np.fft.rfftfreq(n) * n
    ky = np.fft.fftfreq(n) * n
    kz = np.fft.fftfreq(n) * n
    KZ, KY, KX = np.meshgrid(kz, ky, kx, indexing="ij")
    idx = np.rint(np.sqrt(KX * KX + KY * KY + KZ * KZ)).astype(np.int64)
    w = np.where((KX > 0) & (KX < n // 2), 2.0, 1.0)
    e = 0.5 * (np.abs(uh) ** 2).sum(0) * w
    return np.bincount(idx.reshape(-1), weights=e.reshape(-1)) / n ** 3
