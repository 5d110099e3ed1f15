"""CPU checks of the learned-closure oracle (oracle/les.py): the hand-written
backward against torch autograd in float64, Adam, the bf16 rounding, the
feature map's invariances and the filtered-DNS sample algebra."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import les as L
from oracle import lbm as O


def _torch_loss(theta, z, t, w):
    p = {}
    o = 0
    for name, shape in L.SIZES:
        n = int(np.prod(shape))
        p[name] = theta[o:o + n].reshape(shape)
        o += n
    h = z
    for wn, bn in (("W1", "b1"), ("W2", "b2"), ("W3", "b3")):
        h = torch.nn.functional.silu(h @ p[wn].T + p[bn])
    y = h @ p["w4"] + p["b4"][0]
    r = torch.nn.functional.softplus(y) - t
    return (w * r * r).sum() / z.shape[0]


def test_backward_matches_autograd_f64():
    rng = np.random.default_rng(3)
    theta = L.init_params(5).astype(np.float64)
    z = rng.standard_normal((200, L.N_FEAT))
    t = np.abs(rng.standard_normal(200))
    w = rng.uniform(0.2, 2.0, 200)
    loss, g = L.loss_and_grad(theta, z, t, w)
    th = torch.tensor(theta, requires_grad=True)
    lt = _torch_loss(th, torch.tensor(z), torch.tensor(t), torch.tensor(w))
    lt.backward()
    assert abs(loss - float(lt.detach())) <= 1e-12 * abs(loss)
    assert np.max(np.abs(g - th.grad.numpy())) <= 1e-10 * np.max(np.abs(g))


def test_backward_finite_differences():
    rng = np.random.default_rng(4)
    theta = L.init_params(6).astype(np.float64)
    z = rng.standard_normal((40, L.N_FEAT))
    t = np.abs(rng.standard_normal(40))
    w = np.ones(40)
    _, g = L.loss_and_grad(theta, z, t, w)
    for i in rng.choice(theta.size, 25, replace=False):
        e = np.zeros_like(theta)
        e[i] = 1e-6
        fd = (L.loss_and_grad(theta + e, z, t, w)[0] - L.loss_and_grad(theta - e, z, t, w)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


def test_adam_matches_torch():
    rng = np.random.default_rng(5)
    theta = rng.standard_normal(50)
    th = torch.tensor(theta.copy(), requires_grad=True)
    opt = torch.optim.Adam([th], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    m = np.zeros(50)
    v = np.zeros(50)
    for step in range(1, 6):
        grad = rng.standard_normal(50)
        theta, m, v = L.adam(theta, grad, m, v, step, 1e-2)
        th.grad = torch.tensor(grad)
        opt.step()
    assert np.max(np.abs(theta - th.detach().numpy())) < 1e-12


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(6)
    a = (rng.standard_normal(10000) * np.exp(rng.uniform(-20, 20, 10000))).astype(np.float32)
    want = torch.tensor(a).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(L.bf16(a), want)


def test_features_rotation_invariant():
    rng = np.random.default_rng(7)
    a = rng.standard_normal((3, 3)) * 1e-3
    p = a + a.T
    q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    pr = q @ p @ q.T
    six = lambda m: (m[0, 0], m[1, 1], m[2, 2], m[0, 1], m[0, 2], m[1, 2])  # noqa: E731
    x1 = L.features(six(p), 1.01, 0.52)
    x2 = L.features(six(pr), 1.01, 0.52)
    assert np.allclose(x1, x2, rtol=1e-9, atol=1e-12)
    # the Smagorinsky feature agrees with the oracle's turbulence.py restatement
    full = np.sqrt(np.sum(p * p))
    ts = O.smagorinsky_tau(0.52, np.array(full), np.array(1.01), 0.17)
    assert abs(x1[6] - (float(ts) - 0.52)) < 1e-12


def test_samples_of_a_filtered_laminar_shear_have_zero_sgs():
    # a shear flow u_x(y) sampled one cell per block (factor 1): no subgrid stress
    n = 16
    y = np.arange(n, dtype=np.float64)
    ux = np.broadcast_to((1e-3 * np.sin(2 * np.pi * y / n))[None, :, None], (n, n, n))
    u = np.stack([ux, np.zeros_like(ux), np.zeros_like(ux)])
    mom = L.filtered_moments(np.ones((n, n, n)), u, 1)
    x, nu, ss = L.les_samples(mom, 0.52)
    assert np.allclose(nu, 0.0, atol=1e-14)
    assert x.shape == (n ** 3, 9) and np.all(np.isfinite(x))


def test_energy_spectrum_parseval():
    rng = np.random.default_rng(8)
    u = rng.standard_normal((3, 16, 16, 16))
    e = L.energy_spectrum(u)
    assert abs(e.sum() - 0.5 * np.mean(np.sum(u * u, axis=0))) < 1e-12


@pytest.mark.parametrize("a_lin", [0.0, 1e-3])
def test_forced_bgk_adds_the_force(a_lin):
    # exact-difference forcing: the momentum gains A rho u per step, mass unchanged
    rng = np.random.default_rng(9)
    sp = (4, 4, 32)
    rho = 1.0 + 0.01 * rng.standard_normal(sp)
    u = [0.02 * rng.standard_normal(sp) for _ in range(3)]
    f = O.equilibrium(19, rho, *u) + 1e-4 * rng.standard_normal((19,) + sp)
    r0, ux0, uy0, uz0 = O.macroscopic(f)
    out = L.forced_bgk(f, 0.6, a_lin)
    r1, ux1, uy1, uz1 = O.macroscopic(out)
    assert np.allclose(r1, r0, rtol=0, atol=1e-13)
    assert np.allclose(r1 * ux1, r0 * ux0 * (1 + a_lin), rtol=0, atol=1e-13)
