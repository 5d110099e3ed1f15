"""GPU parity of the learned LES closure against the CPU oracle (oracle/les.py):
training gradients and Adam, fp32 and tensor-core inference, filtered-DNS
samples, the fused LES step and the forced generic step."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import lbm as O
from oracle import les as L

pytestmark = pytest.mark.gpu


def T(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def N(t):
    return t.detach().cpu().numpy()


def _model(dev, seed=1, n_stats=4000):
    from tensorlbm_b200.ai import EddyViscosityMLP3D

    m = EddyViscosityMLP3D(dev, seed=seed)
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n_stats, 9)).astype(np.float32) * np.linspace(0.5, 3.0, 9, dtype=np.float32) + 0.3
    m.set_feature_stats(T(x, dev), margin=0.05)
    m.nu_scale = 0.01
    return m


def test_param_layout_matches_oracle(cuda):
    from tensorlbm_b200 import _lib

    assert int(_lib.load().tlbm_mlp_param_count()) == L.N_PARAMS
    assert int(_lib.load().tlbm_mlp_blob_bytes()) % 128 == 0


@pytest.mark.parametrize("count", [64, 300])
def test_grad_kernel_matches_oracle(cuda, count):
    from tensorlbm_b200 import _lib

    m = _model(cuda)
    rng = np.random.default_rng(2)
    n_rows = 500
    x = (rng.standard_normal((n_rows, 9)) * 1.5 + 0.3).astype(np.float32)
    t = np.abs(rng.standard_normal(n_rows)).astype(np.float32)
    w = rng.uniform(0.3, 2.0, n_rows).astype(np.float32)
    idx = rng.permutation(n_rows)[:count].astype(np.int64)
    lib = _lib.load()
    nb = int(lib.tlbm_mlp_grad_blocks(count))
    partial = torch.empty(nb * (L.N_PARAMS + 1), dtype=torch.float32, device=cuda)
    xd, td, wd, idd = T(x, cuda), T(t, cuda), T(w, cuda), T(idx, cuda)
    istd = m.istd
    _lib.check(lib.tlbm_mlp_grad(m.theta.data_ptr(), m.mean.data_ptr(), istd.data_ptr(), xd.data_ptr(), td.data_ptr(),
                                 wd.data_ptr(), idd.data_ptr(), count, partial.data_ptr(),
                                 _lib.stream_of(cuda)), "grad")
    g = torch.empty(L.N_PARAMS, dtype=torch.float32, device=cuda)
    loss = torch.empty(1, dtype=torch.float32, device=cuda)
    zeros = torch.zeros_like(m.theta)
    _lib.check(lib.tlbm_mlp_adam(m.theta.data_ptr(), zeros.data_ptr(), zeros.clone().data_ptr(), partial.data_ptr(), nb,
                                 0.0, 0.9, 0.999, 1e-8, 1, g.data_ptr(), loss.data_ptr(), _lib.stream_of(cuda)),
               "adam")
    z = (x[idx] - N(m.mean)) * N(istd)
    lo, go = L.loss_and_grad(N(m.theta), z, t[idx], w[idx])
    assert abs(float(loss.item()) - lo) <= 2e-5 * abs(lo)
    gd = N(g).astype(np.float64)
    assert np.max(np.abs(gd - go)) <= 2e-4 * np.max(np.abs(go))
    assert np.array_equal(N(m.theta), N(_model(cuda).theta))  # lr = 0: no update


def test_adam_matches_oracle(cuda):
    from tensorlbm_b200 import _lib

    m = _model(cuda)
    rng = np.random.default_rng(3)
    count = 256
    x = (rng.standard_normal((count, 9)) + 0.3).astype(np.float32)
    t = np.abs(rng.standard_normal(count)).astype(np.float32)
    lib = _lib.load()
    nb = int(lib.tlbm_mlp_grad_blocks(count))
    partial = torch.empty(nb * (L.N_PARAMS + 1), dtype=torch.float32, device=cuda)
    mm, vv = torch.zeros_like(m.theta), torch.zeros_like(m.theta)
    g = torch.empty_like(m.theta)
    theta_o = N(m.theta).astype(np.float64)
    mo, vo = np.zeros_like(theta_o), np.zeros_like(theta_o)
    xd, td = T(x, cuda), T(t, cuda)
    for step in range(1, 4):
        _lib.check(lib.tlbm_mlp_grad(m.theta.data_ptr(), m.mean.data_ptr(), m.istd.data_ptr(), xd.data_ptr(),
                                     td.data_ptr(), None, None, count, partial.data_ptr(), _lib.stream_of(cuda)), "g")
        _lib.check(lib.tlbm_mlp_adam(m.theta.data_ptr(), mm.data_ptr(), vv.data_ptr(), partial.data_ptr(), nb, 1e-3,
                                     0.9, 0.999, 1e-8, step, g.data_ptr(), None, _lib.stream_of(cuda)), "adam")
        theta_o, mo, vo = L.adam(theta_o, N(g).astype(np.float64), mo, vo, step, 1e-3)
    assert np.max(np.abs(N(m.theta) - theta_o)) < 1e-6


def test_eval_and_tensor_core_inference(cuda):
    m = _model(cuda, seed=4)
    rng = np.random.default_rng(5)
    count = 1000  # not a multiple of the 256-row tile
    x = (rng.standard_normal((count, 9)) * np.linspace(0.5, 3.0, 9) + 0.3).astype(np.float32)
    z = (x - N(m.mean)) * N(m.istd)
    y32 = N(m.forward(T(x, cuda)))
    y64, _ = L.forward(N(m.theta), z)
    assert np.max(np.abs(y32 - y64)) <= 1e-4 * (1.0 + np.max(np.abs(y64)))
    ytc = N(m.infer(T(x, cuda)))
    ybf = L.forward_bf16(N(m.theta), z.astype(np.float32))
    scale = 1.0 + np.max(np.abs(ybf))
    # same bf16 operands; only the fp32 accumulation order and SiLU's exp differ
    assert np.max(np.abs(ytc - ybf)) <= 2e-2 * scale
    assert np.mean(np.abs(ytc - ybf)) <= 2e-3 * scale
    # and bf16 inference stays close to the fp32 network
    assert np.max(np.abs(ytc - y64)) <= 6e-2 * scale


def test_filtered_moments_and_samples_match_oracle(cuda):
    from tensorlbm_b200.ai import filtered_moments, les_samples

    rng = np.random.default_rng(6)
    sp = (16, 32, 64)
    rho = (1.0 + 0.01 * rng.standard_normal(sp)).astype(np.float32)
    u = [(0.03 * rng.standard_normal(sp)).astype(np.float32) for _ in range(3)]
    f = O.equilibrium(19, rho, *u)
    a_lin = 2e-3
    mom = filtered_moments(T(f, cuda), 2, a_lin)
    r64, ux, uy, uz = O.macroscopic(f.astype(np.float64))
    k = 1.0 + 0.5 * a_lin
    want = L.filtered_moments(r64, (ux * k, uy * k, uz * k), 2)
    got = N(mom).astype(np.float64)
    assert np.max(np.abs(got - want)) <= 1e-6 * np.max(np.abs(want))
    x, t, w = les_samples(mom, 0.53, 0.17)
    xo, to, wo = L.les_samples(got, 0.53)
    assert np.max(np.abs(N(w) - wo)) <= 1e-6 * np.max(wo)
    assert np.max(np.abs(N(t) - to)) <= 1e-4 * np.max(np.abs(to))
    xg = N(x).astype(np.float64)
    for j in range(9):
        scale = max(np.max(np.abs(xo[:, j])), 1e-30)
        assert np.max(np.abs(xg[:, j] - xo[:, j])) <= 1e-5 * scale, j


def _les_oracle(f_post, tau0, c_s, a_lin, model):
    """One fused LES step in float64 except the network (bf16 arithmetic).
    Returns (relax(tau) -> post-collision field, tau_eff, in-range mask)."""
    f = O.stream(f_post.astype(np.float64))
    rho, ux, uy, uz = O.macroscopic(f)
    feq = O.equilibrium(19, rho, ux, uy, uz)
    p6 = O.neq_stress(f - feq)
    x = L.features(p6, rho, tau0, c_s).reshape(-1, 9)
    lo, hi = N(model.lo), N(model.hi)
    x32 = x.astype(np.float32)  # the kernel tests its float32 features
    inr = np.all((x32 >= lo) & (x32 <= hi), axis=1)
    z = ((x32 - N(model.mean)) * N(model.istd)).astype(np.float32)
    y = L.forward_bf16(N(model.theta), z).astype(np.float64)
    nu = model.nu_scale * L.softplus(y)
    tmax = max(1.0, tau0 + 0.5)
    tau = np.clip(tau0 + 3.0 * nu, 0.5001, tmax)
    tau = np.where(inr, tau, x[:, 6] + tau0).reshape(rho.shape)

    def relax(tau_eff):
        out = f - (f - feq) / tau_eff[None]
        if a_lin:
            k = 1.0 + a_lin
            out = out + O.equilibrium(19, rho, ux * k, uy * k, uz * k) - feq
        return out

    return relax, tau, inr.reshape(rho.shape)


@pytest.mark.parametrize("cut", [False, True])
def test_fused_les_step_matches_oracle(cuda, cut):
    from tensorlbm_b200.ai import LearnedLESSolver

    rng = np.random.default_rng(7)
    sp = (16, 32, 64)
    rho = (1.0 + 0.005 * rng.standard_normal(sp)).astype(np.float32)
    u = [(0.04 * rng.standard_normal(sp)).astype(np.float32) for _ in range(3)]
    f0 = (O.equilibrium(19, rho, *u) * (1.0 + 0.01 * rng.standard_normal((19,) + sp))).astype(np.float32)
    tau0, c_s, a_lin = 0.52, 0.17, 1e-3
    model = _model(cuda, seed=8)
    # features of this field, so that the fallback range is meaningful
    fo = O.stream(f0.astype(np.float64))
    r, a, b, c = O.macroscopic(fo)
    xs = L.features(O.neq_stress(fo - O.equilibrium(19, r, a, b, c)), r, tau0, c_s).reshape(-1, 9)
    model.set_feature_stats(T(xs.astype(np.float32), cuda), margin=0.5)
    if cut:  # cells whose stress magnitude exceeds the median take the fallback
        model.hi[0] = float(np.median(xs[:, 0]))
        model.invalidate()
    s = LearnedLESSolver(sp, tau0, model, force_lin=a_lin, c_s=c_s, device=cuda, track_tau=True)
    s.load(T(f0, cuda)).step(1)
    torch.cuda.synchronize(cuda)
    assert int(s.status.item()) == 0
    relax, tau_w, inr = _les_oracle(f0, tau0, c_s, a_lin, model)
    got = N(s.state).astype(np.float64)
    tau_g = N(s.tau).astype(np.float64)
    if cut:  # borderline cells may fall either side of the cut
        assert 0 < int(s.fallback.item()) < np.prod(sp)
    else:
        assert int(s.fallback.item()) == int((~inr).sum()) == 0
    # tau_eff: the network in bf16 on the tensor cores against its bf16
    # restatement; the hardware bf16x2 tanh and the bf16 roundings between
    # layers leave a few percent of nu_t (the y bound of the inference test)
    dnu = np.abs(tau_g - tau_w)
    span = np.max(tau_w - tau0)
    assert np.max(dnu) <= 5e-2 * span
    assert np.mean(dnu) <= 1e-2 * span
    # the LBM arithmetic around it (pull, moments, relaxation, forcing) at the kernel's own tau
    # (together with the tau bound above this bounds the whole step against the oracle)
    want = relax(tau_g)
    assert np.max(np.abs(got - want)) <= 2e-6 * np.max(np.abs(want))


def _forced(f, coll, tau, a_lin):
    """collide (oracle, float64) then the exact-difference force term"""
    f = np.asarray(f, np.float64)
    rho, ux, uy, uz = O.macroscopic(f)
    k = 1.0 + a_lin
    out = O.COLLIDERS[coll](f, tau)
    return out + O.equilibrium(19, rho, ux * k, uy * k, uz * k) - O.equilibrium(19, rho, ux, uy, uz)


@pytest.mark.parametrize("coll", ["bgk", "mrt", "smagorinsky"])
def test_forced_generic_step_matches_oracle(cuda, coll):
    from tensorlbm_b200 import LBMSolver

    rng = np.random.default_rng(9)
    sp = (8, 16, 64)
    rho = (1.0 + 0.01 * rng.standard_normal(sp)).astype(np.float32)
    u = [(0.03 * rng.standard_normal(sp)).astype(np.float32) for _ in range(3)]
    f0 = O.equilibrium(19, rho, *u) * (1.0 + 0.002 * rng.standard_normal((19,) + sp)).astype(np.float32)
    a_lin, tau = 2e-3, 0.56
    kw = {"c_smag": 0.1} if coll == "smagorinsky" else {}
    s = LBMSolver("D3Q19", sp, tau, coll, device=cuda, force_lin=a_lin, **kw)
    s.load(T(f0, cuda)).step(2)
    ref = _forced(f0, coll, tau, a_lin)
    for _ in range(2):
        ref = _forced(O.stream(ref), coll, tau, a_lin)
    # the stored post-collision state P_2
    got = N(s._buf[s._cur]).astype(np.float64)
    assert np.max(np.abs(got - ref)) <= 2e-6 * np.max(np.abs(ref))
