"""CPU checks of the learned proposer's oracle and host logic: BF16 rounding,
the analytic gradient against central finite differences, and the host-side
initialisation / standardisation of hhg_mlp_init (no kernel is launched)."""
import numpy as np
import pytest
import torch

from higherharmonics_b200 import api
from oracle import mlp_oracle as MO


def _records(n, seed=3):
    rng = np.random.default_rng(seed)
    rec = np.zeros((n, api.HIST_FIELDS), np.float32)
    rec[:, :8] = rng.normal(size=(n, 8)) * np.array([0.5, 0.5, 1.0, 0.05, 0.6, 0.6, 0.5, 2.0]) + \
        np.array([0.0, 0.0, 0.0, 0.0, 0.0, 0.0, -0.5, -3.0])
    x = rec[:, :8].astype(np.float64)
    rec[:, 8] = 2.0 + np.sin(3 * x[:, 0]) + 0.5 * x[:, 2] ** 2 + 4 * np.abs(x[:, 3]) + 0.3 * x[:, 7]
    return rec


def test_bf16_rounding_matches_torch():
    assert MO.bf16(np.float32(1.0)) == 1.0
    assert MO.bf16(np.float32(1 + 2 ** -8)) == 1.0                    # tie -> even
    assert MO.bf16(np.float32(1 + 3 * 2 ** -8)) == np.float32(1 + 2 ** -6)
    x = np.random.default_rng(0).normal(size=100000).astype(np.float32) * 10.0 ** \
        np.random.default_rng(1).integers(-20, 20, size=100000)
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(MO.bf16(x), ref)


def test_layout_matches_abi():
    assert MO.N_PARAMS == api.MLP_N_PARAMS
    assert MO.LAYOUT == api.MLP_LAYOUT


def test_gradient_matches_finite_differences():
    rec = _records(64)
    net = api.mlp_init(7, rec)
    flat = net.param_array().astype(np.float64)
    args = (np.array(net.in_mu), np.array(net.in_isig), net.out_mu, net.out_sigma)
    loss, g = MO.loss_and_grad(flat, rec, *args, emulate=False)
    rng = np.random.default_rng(5)
    idx = np.concatenate([rng.choice(MO.N_PARAMS, 60, replace=False), [MO.N_PARAMS - 1]])
    eps = 1e-6
    for i in idx:
        fp, fm = flat.copy(), flat.copy()
        fp[i] += eps
        fm[i] -= eps
        lp, _ = MO.loss_and_grad(fp, rec, *args, emulate=False)
        lm, _ = MO.loss_and_grad(fm, rec, *args, emulate=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_emulated_gradient_close_to_exact():
    rec = _records(512)
    net = api.mlp_init(11, rec)
    args = (np.array(net.in_mu), np.array(net.in_isig), net.out_mu, net.out_sigma)
    l0, g0 = MO.loss_and_grad(net.param_array(), rec, *args, emulate=False)
    l1, g1 = MO.loss_and_grad(net.param_array(), rec, *args, emulate=True)
    assert abs(l1 - l0) <= 2e-2 * l0
    assert np.linalg.norm(g1 - g0) <= 3e-2 * np.linalg.norm(g0)


def test_mlp_init_is_deterministic_and_fits_standardisation():
    rec = _records(5000)
    a = api.mlp_init(42, rec)
    b = api.mlp_init(42, rec)
    c = api.mlp_init(43, rec)
    assert np.array_equal(a.param_array(), b.param_array())
    assert not np.array_equal(a.param_array(), c.param_array())
    t = a.tensors()
    assert np.all(np.abs(t["w1"]) <= 1 / np.sqrt(8) + 1e-7)
    assert np.all(np.abs(t["w2"]) <= 1 / 8 + 1e-7)
    assert t["b4"][0] == 0.0
    x = rec[:, :8].astype(np.float64)
    assert np.allclose(np.array(a.in_mu), x.mean(0), rtol=1e-5, atol=1e-6)
    assert np.allclose(np.array(a.in_isig), 1 / x.std(0), rtol=1e-4)
    assert np.isclose(a.out_mu, rec[:, 8].astype(np.float64).mean(), rtol=1e-5)
    assert np.isclose(a.out_sigma, rec[:, 8].astype(np.float64).std(), rtol=1e-4)
    assert a.level_margin == pytest.approx(-0.5)
    # a constant input keeps isig = 1
    rec2 = rec.copy()
    rec2[:, 1] = 0.5
    d = api.mlp_init(1, rec2)
    assert d.in_isig[1] == 1.0

