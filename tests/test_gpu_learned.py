"""The learned self-energy update: device forward/backward kernels against the CPU oracle,
training, the extrapolation kernel against the numpy feature definition, and what the trained
network gains over the plain damped loop (same fixed point, fewer GW evaluations)."""
import numpy as np
import pytest

from coqui_b200 import capi, learned
from coqui_b200.iaft import IAFT
from coqui_b200.synthetic import make_system
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def test_forward_and_gradient_match_oracle():
    net = capi.Mlp(4, 256, 2, seed=1)
    rng = np.random.default_rng(0)
    X = rng.standard_normal((512, 4)).astype(np.float32)
    T = rng.standard_normal((512, 2)).astype(np.float32)
    p = net.params()
    Y_ref, _ = M.forward(p, X, 4, 256, 2)
    assert np.abs(net.forward(X) - Y_ref).max() < 1e-5 * max(1.0, np.abs(Y_ref).max())
    loss, g = net.gradient(X, T)
    loss_ref, g_ref = M.loss_and_grad(p, X, T, 4, 256, 2)
    assert abs(loss - loss_ref) < 1e-5 * loss_ref
    assert np.abs(g - g_ref).max() < 1e-5 * np.abs(g_ref).max()
    net.close()


def test_training_learns_geometric_extrapolation():
    rng = np.random.default_rng(2)
    n = 65536
    rho = rng.uniform(0.05, 0.8, n) * np.exp(1j * rng.uniform(-0.3, 0.3, n))
    X = np.stack([rho.real, rho.imag, rho.real, rho.imag], 1).astype(np.float32)
    tgt = rho / (1 - rho)  # remaining distance of a geometric sequence in units of its last step
    T = np.stack([tgt.real, tgt.imag], 1).astype(np.float32)
    net = capi.Mlp(4, 256, 2, seed=3)
    loss0, _ = net.gradient(X, T)
    hist = net.train(X, T, batch=512, epochs=15, lr=2e-3)  # ~1900 Adam steps
    loss1, _ = net.gradient(X, T)
    assert loss1 < 0.05 * loss0 and loss1 < 1e-2 and hist[-1] < hist[0]
    net.close()


def test_extrapolation_kernel_matches_feature_definition():
    rng = np.random.default_rng(4)
    n = 5000
    s_inf = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    rho = rng.uniform(0.1, 0.7, n)
    d = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * 1e-2
    hist = np.array([s_inf - d * rho ** j / (1 - rho) for j in range(4)])  # geometric approach
    hist[:, :10] = hist[3, :10]  # converged elements: no correction
    net = capi.Mlp(4, 256, 2, seed=5)
    delta = net.extrapolate(hist, max_jump=5.0)
    X, d1, valid = learned.features(hist)
    Y = net.forward(X).astype(np.float64)
    ref = np.where(valid, d1 * (Y[:, 0] + 1j * Y[:, 1]), 0)
    lim = 5.0 * np.abs(d1)
    ref = np.where(np.abs(ref) > lim, ref * lim / np.maximum(np.abs(ref), 1e-300), ref)
    assert not valid[:10].any() and np.all(delta[:10] == 0)
    assert np.abs(delta - ref).max() < 1e-6 * np.abs(ref).max()
    net.close()


def test_learned_loop_needs_fewer_evaluations_and_keeps_the_fixed_point():
    ft = IAFT(1000.0, 10.0, "low")
    trajs = [learned.trajectory(make_system(2, 8, 4, 32, seed=100 + i), ft) for i in range(6)]
    X, T = learned.dataset(trajs, max_samples=400_000)
    net, loss = learned.train(X, T, epochs=12, batch=4096, lr=1e-3)
    assert loss[-1] < loss[0]
    plain = mlp = 0
    for seed in (900, 901):
        s = make_system(2, 8, 4, 32, seed=seed)
        c = learned.make_context(s, ft, capi.FP64)
        a = learned.run_loop(c, s.G0(ft), tol_e=1e-8, tol_r=1e-8)
        b = learned.run_loop(c, s.G0(ft), mlp=net, tol_e=1e-8, tol_r=1e-8)
        assert abs(a["e_tot"] - b["e_tot"]) < 1e-6
        plain += a["evaluations"]
        mlp += b["evaluations"]
        c.close()
    assert mlp < plain
    net.close()
