"""Learned self-energy update of the self-consistent GW loop: trajectories of the plain damped
loop, the training set, device training, and loops with and without the network.

The network sees, for every diagonal element Sigma_ii^k(i w_n), the last four iterates of the
damped loop through the ratios of successive differences q1 = d1/d2, q2 = d2/d3 (d1 the newest
difference) and proposes (Sigma_inf - s3)/d1, the remaining distance to the fixed point in
units of the last step.  The loop adds the proposal and keeps it only if the next residual
max|Sigma_GW - Sigma_in| does not grow (coqui_b200_scgw_set_mlp), so the converged fixed point
is that of the plain iteration.  The feature definition here is the one of the device kernel
(k_extrap_features) used at inference.
"""
import time

import numpy as np

from . import capi


def features(hist):
    """hist (4, n) complex, oldest first -> (X (n, 4) float32, d1 (n,), valid (n,) bool)."""
    s0, s1, s2, s3 = hist
    d1, d2, d3 = s3 - s2, s2 - s1, s1 - s0
    scale = np.maximum(np.abs(s3), 1e-300)
    valid = (np.abs(d1) > 1e-14 * scale) & (np.abs(d2) > 1e-14 * scale) & (np.abs(d3) > 1e-14 * scale)
    with np.errstate(divide="ignore", invalid="ignore"):
        q1 = np.where(valid, d1 / np.where(valid, d2, 1), 0)
        q2 = np.where(valid, d2 / np.where(valid, d3, 1), 0)
    X = np.stack([q1.real, q1.imag, q2.real, q2.imag], 1).clip(-4, 4).astype(np.float32)
    return X, d1, valid


def make_context(s, ft, mode=capi.MIXED):
    H0, S, F = s.mean_field()
    c = capi.Context(s.nk, s.nb, s.Np, ft.nt_f, ft.nw_b, s.kp_grid, mode=mode)
    c.set_ir(ft)
    c.set_ir_fermi(ft)
    c.set_kmesh(s.kpts, s.lattv, s.chi_bar)
    c.set_thc(s.X, s.V)
    c.set_mean_field(H0, S, F, s.mu)
    return c


def run_loop(c, G0, mixing=0.7, alg="damping", mlp=None, max_jump=5.0, tol_e=1e-6, tol_r=1e-6,
             max_iter=80, record=False):
    """Iterate until |E_tot(t) - E_tot(t-1)| < tol_e and the residual < tol_r.  Returns a dict with
    iterations, GW evaluations, wall time, energies, and (record) the diag Sigma_in(i w) per
    iteration."""
    c.set_iter_alg(alg, mixing, 5, 5 if alg == "diis" else 1)
    c.set_mlp(mlp, mlp is not None, max_jump)
    e_prev, evals, hist, rec = None, 0, [], []
    t0 = time.perf_counter()
    it = 0
    for it in range(1, max_iter + 1):
        st = c.scgw_iteration(it, G0 if it == 1 else None)
        evals += st["evaluations"]
        hist.append(st)
        if record:
            rec.append(c.sigma_diag_w())
        done = e_prev is not None and abs(st["e_tot"] - e_prev) < tol_e and st["residual"] < tol_r
        e_prev = st["e_tot"]
        if done:
            break
    wall = time.perf_counter() - t0
    out = dict(iterations=it, evaluations=evals, wall_s=wall, e_tot=hist[-1]["e_tot"],
               e_corr=hist[-1]["e_corr"], history=hist,
               learned_steps=sum(1 for h in hist if h["learned"] == 1),
               withdrawn=sum(1 for h in hist if h["learned"] == -1))
    if record:
        out["diag_w"] = np.array(rec)
    return out


def trajectory(s, ft, mixing=0.7, tol=1e-11, max_iter=40, mode=capi.FP64):
    """diag Sigma_in(i w) of every iteration of the plain damped loop, run to tol (FP64 by
    default, so that the tail of the trajectory is not mixed-precision noise)."""
    c = make_context(s, ft, mode)
    r = run_loop(c, s.G0(ft), mixing=mixing, tol_e=tol, tol_r=tol, max_iter=max_iter, record=True)
    c.close()
    return r["diag_w"].reshape(r["diag_w"].shape[0], -1)


def dataset(trajs, max_samples=2_000_000, target_clip=5.0, min_step=1e-9, seed=0):
    """(X, T) from trajectories (list of (n_iter, n_el) complex): every window of four iterates
    whose differences exceed min_step |s3| (well above the rounding of the converged tail),
    target (s_final - s3)/d1 clipped to target_clip."""
    Xs, Ts = [], []
    for tr in trajs:
        s_inf = tr[-1]
        for t in range(3, tr.shape[0] - 1):
            X, d1, valid = features(tr[t - 3:t + 1])
            w = tr[t - 3:t + 1]
            floor = min_step * np.maximum(np.abs(w[3]), 1e-300)
            valid &= (np.abs(w[1] - w[0]) > floor) & (np.abs(w[2] - w[1]) > floor) & (np.abs(d1) > floor)
            tgt = (s_inf - tr[t])[valid] / d1[valid]
            a = np.abs(tgt)
            tgt = np.where(a > target_clip, tgt * target_clip / np.maximum(a, 1e-300), tgt)
            Xs.append(X[valid])
            Ts.append(np.stack([tgt.real, tgt.imag], 1).astype(np.float32))
    X, T = np.concatenate(Xs), np.concatenate(Ts)
    if X.shape[0] > max_samples:
        idx = np.random.default_rng(seed).choice(X.shape[0], max_samples, replace=False)
        X, T = X[idx], T[idx]
    return X, T


def train(X, T, width=256, epochs=20, batch=4096, lr=1e-3, seed=0):
    net = capi.Mlp(4, width, 2, seed=seed)
    loss = net.train(X, T, batch=batch, epochs=epochs, lr=lr, seed=seed)
    return net, loss


def report(n_train=64, n_test=4, grid=3, nb=48, nocc=24, Np=384, epochs=20, tol=1e-9, seed=0,
           mode=capi.FP64):
    """Config-5 style study: train on n_train seeded systems' plain-loop trajectories, then
    compare plain damping, damping + network and DIIS on n_test held-out systems run to
    |dE| < tol and residual < tol; for each run also the first iteration whose total energy is
    within 1e-6 Ha of the converged one.  Returns a dict of the measurements."""
    from .iaft import IAFT
    from .synthetic import make_system
    ft = IAFT(1000.0, 10.0, "low")
    t0 = time.perf_counter()
    trajs = [trajectory(make_system(grid, nb, nocc, Np, seed=1000 + i), ft) for i in range(n_train)]
    t_traj = time.perf_counter() - t0
    X, T = dataset(trajs, seed=seed)
    t0 = time.perf_counter()
    net, loss = train(X, T, epochs=epochs, seed=seed)
    t_train = time.perf_counter() - t0
    runs = []
    for i in range(n_test):
        s = make_system(grid, nb, nocc, Np, seed=5000 + i)
        c = make_context(s, ft, mode)
        G0 = s.G0(ft)
        row = {}
        for name, kw in (("damping", dict()), ("damping+mlp", dict(mlp=net)),
                         ("diis", dict(alg="diis", mixing=0.2))):
            r = run_loop(c, G0, tol_e=tol, tol_r=tol, **kw)
            e = [h["e_tot"] for h in r["history"]]
            evals = np.cumsum([h["evaluations"] for h in r["history"]])
            first = next(i for i in range(len(e)) if all(abs(x - e[-1]) < 1e-6 for x in e[i:]))
            row[name] = dict(iterations=r["iterations"], evaluations=r["evaluations"],
                             wall_s=r["wall_s"], e_tot=r["e_tot"], learned_steps=r["learned_steps"],
                             withdrawn=r["withdrawn"], iterations_to_1e6=first + 1,
                             evaluations_to_1e6=int(evals[first]),
                             residuals=[h["residual"] for h in r["history"]])
        runs.append(row)
        c.close()
    net.close()
    return dict(config=dict(grid=grid, nb=nb, nocc=nocc, Np=Np, n_train=n_train, n_test=n_test,
                            tol=tol, mixing=0.7, mode="fp64" if mode == capi.FP64 else "mixed"),
                trajectories_s=t_traj, train_s=t_train, samples=int(X.shape[0]),
                loss_first=float(loss[0]), loss_last=float(loss[-1]), runs=runs)


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="learned self-energy update study")
    ap.add_argument("--train", type=int, default=64)
    ap.add_argument("--test", type=int, default=4)
    ap.add_argument("--grid", type=int, default=3)
    ap.add_argument("--nb", type=int, default=48)
    ap.add_argument("--nocc", type=int, default=24)
    ap.add_argument("--Np", type=int, default=384)
    ap.add_argument("--epochs", type=int, default=20)
    a = ap.parse_args()
    print(json.dumps(report(a.train, a.test, a.grid, a.nb, a.nocc, a.Np, a.epochs), indent=1))
