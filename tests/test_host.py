"""Host-side logic that needs no GPU: synthetic inputs, argument validation."""
import os

import numpy as np
import pytest

from coqui_b200 import capi, solvers
from coqui_b200.iaft import IAFT
from coqui_b200.synthetic import WORKLOADS, kgrid, make_system


def test_synthetic_distributions():
    s = make_system(2, 16, 8, 64, seed=11)
    assert s.X.shape == (1, 8, 64, 16) and s.V.shape == (8, 64, 64)
    np.testing.assert_allclose(s.V, np.conj(np.swapaxes(s.V, -1, -2)), atol=1e-15)
    assert np.linalg.eigvalsh(s.V).min() > 1e-3 - 1e-12
    assert np.all(s.eps[0, :, :8] < -0.1 + 1e-15) and np.all(s.eps[0, :, 8:] > 0.1 - 1e-15)
    # seeded
    t = make_system(2, 16, 8, 64, seed=11)
    np.testing.assert_array_equal(s.X, t.X)


def test_kgrid_lexicographic():
    k = kgrid((2, 3, 1))
    assert k.shape == (6, 3)
    np.testing.assert_allclose(k[4] / (2 * np.pi), [1 / 2, 1 / 3, 0])


def test_g0_shape_and_sign():
    ft = IAFT(1000.0, 10.0, "low")
    s = make_system(1, 6, 3, 8, seed=2)
    G = s.G0(ft)
    assert G.shape == (ft.nt_f, 1, 1, 6, 6)
    assert np.all(G.real[:, 0, 0, np.arange(6), np.arange(6)] <= 0)
    # occupied: -G(beta^-) = 1; virtual: 0
    Dm = -np.einsum("t,tskij->skij", ft.T_beta_t_ff, G)
    np.testing.assert_allclose(np.diag(Dm[0, 0]).real, [1, 1, 1, 0, 0, 0], atol=1e-5)  # "low" IR: 1e-6


def test_workloads_named():
    assert WORKLOADS["g0w0_k4_nb64_np512"]["Np"] == 512


def test_solver_argument_checks():
    ft = IAFT(1000.0, 10.0, "low")
    with pytest.raises(ValueError):
        solvers.scr_coulomb_t(ft, screen_type="edmft")
    for div in ("ignore_g0", "gygi", "gygi_extrplt", "gygi_extrplt_2d"):
        assert solvers.gw_t(ft, div_treatment=div).div_treatment == div
    with pytest.raises(ValueError):
        solvers.gw_t(ft, div_treatment="ewald")
    with pytest.raises(capi.CoquiB200Error):
        solvers.gw_t(ft).evaluate(solvers.MBState(), None)


def test_shape_validation_before_device():
    with pytest.raises(ValueError):
        capi._c128(np.zeros((2, 3)), (3, 2), "x")
    with pytest.raises(ValueError):
        capi._ptr(np.zeros((4, 4))[:, ::2], "x")


def test_mlp_oracle_gradient_matches_finite_differences():
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(3)
    din, width, dout = 4, 16, 2
    n = width * din + width + width * width + width + dout * width + dout
    p = rng.standard_normal(n) * 0.3
    X, T = rng.standard_normal((7, din)), rng.standard_normal((7, dout))
    _, g = M.loss_and_grad(p, X, T, din, width, dout, round_params=False)
    for i in rng.choice(n, 12, replace=False):
        e = np.zeros(n)
        e[i] = 1e-6
        lp, _ = M.loss_and_grad(p + e, X, T, din, width, dout, round_params=False)
        lm, _ = M.loss_and_grad(p - e, X, T, din, width, dout, round_params=False)
        assert abs((lp - lm) / 2e-6 - g[i]) < 1e-7 * max(1.0, abs(g[i]))


def test_bf16_rounding_ties_to_even():
    from oracle import mlp_oracle as M
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.14159], np.float32)
    r = M.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-12


def test_oracle_commutator_diis_converges_faster_than_damping():
    from coqui_b200.synthetic import make_system
    from oracle import thc_oracle as O
    s = make_system(2, 8, 4, 32, seed=5)
    ft = O.IAFT(1000.0, 10.0, "low")
    H0, S, F = s.mean_field()
    G0 = s.G0(ft)
    runs = {}
    for alg, mix in (("damping", 0.7), ("diis", 0.2)):
        hist, _, _ = O.scgw_loop(G0, s.X, s.V, H0, S, F, 0.0, ft, s.kpts, s.lattv, s.kp_grid,
                                 30, 1e-9, alg=alg, mixing=mix, diis_start=3)
        runs[alg] = hist
    assert len(runs["diis"]) < len(runs["damping"])
    assert abs(runs["diis"][-1]["e_tot"] - runs["damping"][-1]["e_tot"]) < 1e-8


def test_learned_features_of_a_geometric_sequence():
    from coqui_b200 import learned
    rho = np.array([0.3, 0.5 * np.exp(0.2j)])
    s_inf = np.array([1.0 + 1j, -2.0])
    d = np.array([0.1, 0.05j])
    hist = np.array([s_inf - d * rho ** j / (1 - rho) for j in range(4)])
    X, d1, valid = learned.features(hist)
    assert valid.all()
    np.testing.assert_allclose(X[:, 0] + 1j * X[:, 1], rho, rtol=1e-6)  # q1 = d1 / d2
    np.testing.assert_allclose(X[:, 2] + 1j * X[:, 3], rho, rtol=1e-6)  # q2 = d2 / d3
    # the target of a geometric sequence is rho / (1 - rho) in units of the last step
    tgt = (s_inf - hist[3]) / d1
    np.testing.assert_allclose(tgt, rho / (1 - rho), rtol=1e-12)
    Xd, Td = learned.dataset([np.concatenate([hist, s_inf[None]])], max_samples=10)
    assert Xd.shape == (2, 4) and Td.shape == (2, 2)


def test_bench_clock_record_reports_reasons_and_median():
    """The bench's clock record (used to accept or reject a timed region): median SM clock,
    the highest maximum clock, and every throttle reason seen active in any sample; rows
    without a power reading or maximum clock still count."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    clk = bench.Clocks(0)
    clk.src, clk.fails = {"nvml"}, 0
    na, act = "Not Active", "Active"
    clk.rows = [["1905", "1965", "812.5", na, na, na, act],
                ["1890", "1965", "", na, na, na, na],
                ["1920", "", "799.0", na, act, na, na]]
    s = clk.summary()
    assert s["sm_mhz"] == 1905.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert s["samples"] == 3 and s["source"] == ["nvml"] and s["failed_queries"] == 0
    empty = bench.Clocks(0)
    assert empty.summary()["reasons"] == ["unsampled"]


def test_bench_cpu_sample_counts_and_scaling():
    """The CPU baseline's extrapolation: unit counts of one GW iteration of the reference
    algorithm, and per-unit samples that scale to positive per-iteration times."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from coqui_b200.iaft import IAFT
    from coqui_b200.synthetic import make_system

    s = make_system(2, 8, 4, 32, seed=3)
    ft = IAFT(1000.0, 10.0, "low")
    c = bench.reference_unit_counts(s, ft)
    assert c["proj_p2a"] == 4 * ft.nt_half * s.nk and c["proj_a2p"] == 2 * ft.nt_half * s.nk
    assert c["dft"] == 9 * ft.nt_half and c["dyson"] == s.nk * ft.nw_half
    total, parts = bench.cpu_sample(s, ft, reps=1)
    assert set(parts) == set(c) and all(v > 0 for v in parts.values())
    assert abs(total - sum(parts.values())) < 1e-9 * total


def test_bench_group_rates_count_projection_problems():
    """Kernel-group rates: the projections count flops per (tau, k) problem the library
    reports (a G(tau) projected again for the self-energy counts again); per-iteration and
    per-launch amounts are unchanged; groups without an amount get no rate."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from coqui_b200.iaft import IAFT
    from coqui_b200.synthetic import make_system

    s = make_system(2, 8, 4, 32, seed=3)
    ft = IAFT(1000.0, 10.0, "low")
    work = bench.algorithmic_work(None, s, ft)
    per_problem = bench.gemm_flops_c(s.Np, s.nb, s.nb) + bench.gemm_flops_c(s.Np, s.Np, s.nb)
    assert work["proj_p2a"][3] == per_problem
    steps, problems = 2, 3 * s.nk
    stats = {"proj_p2a": (4.0, 6), "pi_fused": (2.0, 4), "dyson_M_gemm": (1.0, 2),
             "other": (1.0, 2)}
    g = bench.group_rates(stats, steps, work, 6000.0, 1600.0, 30.0, 29.0,
                          units={"proj_p2a": problems * steps})
    assert g["proj_p2a"]["units_per_step"] == problems
    tflops = per_problem * problems / (2.0e-3) / 1e12
    assert abs(g["proj_p2a"]["achieved_TFLOPs"] - tflops) < 1e-9 * tflops
    # per launch group (bytes) and per iteration (flops)
    gbps = work["pi_fused"][1] * 2 / (1.0e-3) / 1e9
    assert abs(g["pi_fused"]["achieved_GBps"] - gbps) < 1e-9 * gbps
    mf = work["dyson_M_gemm"][2] / (0.5e-3) / 1e12
    assert abs(g["dyson_M_gemm"]["achieved_TFLOPs"] - mf) < 1e-9 * mf
    # the M products count the part of P1 on and above the diagonal: Np^3 / 3 + Np^3 / 6
    P = s.nk * ft.nw_half
    assert abs(work["dyson_M_gemm"][2] - 0.5 * 8 * float(s.Np) ** 3 * P) < 1e-6 * work["dyson_M_gemm"][2]
    assert "achieved_TFLOPs" not in g["other"] and "achieved_GBps" not in g["other"]
    # without reported units the projection group has no rate rather than a guessed one
    g0 = bench.group_rates(stats, steps, work, 6000.0, 1600.0, 30.0)
    assert "achieved_TFLOPs" not in g0["proj_p2a"]


def test_truncated_ir_table_is_an_error(tmp_path, monkeypatch):
    """A damaged IR table is refused when it is loaded, before any device work."""
    import shutil
    from coqui_b200 import iaft
    src = os.path.join(iaft.IR_DIR, "1e4.1e-06.npz")
    data = open(src, "rb").read()
    d = tmp_path / "ir"
    d.mkdir()
    (d / "1e4.1e-06.npz").write_bytes(data[: len(data) // 2])
    monkeypatch.setattr(iaft, "IR_DIR", str(d))
    with pytest.raises(Exception):
        iaft.IAFT(1000.0, 10.0, "low")
    shutil.rmtree(d)


def test_hartree_fock_refuses_symmetry_reduced_data_before_any_device_work():
    """THC Hartree-Fock runs on the whole k-mesh: THCData carrying bz maps is refused with
    EUNSUPPORTED by the solver mirror before a context is created."""
    import numpy as np
    import pytest
    from coqui_b200 import capi, solvers
    from coqui_b200.symmetry import SWAP, bz_symmetry
    sym = bz_symmetry((2, 2, 1), [np.eye(3, dtype=int), SWAP], False)
    thc = solvers.THCData(X=np.zeros((1, 4, 4, 2), complex), V=np.zeros((4, 4, 4), complex),
                          kpts=np.zeros((4, 3)), lattv=np.eye(3), kp_grid=(2, 2, 1), bz=sym)
    F = np.zeros((1, 4, 2, 2), complex)
    with pytest.raises(capi.CoquiB200Error) as e:
        solvers.hf_t().evaluate(F, F, thc, F)
    assert e.value.code == -2
