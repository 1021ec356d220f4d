"""Internal identities of the FP64 oracle (Pi, W, Sigma, E_c have no reference golden
vectors on synthetic THC inputs; these checks pin the restatement's conventions)."""
import numpy as np
import pytest

from coqui_b200.synthetic import make_system
from oracle import thc_oracle as O


@pytest.fixture(scope="module")
def small(ft_low):
    s = make_system(2, 8, 4, 24, seed=3)
    return s, s.G0(ft_low)


def test_dense_dft_equals_fft(small):
    s, _ = small
    f_Rk = O.k_to_R_coefficients(s.kpts, s.lattv, s.kp_grid)
    x = np.random.default_rng(0).standard_normal((s.nk, 5)) + 0j
    ref = (np.fft.fftn(x.reshape(2, 2, 2, 5), axes=(0, 1, 2)) / s.nk).reshape(s.nk, 5)
    np.testing.assert_allclose(f_Rk @ x, ref, atol=1e-14)
    f_kR = O.R_to_k_coefficients(s.kpts, s.lattv, s.kp_grid)
    np.testing.assert_allclose(f_kR @ f_Rk, np.eye(s.nk), atol=1e-14)


def test_dft_non_cubic_grid():
    s = make_system((1, 2, 3), 4, 2, 8, seed=1)
    f_Rk = O.k_to_R_coefficients(s.kpts, s.lattv, s.kp_grid)
    x = np.random.default_rng(1).standard_normal((6, 3)) + 0j
    ref = (np.fft.fftn(x.reshape(1, 2, 3, 3), axes=(0, 1, 2)) / 6).reshape(6, 3)
    np.testing.assert_allclose(f_Rk @ x, ref, atol=1e-14)


def test_pi_hermitian_negative(small, ft_low):
    s, G = small
    Pi = O.eval_Pi_rpa_Rspace(G, s.X, s.kpts, s.lattv, s.kp_grid)
    assert Pi.shape == (ft_low.nt_half, s.nk, 24, 24)
    np.testing.assert_allclose(Pi, np.conj(np.swapaxes(Pi, -1, -2)), atol=1e-15)
    Pw = ft_low.tau_to_w_PHsym(Pi)
    assert np.linalg.eigvalsh(Pw).max() < 1e-12  # Pi(iW) is negative semidefinite


def test_dyson_lu_equals_cholesky_form(small, ft_low):
    s, G = small
    Pw = ft_low.tau_to_w_PHsym(O.eval_Pi_rpa_Rspace(G, s.X, s.kpts, s.lattv, s.kp_grid))
    W1 = O.dyson_W_in_place(Pw, s.V)
    W2 = O.dyson_W_cholesky(Pw, s.V)
    np.testing.assert_allclose(W1, W2, atol=1e-13)


def test_rpa_logdet_equals_cholesky(small, ft_low):
    s, G = small
    Pw = ft_low.tau_to_w_PHsym(O.eval_Pi_rpa_Rspace(G, s.X, s.kpts, s.lattv, s.kp_grid))
    A = Pw[3, 1] @ s.V[1]
    L = np.linalg.cholesky(s.V[1])
    C = np.linalg.cholesky(np.eye(24) - L.conj().T @ Pw[3, 1] @ L)
    np.testing.assert_allclose(np.log(np.linalg.det(np.eye(24) - A).real),
                               2 * np.log(np.diag(C).real).sum(), atol=1e-12)


def test_gamma_only_path_skips_dft(ft_low):
    s = make_system(1, 6, 3, 16, seed=5)
    G = s.G0(ft_low)
    Pi = O.eval_Pi_rpa_Rspace(G, s.X, s.kpts, s.lattv, s.kp_grid)
    it = 2
    Gp = O.primary_to_aux(G[it], s.X)
    Gn = O.primary_to_aux(G[ft_low.nt_f - 1 - it], s.X)
    np.testing.assert_allclose(Pi[it, 0], -2 * (Gp * np.conj(Gn))[0, 0], atol=1e-15)


def test_sigma_hermitian_and_mirror(small, ft_low):
    s, G = small
    dW, head, _ = O.update_w(G, s.X, s.V, ft_low, s.kpts, s.lattv, s.kp_grid, s.chi_bar)
    S = O.eval_Sigma_all_Rspace(G, dW, s.X, s.kpts, s.lattv, s.kp_grid)
    np.testing.assert_allclose(S, np.conj(np.swapaxes(S, -1, -2)), atol=1e-14)
    assert head.shape == (ft_low.nt_half,)
    e = O.eval_corr_energy(G, S, ft_low, np.ones(s.nk) / s.nk)
    assert e < 0


def test_damp_and_hermitize():
    a = np.array([[1 + 1j, 2], [0, 3]])
    b = np.zeros_like(a)
    h, diff = O.damp(a, b, 0.7)
    np.testing.assert_allclose(h, 0.7 * a)
    assert diff == pytest.approx(np.abs(0.7 * a).max())
    hh = O.hermitize(a)
    np.testing.assert_allclose(hh, hh.conj().T)


def _random_dm(rng, nk, nb):
    A = rng.standard_normal((1, nk, nb, nb)) + 1j * rng.standard_normal((1, nk, nb, nb))
    return 0.25 * (A + np.conj(np.swapaxes(A, -1, -2)))


def test_hf_equals_k_convolution():
    """thc_hf's R-space exchange equals K(k) = -(1/nk) sum_q D(k-q) o V(q) and its Hartree
    term J_P = sum_Q V(0)_PQ (2/nk) sum_k D_QQ(k) (no DFT involved)."""
    s = make_system((2, 1, 3), 5, 2, 12, seed=7)
    n0, n1, n2 = s.kp_grid
    nk, Np = s.nk, s.Np
    Dm = _random_dm(np.random.default_rng(2), nk, s.nb)
    F = O.thc_hf(Dm, s.X, s.V, s.kpts, s.lattv, s.kp_grid)
    D = O.primary_to_aux(Dm, s.X)[0]
    ijl = [(i, j, l) for i in range(n0) for j in range(n1) for l in range(n2)]
    minus = lambda a, b: (((a[0] - b[0]) % n0) * n1 + (a[1] - b[1]) % n1) * n2 + (a[2] - b[2]) % n2
    rho = 2.0 / nk * np.einsum("kpp->p", D)
    J = s.V[0] @ rho
    Fp = np.zeros((nk, Np, Np), np.complex128)
    for k in range(nk):
        for q in range(nk):
            Fp[k] -= D[minus(ijl[k], ijl[q])] * s.V[q] / nk
        Fp[k] += np.diag(J)
    ref = O.aux_to_primary(Fp[None], s.X)
    np.testing.assert_allclose(F, ref, atol=1e-12)


def test_hf_gamma_equals_four_index_contraction():
    """At one k-point J_ab = 2 sum_cd (ab|dc) D_cd and K_ab = -sum_cd (ac|db) D_cd with the
    THC integrals (ab|cd) = sum_PQ conj(X_Pa) X_Pb V_PQ conj(X_Qc) X_Qd."""
    s = make_system(1, 6, 3, 10, seed=4)
    Dm = _random_dm(np.random.default_rng(3), 1, s.nb)
    X, V = s.X[0, 0], s.V[0]
    eri = np.einsum("Pa,Pb,PQ,Qc,Qd->abcd", np.conj(X), X, V, np.conj(X), X)
    J = 2.0 * np.einsum("abdc,cd->ab", eri, Dm[0, 0])
    K = -np.einsum("acdb,cd->ab", eri, Dm[0, 0])
    args = (s.X, s.V, s.kpts, s.lattv, s.kp_grid)
    np.testing.assert_allclose(O.thc_hf(Dm, *args, hartree=True, exchange=False)[0, 0], J,
                               atol=1e-12)
    np.testing.assert_allclose(O.thc_hf(Dm, *args, hartree=False, exchange=True)[0, 0], K,
                               atol=1e-12)


def test_hf_gygi_correction(small):
    """HF_K_correction (hf_t.cpp:72-80): gygi adds -madelung S Dm S to the exchange only."""
    s, _ = small
    rng = np.random.default_rng(5)
    Dm = _random_dm(rng, s.nk, s.nb)
    S = np.eye(s.nb)[None, None] + 0.1 * _random_dm(rng, s.nk, s.nb)
    args = (s.X, s.V, s.kpts, s.lattv, s.kp_grid, S)
    F0 = O.thc_hf(Dm, *args)
    F1 = O.thc_hf(Dm, *args, div="gygi", madelung=0.37)
    np.testing.assert_allclose(F1 - F0, -0.37 * S @ Dm @ S, atol=1e-13)
    J1 = O.thc_hf(Dm, *args, exchange=False, div="gygi", madelung=0.37)
    np.testing.assert_allclose(J1, O.thc_hf(Dm, *args, exchange=False), atol=0)


def test_smallest_nonzero_q_selects_the_head(small, ft_low):
    """find_smallest_qabs (g0_div_utils.hpp:263-282) skips q = 0, whose head prefactor
    |q|^2 Omega / 4 pi vanishes: on a grid of more than one q-point the head is taken at the
    first smallest nonzero |q| and is not zero."""
    from coqui_b200.synthetic import kgrid
    assert O.find_smallest_qabs(kgrid(2)) == 1  # (0, 0, pi) comes before (0, pi, 0)
    assert O.find_smallest_qabs(kgrid((1, 2, 3))) == 1
    assert O.find_smallest_qabs(kgrid((3, 1, 1))) == 1
    assert O.find_smallest_qabs(kgrid(1)) == 0
    q = np.array([[0, 0, 0], [0.5, 0, 0], [0, 0.3, 0], [0, 0, 0.3]])
    assert O.find_smallest_qabs(q) == 2
    s, G = small
    _, head, eps_tq = O.update_w(G, s.X, s.V, ft_low, s.kpts, s.lattv, s.kp_grid, s.chi_bar)
    np.testing.assert_array_equal(head, eps_tq[:, 1])
    assert np.abs(eps_tq[:, 0]).max() == 0.0 and np.abs(head).max() > 0.0


def _scaled_grid(n, L):
    """Gamma-centred grid of an L x L x L cubic cell (lattv = L I)."""
    from coqui_b200.synthetic import kgrid
    return kgrid(n) / L, np.eye(3) * L


def test_filter_and_extrapolation(ft_low):
    """filter_qpts / extrapolate_to_q0 / eps_inv_head_t (g0_div_utils.hpp:26-111): distinct
    |q| within q_max in q order; a quadratic in |q| is extrapolated exactly; the extrapolated
    head of a q-independent eps is its tau -> w -> tau round trip."""
    Q, _ = _scaled_grid(4, 10.0)
    idx = O.filter_qpts(Q, 0.8, 1)
    norms = np.sqrt((Q[idx] ** 2).sum(axis=1))
    # distinct as doubles (the reference's std::set<double>): |q| of permuted components can
    # differ in the last bit and then both are kept
    assert idx[0] == 1 and len(set(norms.tolist())) == len(idx)
    assert (norms > 0).all() and (norms <= 0.8).all()
    assert all(np.isclose(np.sqrt((Q[i] ** 2).sum()), norms).any() for i in range(1, len(Q))
               if 0 < np.sqrt((Q[i] ** 2).sum()) <= 0.8)
    idx2d = O.filter_qpts(Q, 0.8, 1, two_dim=True)
    assert all(Q[i][2] == 0.0 for i in idx2d)
    q = np.array([0.1, 0.2, 0.35, 0.5])
    assert abs(O.extrapolate_to_q0(q, 0.3 - 2j + (1 + 1j) * q - 0.7 * q ** 2) - (0.3 - 2j)) < 1e-12
    nth = ft_low.nt_half
    a = np.linspace(-0.5, -0.1, nth) + 0j
    eps = np.repeat(a[:, None], len(Q), axis=1)
    eps[:, 0] = 0.0  # q = 0: vanishing prefactor
    head = O.eps_inv_head_t(eps, Q, ft_low, "gygi_extrplt")
    np.testing.assert_allclose(head, ft_low.w_to_tau_PHsym(ft_low.tau_to_w_PHsym(a)), atol=1e-12)
    np.testing.assert_array_equal(O.eps_inv_head_t(eps, Q, ft_low, "gygi"), eps[:, 1])
    # one q-point: ignore_g0 whatever the treatment
    np.testing.assert_array_equal(O.eps_inv_head_t(eps[:, :1], Q[:1], ft_low, "gygi_extrplt"),
                                  eps[:, 0])
    with pytest.raises(ValueError):
        O.eps_inv_head_t(eps, Q * 100, ft_low, "gygi_extrplt")  # no q within q_max


def test_sigma_div_correction_form(small):
    """Sigma_div_correction: T = X^H diag(conj chi_head) X per k, Delta(t) = f(t_pos) T G T^H,
    nothing for ignore_g0 or one q-point."""
    s, G = small
    rng = np.random.default_rng(9)
    chi = (rng.standard_normal(s.Np) + 1j * rng.standard_normal(s.Np)) / np.sqrt(s.Np)
    nth = (G.shape[0] + 1) // 2
    head = rng.standard_normal(nth) + 0.1j
    S0 = np.zeros_like(G)
    D = O.sigma_div_correction(S0, G, s.X, chi, head, 0.6, "gygi")
    X = s.X[0, 1]
    T = np.conj(X).T @ np.diag(np.conj(chi)) @ X
    t = G.shape[0] - 2  # mirrored half: t_pos = 1
    np.testing.assert_allclose(D[t, 0, 1], -0.6 * head[1].real * T @ G[t, 0, 1] @ np.conj(T).T,
                               atol=1e-14)
    assert O.sigma_div_correction(S0, G, s.X, chi, head, 0.6, "ignore_g0") is S0
    assert O.sigma_div_correction(S0, G, s.X, chi, head, 0.6, "gygi", nq=1) is S0
