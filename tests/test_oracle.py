"""CPU tests of the FP64 oracle: the identities that pin the restatement of
the reference math (no reference test vectors exist), and the committed
golden fixtures."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import rpa_oracle as O

GOLDEN = json.loads((Path(__file__).parent / "golden" / "oracle_golden.json").read_text())


def small_system(seed=3, nq=60, no=4, nv=20, lam0=0.7):
    s = O.make_system(nq, no, nv, seed, decay=20.0, lam0=lam0)
    x, w = O.grid_for(s, 10)
    return s, x, w


def test_gauss_legendre_matches_numpy():
    for n in (2, 7, 8, 16, 33, 64):
        x, w = O.gauss_legendre(n)
        xr, wr = np.polynomial.legendre.leggauss(n)
        assert np.max(np.abs(x - xr)) < 1e-14
        assert np.max(np.abs(w - wr)) < 1e-13


def test_casimir_polder_integrates_lorentzian():
    # identity (iv): sum_k w_k/(d^2+u_k^2) -> pi/(2d) with the optimised scale
    e = np.concatenate([np.linspace(-1.2, -0.3, 12), np.exp(np.linspace(np.log(0.02), np.log(5.0), 120))])
    vals, wts = O.dai_histogram(e, 12, 120)
    x, w = O.optimize_freq_quad(vals, wts)
    rel, rmsd = O.freq_quad_error(x, w, vals, wts)
    assert rmsd < O.TARGET_ERROR_FREQ and rel < O.TARGET_REL_ERROR_FREQ
    assert O.RPA_MIN_NFREQS <= len(x) <= O.RPA_MAX_NFREQS
    assert np.all(np.diff(x) > 0) and np.all(w > 0)


def test_histogram_edges_and_gap_error():
    e = np.array([-1.0, -0.5, 0.1, 0.2, 3.0])
    vals, wts = O.dai_histogram(e, 2, 3, nbins=10)
    assert math.isclose(wts.sum(), 1.0)
    assert vals[0] == pytest.approx(0.6) and wts[0] > 0 and wts[-1] > 0
    with pytest.raises(ValueError):
        O.dai_histogram(np.array([-1.0, 0.5, 0.4]), 2, 1)


def test_ncore_frozen():
    e = np.array([-20.0, -19.5, -1.0, -0.5, 0.2])
    assert O.ncore(e, 4) == 2
    assert O.ncore(e, 4, core_thresh=-30.0) == 0


def test_logdet_qr_cholesky_eigen_agree():
    # identity (iii)
    s, x, w = small_system()
    pi = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
    for p in pi[:3]:
        A = np.eye(s.nq) + p
        lq = O.logdet_qr(A)
        lc = O.logdet_cholesky(A)
        le = math.fsum(np.log1p(np.linalg.eigvalsh(p)).tolist())
        assert abs(lq - lc) < 1e-12 * max(1.0, abs(lq))
        assert abs(lq - le) < 1e-11 * max(1.0, abs(lq))


def test_pi_block_algorithm_equals_dense():
    s, x, w = small_system()
    pi = O.pi_matrices(s.R, s.eps_o, s.eps_v, x, block_dim=7)
    d = O.dai(s.eps_o, s.eps_v)
    for k in (0, len(x) - 1):
        ref = 4.0 * (s.R * O.chi_factor(d, x[k])[None, :]) @ s.R.T
        assert np.max(np.abs(pi[k] - ref)) < 1e-13 * np.max(np.abs(ref))


def test_mp2_limit():
    # identity (ii): E_c(eps R)/eps^4 -> direct MP2 as eps -> 0 (up to quadrature error)
    s, x, w = small_system(lam0=None)
    emp2 = O.direct_mp2(s.R, s.eps_o, s.eps_v)
    eps = 1e-3
    ec, _ = O.ec_rpa(eps * s.R, s.eps_o, s.eps_v, x, w)
    assert abs(ec / eps ** 4 - emp2) < 2e-3 * abs(emp2)


def test_t2_eigenvalue_energy_matches_logdet_energy():
    # identity (i): sum_mu 2 A_mu |R U_mu|^2 == E_c from ln det (RPA == drCCD)
    s, x, w = small_system(seed=5, nq=40, no=3, nv=12, lam0=0.6)
    pi = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
    ec, _ = O.ec_rpa_analytic(pi, w)
    vals, vecs = O.diagonalize_pi(pi)
    rng = np.random.default_rng(0)
    G = min(int(math.ceil(3.0 * s.nq)), s.no * s.nv)
    omega = rng.uniform(size=(s.no * s.nv, G)) - 0.5
    A, U, K = O.t2_direct_ring(s.R, s.eps_o, s.eps_v, x, w, vals, vecs, omega, cutoff_thresh=1e-12)
    eig = O.t2_eig_rpa(U, A, s.R)
    assert abs(eig.sum() - ec) < 1e-6 * abs(ec)
    # T2 eigenvectors are orthonormal, eigenvalues in (-1/2, 0]
    assert np.allclose(U.T @ U, np.eye(U.shape[1]), atol=1e-8)
    assert np.all(A < 0) and np.all(A > -0.5)


def test_sosex_pair_loop_equals_dense_contraction():
    s, x, w = small_system(seed=6, nq=30, no=3, nv=8, lam0=0.6)
    nt = 11
    rng = np.random.default_rng(1)
    V = rng.standard_normal((nt, s.no * s.nv))
    A = -0.1 * rng.uniform(size=nt)
    ex = O.exchange_sosex(V, A, s.R, s.no, s.nv)
    # dense: -sum_{abij} (aj|bi) T_aibj, T = V^T diag(A) V
    T = (V.T * A[None, :]) @ V
    Rr = s.R.reshape(s.nq, s.nv, s.no, order="F")
    Tr = T.reshape(s.nv, s.no, s.nv, s.no, order="F")  # T[a,i,b,j]
    Kx = np.einsum("qaj,qbi->aibj", Rr, Rr)            # (aj|bi) indexed [a,i,b,j]
    assert ex == pytest.approx(-np.sum(Kx * Tr), rel=1e-12)


def test_mbe_size_consistency_block_diagonal():
    # identity (v): non-interacting fragments -> interaction energy vanishes
    a = O.make_system(30, 3, 8, 11, decay=10.0, lam0=0.5)
    b = O.make_system(25, 2, 9, 12, decay=10.0, lam0=0.5)
    eo = np.concatenate([a.eps_o, b.eps_o])
    ev = np.concatenate([a.eps_v, b.eps_v])
    no, nv = len(eo), len(ev)
    R = np.zeros((a.nq + b.nq, no * nv))
    for (sysx, q0, i0, a0) in ((a, 0, 0, 0), (b, a.nq, a.no, a.nv)):
        Rr = sysx.R.reshape(sysx.nq, sysx.nv, sysx.no, order="F")
        for i in range(sysx.no):
            for aa in range(sysx.nv):
                R[q0:q0 + sysx.nq, (a0 + aa) + nv * (i0 + i)] = Rr[:, aa, i]
    x, w = O.casimir_polder(16, 0.7)
    eab, _ = O.ec_rpa(R, eo, ev, x, w)
    ea, _ = O.ec_rpa(a.R, a.eps_o, a.eps_v, x, w)
    eb, _ = O.ec_rpa(b.R, b.eps_o, b.eps_v, x, w)
    assert abs(O.eint_2body(eab, ea, eb)) < 1e-13


def test_gradient_against_finite_differences():
    s, x, w = small_system(seed=8, nq=24, no=3, nv=7, lam0=0.6)
    dR, deo, dev = O.ec_grad(s.R, s.eps_o, s.eps_v, x, w)
    h = 1e-5
    rng = np.random.default_rng(2)
    for _ in range(8):
        q, ai = rng.integers(s.nq), rng.integers(s.no * s.nv)
        Rp, Rm = s.R.copy(), s.R.copy()
        Rp[q, ai] += h
        Rm[q, ai] -= h
        fd = (O.ec_rpa(Rp, s.eps_o, s.eps_v, x, w)[0] - O.ec_rpa(Rm, s.eps_o, s.eps_v, x, w)[0]) / (2 * h)
        assert fd == pytest.approx(dR[q, ai], rel=1e-6, abs=1e-11)
    for i in range(s.no):
        ep, em = s.eps_o.copy(), s.eps_o.copy()
        ep[i] += h
        em[i] -= h
        fd = (O.ec_rpa(s.R, ep, s.eps_v, x, w)[0] - O.ec_rpa(s.R, em, s.eps_v, x, w)[0]) / (2 * h)
        assert fd == pytest.approx(deo[i], rel=1e-6, abs=1e-11)


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_golden_fixtures(name):
    from tests.golden.make_golden import system
    g = GOLDEN[name]
    s, x, w = system(name)
    assert s.R.sum() == pytest.approx(g["R_sum"], rel=1e-12, abs=1e-12)
    assert np.allclose(x, g["freqs"], rtol=1e-13) and np.allclose(w, g["weights"], rtol=1e-13)
    if "R" in g:
        assert np.array_equal(s.R, np.array(g["R"]))
    pi = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
    ec, eu = O.ec_rpa_analytic(pi, w)
    assert ec == pytest.approx(g["Ec"], abs=1e-12)
    assert np.allclose(eu, g["Eu"], rtol=1e-11, atol=1e-13)


def test_mbpt3_lyapunov_solution_and_pair_sum():
    s, x, w = small_system(seed=9, nq=40, no=3, nv=12, lam0=0.6)
    pi = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
    vals, vecs = O.diagonalize_pi(pi)
    omega = np.random.default_rng(3).uniform(size=(s.no * s.nv, s.no * s.nv)) - 0.5
    A, U, K = O.t2_direct_ring(s.R, s.eps_o, s.eps_v, x, w, vals, vecs, omega, cutoff_thresh=1e-4)
    ex, X = O.exchange_mbpt3_1(U, A, s.R, s.eps_o, s.eps_v)
    d = O.dai(s.eps_o, s.eps_v)
    RU = s.R @ U
    Ukl, Dkl = RU.T @ RU, U.T @ (d[:, None] * U)
    Bm = Dkl + 2 * Ukl + 4 * Ukl * A[None, :]
    Am = A[:, None] * Dkl + Dkl * A[None, :]
    assert np.allclose(Bm.T @ X + X @ Bm, Am, atol=1e-12 * np.abs(Am).max())
    assert np.allclose(X, X.T, atol=1e-10 * np.abs(X).max())
    # dense form: -sum_{abij} (aj|bi) (dT)_aibj with dT = U X U^T
    dT = U @ X @ U.T
    Rr = s.R.reshape(s.nq, s.nv, s.no, order="F")
    Kx = np.einsum("qaj,qbi->aibj", Rr, Rr)
    assert ex == pytest.approx(-np.sum(Kx * dT.reshape(s.nv, s.no, s.nv, s.no, order="F")), rel=1e-10)


def test_piu_basis_eigen_trace_error_and_energy():
    s, x, w = small_system(seed=12, nq=60, no=4, nv=20)
    pi1 = O.pi_matrices(s.R, s.eps_o, s.eps_v, x[:1])[0]
    G, nv_, err, exact = O.piu_basis(pi1, 1e-3)
    lam = np.linalg.eigvalsh(pi1)[::-1]
    assert exact == pytest.approx(np.trace(pi1), rel=1e-14)
    assert 1 <= nv_ <= s.nq
    # the dropped tail (indices nvecs-1 .. N-1, the reference's accounting) is below the target
    assert err == pytest.approx(lam[nv_ - 1:].sum(), rel=1e-10, abs=1e-16) and err < 1e-3
    if nv_ > 1:
        assert lam[nv_ - 2:].sum() >= 1e-3
    # projected R' = G^T R reproduces E_c up to the dropped part of the spectrum
    Rp = G[:, :nv_].T @ s.R
    e_full, _ = O.ec_rpa(s.R, s.eps_o, s.eps_v, x, w)
    e_proj, _ = O.ec_rpa(Rp, s.eps_o, s.eps_v, x, w)
    assert abs(e_proj - e_full) < 1e-2 * abs(e_full)
    # full basis: identity, no truncation; random basis spans the dominant subspace
    Gf, nf, ef, _ = O.piu_basis(pi1, 1e-3, O.RPA_BASIS_FULL_CHOLESKY)
    assert nf == s.nq and ef == 0.0 and np.array_equal(Gf, np.eye(s.nq))
    g0 = np.random.default_rng(0).standard_normal((s.nq, s.nq))
    Gr, nr, er, _ = O.piu_basis(pi1, 1e-3, O.RPA_BASIS_RANDOM, guess=g0)
    assert np.allclose(Gr.T @ Gr, np.eye(s.nq), atol=1e-10) and er < 1e-3


def test_thc_r_matches_explicit_sum():
    Z, Xa, Xi, eo, ev = O.make_thc_factors(40, 12, 3, 5, 7)
    R = O.thc_r(Z, Xa, Xi)
    for (k, a, i) in ((0, 0, 0), (5, 4, 2), (11, 2, 1)):
        ref = math.fsum(Z[g, k] * Xa[g, a] * Xi[g, i] for g in range(40))
        assert R[k, a + 5 * i] == pytest.approx(ref, rel=1e-12, abs=1e-15)


def test_jctc2024_pno_rpa_energy_and_sosex_limit():
    # with every PNO kept (cutoff 0) the PNO direct-ring term equals the T2 eigenvalue energy
    # sum_mu 2 A_mu |R U_mu|^2 = 2 sum (ai|bj) T_aibj, and Ec1b equals -2x the exchange sum
    Z, Xa, Xi, eo, ev = O.make_thc_factors(60, 20, 3, 7, 21)
    R = O.thc_r(Z, Xa, Xi)
    rng = np.random.default_rng(2)
    nt = 9
    U, _ = np.linalg.qr(rng.standard_normal((R.shape[1], nt)))
    A = -0.1 * rng.uniform(size=nt)
    ec_rpa, ec1b, e2bcd, e2ghij = O.jctc2024_corrections(Z, Xi, Xa, U, A, cutoff_pno=0.0)
    eig = O.t2_eig_rpa(U, A, R)
    assert ec_rpa == pytest.approx(eig.sum(), rel=1e-10)
    ex = O.exchange_sosex(np.ascontiguousarray(U.T), A, R, 3, 7, alpha=1.0)
    assert 0.5 * ec1b == pytest.approx(ex, rel=1e-10)
    # localisation by an orthogonal Lik leaves every term unchanged
    L, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    loc = O.jctc2024_corrections(Z, Xi, Xa, U, A, Lik=L, cutoff_pno=0.0)
    assert np.allclose(loc, (ec_rpa, ec1b, e2bcd, e2ghij), rtol=1e-9, atol=1e-14)
