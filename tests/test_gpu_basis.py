"""GPU tests of the compressed Pi basis (rpa_b200_piu_basis, replacing rpa_G) and the
projection R' = G^T R (rpa_b200_project_basis) against the oracle.

Tolerances: NVecs equal; trace error and Tr Pi to 1e-10 relative; the kept subspace equal to
the oracle's (projector difference 1e-8; random basis: columns equal up to sign to 1e-8);
energies in the compressed basis to 1e-10 Eh (FP64).
"""
import numpy as np
import pytest

from oracle import rpa_oracle as O

pytestmark = pytest.mark.gpu


def _case(seed=31, nq=300, no=6, nv=50):
    s = O.make_system(nq, no, nv, seed, decay=nq / 6.0, lam0=0.8)
    x, w = O.grid_for(s, 10)
    return s, x, w


@pytest.mark.parametrize("target", [1e-6, 1e-4, O.TARGET_ERROR_RANDOM])
def test_eigen_basis_matches_oracle(handle, target):
    s, x, w = _case()
    pi1 = O.pi_matrices(s.R, s.eps_o, s.eps_v, x[:1])[0]
    Gr, nr, er, exr = O.piu_basis(pi1, target)
    G, terr, tex = handle.piu_basis(s.R, s.eps_o, s.eps_v, x[0], target_error=target, basis="eigen")
    assert G.shape[1] == nr
    assert terr == pytest.approx(er, rel=1e-10, abs=1e-14)
    assert tex == pytest.approx(exr, rel=1e-12)
    P, Pr = G @ G.T, Gr[:, :nr] @ Gr[:, :nr].T
    assert np.max(np.abs(P - Pr)) < 1e-8
    # energies with the compressed Cholesky vectors
    Rp = handle.project_basis(G, s.R)
    assert np.allclose(Rp, G.T @ s.R, rtol=0, atol=1e-12 * np.abs(s.R).max())
    ec, _ = handle.ec_rpa(Rp, s.eps_o, s.eps_v, x, w, prec="fp64")
    ref, _ = O.ec_rpa(Gr[:, :nr].T @ s.R, s.eps_o, s.eps_v, x, w)
    assert abs(ec - ref) < 1e-10
    full, _ = O.ec_rpa(s.R, s.eps_o, s.eps_v, x, w)
    assert abs(ec - full) < 1e-2 * abs(full)


def test_full_and_random_bases(handle):
    s, x, w = _case(seed=32, nq=200, no=5, nv=40)
    G, terr, _ = handle.piu_basis(s.R, s.eps_o, s.eps_v, x[0], basis="full")
    assert G.shape == (s.nq, s.nq) and terr == 0.0 and np.array_equal(G, np.eye(s.nq))
    # well-conditioned Pi: the Gram-Schmidt columns equal Householder QR's up to sign
    s = O.make_system(150, 5, 60, 33, decay=1e5, lam0=0.8)
    pi1 = O.pi_matrices(s.R, s.eps_o, s.eps_v, x[:1])[0]
    g0 = np.random.default_rng(4).standard_normal((s.nq, s.nq))
    Gr, nr, er, _ = O.piu_basis(pi1, 1e-4, O.RPA_BASIS_RANDOM, guess=g0)
    G, terr, _ = handle.piu_basis(s.R, s.eps_o, s.eps_v, x[0], target_error=1e-4, basis="random", guess=g0)
    assert G.shape[1] == nr
    assert terr == pytest.approx(er, rel=1e-8, abs=1e-14)
    d = np.abs(np.sum(G * Gr[:, :nr], axis=0))
    assert np.min(d) > 1 - 1e-8


def test_random_basis_of_a_numerically_low_rank_pi_is_reported(handle, pkg):
    # fast-decaying Cholesky vectors: Pi G is numerically rank deficient; the CholeskyQR
    # subspace iteration reports it (the eigenvector basis, the default, handles such Pi)
    s, x, w = _case(seed=34, nq=200, no=5, nv=40)
    g0 = np.random.default_rng(5).standard_normal((s.nq, s.nq))
    with pytest.raises(pkg.RPAError) as e:
        handle.piu_basis(s.R, s.eps_o, s.eps_v, x[0], target_error=1e-4, basis="random", guess=g0)
    assert e.value.status == pkg.RPA_ERR_NOT_SPD
    G, terr, _ = handle.piu_basis(s.R, s.eps_o, s.eps_v, x[0], target_error=1e-4, basis="eigen")
    assert terr < 1e-4 and np.allclose(G.T @ G, np.eye(G.shape[1]), atol=1e-10)
