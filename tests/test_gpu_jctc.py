"""GPU tests of the particle-hole corrections with pair-natural orbitals (rpa_b200_jctc2024,
replacing rpa_JCTC2024_Corrections) against the oracle restatement.

Tolerances: every energy term to 1e-9 relative (FP64 tensor-core GEMMs; the PNO singular
vectors come from the eigenvectors of T T^T, the terms depend only on each pair's U s V^T).
"""
import numpy as np
import pytest

from oracle import rpa_oracle as O

pytestmark = pytest.mark.gpu


def _case(seed, ng, nq, no, nv, nt):
    Z, Xa, Xi, eo, ev = O.make_thc_factors(ng, nq, no, nv, seed)
    rng = np.random.default_rng(seed + 100)
    U, _ = np.linalg.qr(rng.standard_normal((no * nv, nt)))
    A = -0.2 * rng.uniform(size=nt)
    return Z, Xa, Xi, U, A


@pytest.mark.parametrize("shape", [(120, 30, 4, 16, 24), (200, 45, 6, 21, 50)])
@pytest.mark.parametrize("cutoff", [1e-8, 1e-3])
def test_jctc2024_matches_oracle(handle, shape, cutoff):
    Z, Xa, Xi, U, A = _case(41, *shape)
    ref = O.jctc2024_corrections(Z, Xi, Xa, U, A, cutoff_pno=cutoff)
    got, stats = handle.jctc2024(Z, Xi, Xa, U, A, cutoff_pno=cutoff)
    for g, r in zip(got, ref):
        assert g == pytest.approx(r, rel=1e-9, abs=1e-14)
    assert stats[0] <= shape[3] and stats[1] > 0


def test_jctc2024_localised_and_screened(handle):
    Z, Xa, Xi, U, A = _case(42, 150, 40, 5, 18, 30)
    L, _ = np.linalg.qr(np.random.default_rng(7).standard_normal((5, 5)))
    for boys, cut in ((False, 1e-6), (True, 1e-3), (True, 1e3)):
        ref = O.jctc2024_corrections(Z, Xi, Xa, U, A, Lik=L, cutoff_pno=1e-6, boys_screening=boys,
                                     cutoff_vabij=cut)
        got, _ = handle.jctc2024(Z, Xi, Xa, U, A, Lik=L, cutoff_pno=1e-6, boys_screening=boys, cutoff_vabij=cut)
        for g, r in zip(got, ref):
            assert g == pytest.approx(r, rel=1e-9, abs=1e-14)
    # a screening threshold above every (ab|ij) bound drops the whole 2g..2j term
    got, _ = handle.jctc2024(Z, Xi, Xa, U, A, Lik=L, cutoff_pno=1e-6, boys_screening=True, cutoff_vabij=1e30)
    assert got[3] == 0.0


def test_jctc2024_full_pno_limits(handle):
    # every PNO kept: the PNO direct ring equals the T2 eigenvalue energy and Ec1b/2 the SOSEX energy
    Z, Xa, Xi, U, A = _case(43, 100, 25, 3, 12, 20)
    R = O.thc_r(Z, Xa, Xi)
    got, _ = handle.jctc2024(Z, Xi, Xa, U, A, cutoff_pno=1e-10)
    assert got[0] == pytest.approx(O.t2_eig_rpa(U, A, R).sum(), rel=1e-8)
    assert 0.5 * got[1] == pytest.approx(O.exchange_sosex(np.ascontiguousarray(U.T), A, R, 3, 12), rel=1e-8)
