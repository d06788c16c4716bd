"""GPU parity of the direct-ring T2 amplitudes and the SOSEX exchange energy
against the FP64 oracle (rpa_THC_CC_T2 / rpa_T2_EigRPA / rpa_CC_Exchange_SOSEX
restatements).  With the same guess vectors the GPU and the oracle follow the
same algorithm, so amplitudes agree to rounding; with the library's own guess
vectors parity is at the converged-subspace level (energies).

Tolerances: A to 1e-8 relative; eigenvectors |<u_gpu, u_ref>| >= 1 - 1e-6;
EigRPA sum and SOSEX energies to 1e-10 Eh (FP64); 1e-6 Eh with the split-BF16
Pi or a different guess set.
"""
import math

import numpy as np
import pytest

from oracle import rpa_oracle as O

pytestmark = pytest.mark.gpu


def t2_case(seed, nq, no, nv, K, lam0=0.6):
    s = O.make_system(nq, no, nv, seed, decay=nq / 5.0, lam0=lam0)
    x, w = O.grid_for(s, K)
    pi = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
    vals, vecs = O.diagonalize_pi(pi)
    nov = no * nv
    G = min(int(math.ceil(3.0 * nq)), nov)
    omega = np.random.default_rng(seed).uniform(size=(nov, G)) - 0.5
    return s, x, w, pi, vals, vecs, omega


@pytest.mark.parametrize("shape", [(60, 4, 20, 10), (150, 6, 50, 12)])
def test_t2_matches_oracle_with_same_guess(handle, shape):
    nq, no, nv, K = shape
    s, x, w, pi, vals, vecs, omega = t2_case(11, nq, no, nv, K)
    A_ref, U_ref, K_ref = O.t2_direct_ring(s.R, s.eps_o, s.eps_v, x, w, vals, vecs, omega, cutoff_thresh=1e-4)
    res = handle.dring_t2(s.R, s.eps_o, s.eps_v, x, w, prec="fp64", guess=omega, cutoff_thresh=1e-4)
    assert res["NT"] == len(A_ref)
    assert np.allclose(res["A"], A_ref, rtol=1e-8, atol=1e-13)
    dots = np.abs(np.sum(res["U"] * U_ref, axis=0))
    assert np.all(dots > 1 - 1e-6)
    eig_ref = O.t2_eig_rpa(U_ref, A_ref, s.R)
    assert abs(res["EigRPA"].sum() - eig_ref.sum()) < 1e-10
    assert res["common_thresh"] == pytest.approx(K_ref)
    ec_ref, _ = O.ec_rpa_analytic(pi, w)
    assert abs(res["Ec"] - ec_ref) < 1e-10


def test_t2_energy_identity_with_device_guess(handle):
    # identity (i): with every direction kept, sum_mu 2 A_mu |R U_mu|^2 == E_c
    s, x, w, pi, vals, vecs, omega = t2_case(12, 60, 4, 20, 10)
    res = handle.dring_t2(s.R, s.eps_o, s.eps_v, x, w, prec="fp64", seed=7, cutoff_thresh=1e-14)
    ec_ref, _ = O.ec_rpa_analytic(pi, w)
    assert abs(res["EigRPA"].sum() - ec_ref) < 1e-6 * abs(ec_ref)
    # directions kept down to the 1e-10 Gram cutoff carry ~1e-16/1e-10 rounding: orthonormal to ~1e-6
    assert np.allclose(res["U"].T @ res["U"], np.eye(res["NT"]), atol=1e-5)


@pytest.mark.parametrize("ctype,thresh", [(0, 1e-4), (1, 1e-3), (2, 1e-3), (3, 1e-4)])
def test_t2_cutoff_types(handle, ctype, thresh):
    s, x, w, pi, vals, vecs, omega = t2_case(13, 60, 4, 20, 10)
    A_ref, U_ref, K_ref = O.t2_direct_ring(s.R, s.eps_o, s.eps_v, x, w, vals, vecs, omega, cutoff_thresh=thresh,
                                           cutoff_type=ctype, nocc=s.no)
    res = handle.dring_t2(s.R, s.eps_o, s.eps_v, x, w, prec="fp64", guess=omega, cutoff_thresh=thresh,
                          cutoff_type=ctype)
    assert res["NT"] == len(A_ref)
    assert res["common_thresh"] == pytest.approx(K_ref, rel=1e-8)


def test_t2_subsystem_uses_common_threshold(handle):
    s, x, w, pi, vals, vecs, omega = t2_case(14, 60, 4, 20, 10)
    A_ref, _, _ = O.t2_direct_ring(s.R, s.eps_o, s.eps_v, x, w, vals, vecs, omega, common_thresh=3e-3)
    res = handle.dring_t2(s.R, s.eps_o, s.eps_v, x, w, prec="fp64", guess=omega, common_thresh=3e-3)
    assert res["NT"] == len(A_ref) and res["common_thresh"] == 3e-3


def test_t2_split_precision_energy(handle):
    s, x, w, pi, vals, vecs, omega = t2_case(15, 150, 6, 50, 12)
    A_ref, U_ref, _ = O.t2_direct_ring(s.R, s.eps_o, s.eps_v, x, w, vals, vecs, omega, cutoff_thresh=1e-6)
    res = handle.dring_t2(s.R, s.eps_o, s.eps_v, x, w, prec="split", guess=omega, cutoff_thresh=1e-6)
    assert abs(res["EigRPA"].sum() - O.t2_eig_rpa(U_ref, A_ref, s.R).sum()) < 1e-6


def test_t2_split_ring_contractions_track_fp64(handle):
    # prec split: Pi and the two ring contractions of every I(1) application (P = Z M and
    # Z^T P) run as split-BF16 tensor-core GEMMs; the Gram and Rayleigh-Ritz matrices and the
    # eigensolvers stay FP64.  A numpy emulation of the split products gives ~6e-7 relative
    # error in A and ~4e-8 Eh in EigRPA at these sizes; the bounds below leave 10-30x margin.
    s, x, w, pi, vals, vecs, omega = t2_case(19, 200, 8, 60, 12)
    r64 = handle.dring_t2(s.R, s.eps_o, s.eps_v, x, w, prec="fp64", guess=omega, cutoff_thresh=1e-4)
    r16 = handle.dring_t2(s.R, s.eps_o, s.eps_v, x, w, prec="split", guess=omega, cutoff_thresh=1e-4)
    assert r16["NT"] == r64["NT"]
    assert np.max(np.abs(r16["A"] - r64["A"])) < 2e-5 * np.max(np.abs(r64["A"]))
    assert abs(r16["EigRPA"].sum() - r64["EigRPA"].sum()) < 2e-6 * abs(r64["EigRPA"].sum())
    ex16 = handle.exchange_sosex(s.R, s.no, s.nv, r16["U"], r16["A"], prec="split")
    ex64 = handle.exchange_sosex(s.R, s.no, s.nv, r64["U"], r64["A"], prec="fp64")
    assert abs(ex16 - ex64) < 2e-5 * abs(ex64)


@pytest.mark.parametrize("s2", [False, True])
def test_sosex_matches_oracle(handle, s2):
    s, x, w, pi, vals, vecs, omega = t2_case(16, 150, 6, 50, 12)
    A_ref, U_ref, _ = O.t2_direct_ring(s.R, s.eps_o, s.eps_v, x, w, vals, vecs, omega, cutoff_thresh=1e-4)
    ref = O.exchange_sosex(np.ascontiguousarray(U_ref.T), A_ref, s.R, s.no, s.nv, alpha=1.0, s2_operator=s2)
    got = handle.exchange_sosex(s.R, s.no, s.nv, U_ref, A_ref, alpha=1.0, s2_operator=s2)
    assert abs(got - ref) < 1e-11 * max(1.0, abs(ref))


def test_sosex_ragged_shapes(handle):
    # NQ, nv and NT not multiples of the 64/16 tiles
    rng = np.random.default_rng(3)
    nq, no, nv, nt = 77, 5, 19, 45
    R = rng.standard_normal((nq, no * nv)) * 0.1
    U = rng.standard_normal((no * nv, nt)) * 0.2
    A = -0.05 * rng.uniform(size=nt)
    ref = O.exchange_sosex(np.ascontiguousarray(U.T), A, R, no, nv, alpha=2.0)
    got = handle.exchange_sosex(R, no, nv, U, A, alpha=2.0)
    assert abs(got - ref) < 1e-12 * max(1.0, abs(ref))


# Split-BF16 pair contraction (tcgen05): R and U as bf16 hi/lo pairs, three products, FP32
# accumulation in 64-column segments.  The accumulator's round-toward-zero bias leaves a
# relative error of ~1e-6 in E_x on physical amplitudes (a numpy emulation of the
# accumulation gives 6e-7); the bound below is 5e-6 relative.  Random (unphysical) data
# cancels more and is checked to 1e-4 relative.

@pytest.mark.parametrize("s2", [False, True])
def test_sosex_split_matches_oracle(handle, s2):
    s, x, w, pi, vals, vecs, omega = t2_case(16, 150, 6, 50, 12)
    A_ref, U_ref, _ = O.t2_direct_ring(s.R, s.eps_o, s.eps_v, x, w, vals, vecs, omega, cutoff_thresh=1e-4)
    ref = O.exchange_sosex(np.ascontiguousarray(U_ref.T), A_ref, s.R, s.no, s.nv, alpha=1.0, s2_operator=s2)
    got = handle.exchange_sosex(s.R, s.no, s.nv, U_ref, A_ref, alpha=1.0, s2_operator=s2, prec="split")
    assert abs(got - ref) < 5e-6 * abs(ref)
    again = handle.exchange_sosex(s.R, s.no, s.nv, U_ref, A_ref, alpha=1.0, s2_operator=s2, prec="split")
    assert again == got  # fixed-order reductions: bit-identical


def test_sosex_split_ragged_shapes(handle):
    # nv = 19 (padded to 32), NQ = 77 and NT = 45 (partial 128-row tiles)
    rng = np.random.default_rng(3)
    nq, no, nv, nt = 77, 5, 19, 45
    R = rng.standard_normal((nq, no * nv)) * 0.1
    U = rng.standard_normal((no * nv, nt)) * 0.2
    A = -0.05 * rng.uniform(size=nt)
    ref = O.exchange_sosex(np.ascontiguousarray(U.T), A, R, no, nv, alpha=2.0)
    got = handle.exchange_sosex(R, no, nv, U, A, alpha=2.0, prec="split")
    assert abs(got - ref) < 1e-4 * abs(ref)


def test_sosex_split_device_inputs_and_many_tiles(handle):
    # NQ = 300 (3 row tiles), NT = 260 (3 column tiles), nv = 80 (padded to 96: three chunks,
    # two accumulation segments)
    import torch
    rng = np.random.default_rng(8)
    s = O.make_system(300, 4, 80, 31, decay=50.0, lam0=0.7)
    U, _ = np.linalg.qr(rng.standard_normal((s.no * s.nv, 260)))
    A = -0.1 * rng.uniform(size=260)
    ref = O.exchange_sosex(np.ascontiguousarray(U.T), A, s.R, s.no, s.nv)
    Rd = torch.from_numpy(np.ascontiguousarray(s.R.T)).cuda().T
    Ud = torch.from_numpy(np.ascontiguousarray(U.T)).cuda().T
    got = handle.exchange_sosex(Rd, s.no, s.nv, Ud, A, prec="split")
    assert abs(got - ref) < 5e-6 * abs(ref)


# ----------------------------------------------------------------------------- MBPT3 exchange
# Tolerances: E_x to 1e-11 relative (FP64 throughout; the GPU Lyapunov solve
# stops at |res| <= 1e-13 |A|); X to 1e-10 relative to max|X|.

def test_mbpt3_matches_oracle(handle):
    s, x, w, pi, vals, vecs, omega = t2_case(17, 150, 6, 50, 12)
    A_ref, U_ref, _ = O.t2_direct_ring(s.R, s.eps_o, s.eps_v, x, w, vals, vecs, omega, cutoff_thresh=1e-4)
    ref, X_ref = O.exchange_mbpt3_1(U_ref, A_ref, s.R, s.eps_o, s.eps_v)
    got, X = handle.exchange_mbpt3(s.R, s.eps_o, s.eps_v, U_ref, A_ref, return_x=True)
    assert abs(got - ref) < 1e-11 * max(1.0, abs(ref))
    assert np.max(np.abs(X - X_ref)) < 1e-10 * np.max(np.abs(X_ref))


def test_mbpt3_ragged_shapes(handle):
    # NQ, nv and an odd NT not multiples of any tile; orthonormal U, small negative A
    rng = np.random.default_rng(5)
    s = O.make_system(77, 5, 19, 21, decay=12.0, lam0=0.6)
    nt = 45
    U, _ = np.linalg.qr(rng.standard_normal((s.no * s.nv, nt)))
    A = -0.08 * rng.uniform(size=nt)
    ref, X_ref = O.exchange_mbpt3_1(U, A, s.R, s.eps_o, s.eps_v)
    got, X = handle.exchange_mbpt3(s.R, s.eps_o, s.eps_v, U, A, return_x=True)
    assert abs(got - ref) < 1e-11 * max(1.0, abs(ref))
    assert np.max(np.abs(X - X_ref)) < 1e-10 * np.max(np.abs(X_ref))


def test_mbpt3_after_gpu_t2(handle):
    # the CC-path chain: T2 amplitudes from the GPU, then the MBPT3 exchange from them
    s, x, w, pi, vals, vecs, omega = t2_case(18, 120, 5, 40, 10)
    res = handle.dring_t2(s.R, s.eps_o, s.eps_v, x, w, prec="fp64", guess=omega, cutoff_thresh=1e-4)
    ref, _ = O.exchange_mbpt3_1(res["U"], res["A"], s.R, s.eps_o, s.eps_v)
    got = handle.exchange_mbpt3(s.R, s.eps_o, s.eps_v, res["U"], res["A"])
    assert abs(got - ref) < 1e-11 * max(1.0, abs(ref))


def test_mbpt3_split_contraction_matches_oracle(handle):
    s, x, w, pi, vals, vecs, omega = t2_case(17, 150, 6, 50, 12)
    A_ref, U_ref, _ = O.t2_direct_ring(s.R, s.eps_o, s.eps_v, x, w, vals, vecs, omega, cutoff_thresh=1e-4)
    ref, X_ref = O.exchange_mbpt3_1(U_ref, A_ref, s.R, s.eps_o, s.eps_v)
    got, X = handle.exchange_mbpt3(s.R, s.eps_o, s.eps_v, U_ref, A_ref, return_x=True, prec="split")
    assert abs(got - ref) < 5e-6 * abs(ref)
    assert np.max(np.abs(X - X_ref)) < 1e-10 * np.max(np.abs(X_ref))  # the Lyapunov solve stays FP64


def test_mbpt3_indefinite_operator_is_reported(handle, pkg):
    # occupied energies above the virtual ones make D, hence the symmetric part of B, negative
    rng = np.random.default_rng(6)
    s = O.make_system(40, 3, 10, 22, decay=10.0, lam0=0.5)
    U, _ = np.linalg.qr(rng.standard_normal((30, 12)))
    A = -0.05 * rng.uniform(size=12)
    with pytest.raises(pkg.RPAError) as e:
        handle.exchange_mbpt3(s.R, s.eps_v[:3] + 10.0, s.eps_v, U, A)
    assert e.value.status == pkg.RPA_ERR_NOT_CONVERGED
    got = handle.exchange_mbpt3(s.R, s.eps_o, s.eps_v, U, A)  # the handle stays usable
    assert np.isfinite(got)
