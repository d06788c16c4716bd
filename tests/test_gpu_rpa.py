"""GPU parity tests of the Pi(u) build and the RPA energy through the C ABI,
against the FP64 oracle and its golden fixtures.

Tolerances (the precision budget of the split form):
  FP64 path:   Pi entries 1e-12 relative to max|Pi|; E_c 1e-10 Eh.
  split-BF16:  Pi off-diagonal 3e-5 relative to max|Pi| (bf16 hi/lo, FP32
               accumulation), diagonal exact to 1e-12 relative; E_c 1e-6 Eh.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import rpa_oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "oracle_golden.json").read_text())


def golden_system(name):
    from tests.golden.make_golden import system
    return system(name)


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("name", ["ragged", "tiny", "water_dimer_twin"])
def test_pi_fp64_matches_oracle(handle, name):
    s, x, w = golden_system(name)
    ref = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
    got = handle.pi_u(s.R, s.eps_o, s.eps_v, x, prec="fp64")
    assert rel_err(got, ref) < 1e-12
    assert np.array_equal(got, np.transpose(got, (0, 2, 1)))


@pytest.mark.parametrize("name", ["ragged", "tiny", "water_dimer_twin", "scaled_c2"])
def test_pi_split_matches_oracle(handle, name):
    s, x, w = golden_system(name)
    ref = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
    got = handle.pi_u(s.R, s.eps_o, s.eps_v, x, prec="split")
    assert rel_err(got, ref) < 3e-5
    for k in range(len(x)):
        assert rel_err(np.diag(got[k]), np.diag(ref[k])) < 1e-12


@pytest.mark.parametrize("name", sorted(GOLDEN))
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("split", 1e-6)])
def test_ec_matches_golden(handle, name, prec, tol):
    g = GOLDEN[name]
    s, x, w = golden_system(name)
    ec, eu = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec=prec)
    assert abs(ec - g["Ec"]) < tol
    eu_tol = 1e-9 if prec == "fp64" else 2e-5
    assert np.max(np.abs(eu - np.array(g["Eu"]))) < eu_tol


def test_ec_from_pi_matches_qr_logdet(handle):
    s, x, w = golden_system("water_dimer_twin")
    pi = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
    ref, ref_eu = O.ec_rpa_analytic(pi, w)
    ec, eu = handle.ec_from_pi(pi, w)
    assert abs(ec - ref) < 1e-11
    assert np.max(np.abs(eu - ref_eu)) < 1e-10


def test_device_pointers_match_host(handle):
    import torch
    s, x, w = golden_system("ragged")
    host = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="split")
    Rt = torch.from_numpy(np.ascontiguousarray(s.R.T)).cuda()  # (nov, NQ) contiguous -> R = Rt.T column-major
    dev = handle.ec_rpa(Rt.T, torch.from_numpy(s.eps_o).cuda(), torch.from_numpy(s.eps_v).cuda(),
                        torch.from_numpy(x).cuda(), torch.from_numpy(w).cuda(), prec="split")
    assert dev[0] == host[0]
    out = torch.empty((len(x), s.nq, s.nq), dtype=torch.float64, device="cuda")
    handle.pi_u(Rt.T, s.eps_o, s.eps_v, x, prec="fp64", out=out)
    ref = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
    assert rel_err(out.cpu().numpy(), ref) < 1e-12


def test_leading_dimension_larger_than_nq(handle):
    # the rows between NQ and the leading dimension are the caller's padding: never read, never
    # screened (NaN there must not raise RPA_ERR_NONFINITE), in the single and the batched path
    s, x, w = golden_system("ragged")
    big = np.full((s.nq + 13, s.R.shape[1]), np.nan, order="F")
    big[: s.nq] = s.R
    import torch
    Rt = torch.from_numpy(np.ascontiguousarray(big.T)).cuda()
    view = Rt.T[: s.nq]  # stride(1) = NQ + 13
    ec, _ = handle.ec_rpa(view, s.eps_o, s.eps_v, x, w, prec="fp64")
    assert abs(ec - GOLDEN["ragged"]["Ec"]) < 1e-10
    esp, _ = handle.ec_rpa(view, s.eps_o, s.eps_v, x, w, prec="split")
    assert abs(esp - GOLDEN["ragged"]["Ec"]) < 1e-6
    eb, _ = handle.ec_batched([(view, s.eps_o, s.eps_v, x, w)], prec="fp64")
    assert abs(eb[0] - GOLDEN["ragged"]["Ec"]) < 1e-10


def test_repeated_calls_are_deterministic(handle):
    s, x, w = golden_system("scaled_c2")
    a = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="split")
    b = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="split")
    assert a[0] == b[0] and np.array_equal(a[1], b[1])


def test_multi_tile_split_against_fp64(handle):
    # several 128 x 256 tiles, nov not a multiple of 32, K > 16 (two frequency groups)
    s = O.make_system(1000, 9, 227, 31, decay=150.0, lam0=0.8)
    x, w = O.casimir_polder(20, 0.8)
    e64, _ = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="fp64")
    esp, _ = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="split")
    assert abs(e64 - esp) < 1e-6
    p64 = handle.pi_u(s.R, s.eps_o, s.eps_v, x[:3], prec="fp64")
    psp = handle.pi_u(s.R, s.eps_o, s.eps_v, x[:3], prec="split")
    assert rel_err(psp, p64) < 3e-5


EDGE_SIZES = [(1, 1, 1, 1), (7, 1, 3, 2), (64, 2, 32, 1), (65, 3, 21, 3), (129, 2, 64, 5), (257, 4, 65, 17)]


def edge_system(nq, no, nv, nf):
    s = O.make_system(nq, no, nv, 500 + nq, decay=max(nq / 4.0, 1.0), lam0=0.7)
    x, w = O.casimir_polder(nf, 0.7)
    return s, x, w


@pytest.mark.parametrize("nq,no,nv,nf", EDGE_SIZES)
def test_minimum_and_block_boundary_sizes(handle, nq, no, nv, nf):
    # one Cholesky vector, one occupied and one virtual orbital, one frequency; orders at and
    # just past the 64-column Cholesky block, the 128-row SYRK tile and the 256-column outer
    # block; 17 frequencies (two split-BF16 groups)
    s, x, w = edge_system(nq, no, nv, nf)
    ref, ref_eu = O.ec_rpa(s.R, s.eps_o, s.eps_v, x, w)
    e64, eu64 = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="fp64")
    esp, _ = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="split")
    assert abs(e64 - ref) < 1e-10
    assert np.max(np.abs(eu64 - ref_eu)) < 1e-10
    assert abs(esp - ref) < 1e-6
    pi = handle.pi_u(s.R, s.eps_o, s.eps_v, x[:2], prec="split")
    assert rel_err(pi, O.pi_matrices(s.R, s.eps_o, s.eps_v, x[:2])) < 3e-5


def test_batched_minimum_and_block_boundary_sizes(handle):
    sys_ = []
    for nq, no, nv, nf in EDGE_SIZES:
        if nf <= 16:
            s, x, w = edge_system(nq, no, nv, nf)
            sys_.append((s.R, s.eps_o, s.eps_v, x, w))
    for prec, tol in (("fp64", 1e-10), ("split", 1e-6)):
        ec, _ = handle.ec_batched(sys_, prec=prec)
        for (R, eo, ev, x, w), e in zip(sys_, ec):
            assert abs(e - O.ec_rpa(R, eo, ev, x, w)[0]) < tol


# ----------------------------------------------------------------------------- errors

def test_nonfinite_input_is_reported(handle, pkg):
    s, x, w = golden_system("tiny")
    R = s.R.copy()
    R[3, 5] = np.nan
    with pytest.raises(pkg.RPAError) as e:
        handle.ec_rpa(R, s.eps_o, s.eps_v, x, w)
    assert e.value.status == pkg.RPA_ERR_NONFINITE


def test_invalid_gap_is_reported(handle, pkg):
    s, x, w = golden_system("tiny")
    eo = s.eps_o.copy()
    eo[-1] = s.eps_v[0] + 0.1
    with pytest.raises(pkg.RPAError) as e:
        handle.ec_rpa(s.R, eo, s.eps_v, x, w)
    assert e.value.status == pkg.RPA_ERR_INVALID_ARG


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 127, 128, 129, 191, 257, 320])
def test_ec_from_pi_at_block_boundaries(handle, n):
    # orders around the 64-column diagonal blocks (factored with their inverses, a panel solve only
    # below a full block) and the 256-column outer blocks of the blocked Cholesky: E(u) = ln det(1 +
    # Pi) - Tr Pi against LAPACK on the same symmetric positive semidefinite Pi
    rng = np.random.default_rng(1000 + n)
    w = np.array([0.7, 1.1, 0.4])
    pis = []
    for k in range(len(w)):
        B = rng.standard_normal((n, n // 2 + 3))
        P = B @ B.T
        pis.append(P * ((0.3 + 0.25 * k) / np.linalg.eigvalsh(P)[-1]))
    pi = np.stack(pis)
    ref = np.array([np.linalg.slogdet(np.eye(n) + p)[1] - np.trace(p) for p in pis])
    ec, eu = handle.ec_from_pi(pi, w)
    assert np.max(np.abs(eu - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref))), (eu, ref)
    assert abs(ec - float(np.sum(w * ref)) / (2 * np.pi)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_batched_log_det_at_block_boundaries(handle):
    # the variable-order batched Cholesky (orders 63 .. 257 in one order bucket and the next)
    # against the single-system path on the same FP64 Pi
    systems, refs = [], []
    for i, nq in enumerate((63, 64, 65, 129, 257)):
        s = O.make_system(nq, 3, 12 + i, 600 + i, lam0=0.8)
        x, w = O.grid_for(s, 4)
        systems.append((s.R, s.eps_o, s.eps_v, x, w))
        refs.append(handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="fp64")[0])
    ec, _ = handle.ec_batched(systems, prec="fp64")
    assert np.max(np.abs(np.array(ec) - np.array(refs))) <= 1e-11, (ec, refs)


def test_not_spd_is_reported(handle, pkg):
    pi = np.zeros((2, 70, 70))
    pi[0] = np.eye(70) * 0.1
    pi[1] = np.eye(70) * 0.1
    pi[1, 65, 65] = -1.5  # 1 + Pi has a negative eigenvalue
    with pytest.raises(pkg.RPAError) as e:
        handle.ec_from_pi(pi, np.array([0.5, 0.5]))
    assert e.value.status == pkg.RPA_ERR_NOT_SPD
    # the handle stays usable afterwards
    ec, eu = handle.ec_from_pi(pi[:1], np.array([1.0]))
    assert np.isfinite(ec)


def test_bad_dimensions_are_rejected(handle, pkg):
    s, x, w = golden_system("tiny")
    with pytest.raises(pkg.RPAError) as e:
        handle.ec_rpa(s.R, s.eps_o, s.eps_v, np.zeros(65), np.zeros(65))
    assert e.value.status == pkg.RPA_ERR_INVALID_ARG


def test_host_r_pipelined_staging_matches_device_r(handle):
    # host R with several ai pieces: staging overlapped with the split and the SYRK of earlier
    # pieces (FP64 accumulation across pieces), against the one-shot build from device R
    import torch
    s = O.make_system(700, 12, 180, 41, decay=90.0, lam0=0.8)
    x, w = O.casimir_polder(14, 0.8)
    host = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="split")
    Rt = torch.from_numpy(np.ascontiguousarray(s.R.T)).cuda()
    dev = handle.ec_rpa(Rt.T, s.eps_o, s.eps_v, x, w, prec="split")
    # the pieces are summed in FP64 (the one-shot build keeps one FP32 running sum per tile):
    # both are within the split-precision budget and the piecewise sum is no farther from FP64
    assert abs(host[0] - dev[0]) < 1e-7
    assert np.max(np.abs(host[1] - dev[1])) < 1e-7
    e64, _ = handle.ec_rpa(Rt.T, s.eps_o, s.eps_v, x, w, prec="fp64")
    assert abs(host[0] - e64) <= abs(dev[0] - e64) + 1e-9
    ref, _ = O.ec_rpa(s.R, s.eps_o, s.eps_v, x, w)
    assert abs(host[0] - ref) < 1e-6


def test_host_r_pipelined_nonfinite_is_reported(handle, pkg):
    s = O.make_system(700, 12, 180, 41, decay=90.0, lam0=0.8)
    x, w = O.casimir_polder(14, 0.8)
    R = s.R.copy()
    R[5, R.shape[1] - 3] = np.inf  # in the last staged piece
    with pytest.raises(pkg.RPAError) as e:
        handle.ec_rpa(R, s.eps_o, s.eps_v, x, w, prec="split")
    assert e.value.status == pkg.RPA_ERR_NONFINITE
    ec, _ = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="split")  # the handle stays usable
    assert np.isfinite(ec)
