"""GPU tests of the THC path: Cholesky vectors formed from THC factors (rpa_b200_thc_r,
replacing rpa_THC_Rkab/Rkai) and the energy from THC factors (rpa_b200_ec_thc).

Tolerances: R to 1e-12 relative to max|R| (FP64 tensor-core GEMM); E_c to 1e-10 Eh (FP64) and
1e-6 Eh (split-BF16 Pi) against the oracle energy of the oracle's R.
"""
import numpy as np
import pytest

from oracle import rpa_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(300, 120, 5, 30), (517, 90, 7, 33)])
def test_thc_r_matches_oracle(handle, shape):
    ng, nq, no, nv = shape
    Z, Xa, Xi, eo, ev = O.make_thc_factors(ng, nq, no, nv, 11)
    R = handle.thc_r(Z, Xa, Xi)
    ref = O.thc_r(Z, Xa, Xi)
    assert np.max(np.abs(R - ref)) < 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("split", 1e-6)])
def test_ec_thc_matches_oracle(handle, prec, tol):
    Z, Xa, Xi, eo, ev = O.make_thc_factors(400, 150, 6, 40, 12)
    R = O.thc_r(Z, Xa, Xi)
    x, w = O.casimir_polder(12, 0.8)
    ref, ref_eu = O.ec_rpa(R, eo, ev, x, w)
    ec, eu = handle.ec_thc(Z, Xa, Xi, eo, ev, x, w, prec=prec)
    assert abs(ec - ref) < tol
    assert np.max(np.abs(eu - ref_eu)) < 10 * tol


@pytest.mark.parametrize("piece_bytes", [None, 3 * 1024 * 1024])
def test_ec_thc_pieces_never_hold_whole_R(pkg, monkeypatch, piece_bytes):
    # split precision: R is formed and contracted piece by piece (Khatri-Rao block, FP64 GEMM,
    # scale/split, tensor-core SYRK adding into Pi); with a small piece budget the build runs in
    # many pieces and the device holds far less than R plus its split operands
    Z, Xa, Xi, eo, ev = O.make_thc_factors(512, 128, 16, 200, 13)
    R = O.thc_r(Z, Xa, Xi)
    x, w = O.casimir_polder(12, 0.7)
    ref, _ = O.ec_rpa(R, eo, ev, x, w)
    if piece_bytes:
        monkeypatch.setenv("RPA_B200_THC_PIECE_BYTES", str(piece_bytes))
    with pkg.Handle(0) as h:
        ec, _ = h.ec_thc(Z, Xa, Xi, eo, ev, x, w, prec="split")
        used, _ = h.workspace_bytes()
    assert abs(ec - ref) < 1e-6
    whole = R.nbytes + 4 * len(x) * R.size  # R in FP64 + its hi/lo operands for every frequency
    if piece_bytes:
        # 3200 ai columns in pieces of 256: the pieces' buffers, Pi and the staged factors only
        assert used < 0.5 * whole, (used, whole)
