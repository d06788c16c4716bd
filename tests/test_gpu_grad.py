"""GPU tests of the adjoint dE_c/dR, dE_c/de (rpa_b200_ec_grad and the
torch.autograd.Function): against the FP64 oracle gradient and central finite
differences (step 1e-5) on 64 random entries.

Tolerances: FP64 path relative error <= 1e-10 against the oracle gradient and
<= 1e-6 (plus 1e-7 of the largest gradient entry, the O(h^2) truncation of
central differences) against finite differences; split-BF16 Pi relative error <= 3e-4 (the
Pi contraction carries ~1e-5 relative rounding into (1+Pi)^{-1}).
"""
import numpy as np
import pytest

from oracle import rpa_oracle as O

pytestmark = pytest.mark.gpu


def case(seed=21, nq=160, no=5, nv=40, K=10):
    s = O.make_system(nq, no, nv, seed, decay=nq / 6.0, lam0=0.7)
    x, w = O.grid_for(s, K)
    return s, x, w


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("split", 3e-4)])
def test_grad_matches_oracle(handle, prec, tol):
    s, x, w = case()
    dR_ref, do_ref, dv_ref = O.ec_grad(s.R, s.eps_o, s.eps_v, x, w)
    ec, dR, do, dv = handle.ec_grad(s.R, s.eps_o, s.eps_v, x, w, prec=prec)
    assert rel(dR, dR_ref) < tol
    assert rel(do, do_ref) < tol and rel(dv, dv_ref) < tol
    ref_ec, _ = O.ec_rpa(s.R, s.eps_o, s.eps_v, x, w)
    assert abs(ec - ref_ec) < (1e-10 if prec == "fp64" else 1e-6)


def test_grad_central_finite_differences(handle):
    s, x, w = case(seed=22, nq=120, no=4, nv=30, K=10)
    _, dR, do, dv = handle.ec_grad(s.R, s.eps_o, s.eps_v, x, w, prec="fp64")
    h = 1e-5
    rng = np.random.default_rng(5)
    for _ in range(64):
        q, ai = int(rng.integers(s.nq)), int(rng.integers(s.no * s.nv))
        Rp, Rm = s.R.copy(), s.R.copy()
        Rp[q, ai] += h
        Rm[q, ai] -= h
        fd = (handle.ec_rpa(Rp, s.eps_o, s.eps_v, x, w, prec="fp64")[0] -
              handle.ec_rpa(Rm, s.eps_o, s.eps_v, x, w, prec="fp64")[0]) / (2 * h)
        # central differences carry an O(h^2) truncation error (~1e-10 here): relative 1e-6 on the
        # entry plus 1e-7 of the gradient's largest entry
        assert abs(fd - dR[q, ai]) <= 1e-6 * abs(fd) + 1e-7 * np.max(np.abs(dR))
    for i in range(s.no):
        ep, em = s.eps_o.copy(), s.eps_o.copy()
        ep[i] += h
        em[i] -= h
        fd = (handle.ec_rpa(s.R, ep, s.eps_v, x, w, prec="fp64")[0] -
              handle.ec_rpa(s.R, em, s.eps_v, x, w, prec="fp64")[0]) / (2 * h)
        assert abs(fd - do[i]) <= 1e-6 * abs(fd) + 1e-7 * np.max(np.abs(do))


def test_autograd_function_matches_entry_point(handle, pkg):
    import importlib
    import torch
    ag = importlib.import_module("beyond_rpa_b200.autograd")
    s, x, w = case(seed=23, nq=100, no=4, nv=25, K=8)
    Rt = torch.from_numpy(np.ascontiguousarray(s.R.T)).cuda()
    R = Rt.T.detach().requires_grad_(True)
    eo = torch.from_numpy(s.eps_o).cuda().requires_grad_(True)
    ev = torch.from_numpy(s.eps_v).cuda().requires_grad_(True)
    fr = torch.from_numpy(x).cuda()
    wt = torch.from_numpy(w).cuda()
    e = ag.rpa_energy(R, eo, ev, fr, wt, handle, prec="fp64")
    gR, go, gv = torch.autograd.grad(3.0 * e, (R, eo, ev))
    ec, dR, do, dv = handle.ec_grad(s.R, s.eps_o, s.eps_v, x, w, prec="fp64")
    assert abs(e.item() - ec) < 1e-12
    assert rel(gR.cpu().numpy(), 3.0 * dR) < 1e-12
    assert rel(go.cpu().numpy(), 3.0 * do) < 1e-12 and rel(gv.cpu().numpy(), 3.0 * dv) < 1e-12
