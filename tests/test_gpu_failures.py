"""Failure detection on the GPU, without faulting it: a bounded device wait that expires, a
device allocation that fails, and entries the library must not read.

Every spin-wait in the library's kernels gives up after its limit, records a code in the
handle's device error word and returns; the call then reports RPA_ERR_TIMEOUT and the CUDA
context stays usable.  The self-test entry point runs that wait on a barrier that nothing arrives
on.  Device allocation failures are produced on the host by the handle's workspace cap.
"""
import time

import numpy as np
import pytest

from oracle import rpa_oracle as O

pytestmark = pytest.mark.gpu


def _small(seed=11):
    s = O.make_system(160, 4, 30, seed, decay=20.0, lam0=0.7)
    x, w = O.grid_for(s, 6)
    return s, x, w


def test_expired_device_wait_is_reported_and_the_handle_recovers(pkg, handle):
    s, x, w = _small()
    ref, _ = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="fp64")
    t0 = time.perf_counter()
    st = handle.selftest_wait_timeout(25.0)
    dt = time.perf_counter() - t0
    assert st == pkg.RPA_ERR_TIMEOUT
    assert dt >= 0.020  # the wait ran to its limit before giving up
    assert b"bounded wait expired" in handle.lib.rpa_b200_last_error(handle._h)
    # the context and the handle are still usable; the error word starts clean on the next call
    ec, _ = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="fp64")
    assert ec == ref
    ec, _ = handle.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="split")
    assert abs(ec - ref) < 1e-6


def test_selftest_rejects_limits_outside_the_library_range(pkg, handle):
    assert handle.selftest_wait_timeout(0.0) == pkg.RPA_ERR_INVALID_ARG
    assert handle.selftest_wait_timeout(5000.0) == pkg.RPA_ERR_INVALID_ARG


def test_workspace_cap_turns_an_allocation_into_oom(pkg):
    s, x, w = _small(12)
    with pkg.Handle(0) as h:
        h.set_workspace_limit(64 * 1024)  # far below what one energy needs
        with pytest.raises(pkg.RPAError) as err:
            h.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="split")
        assert err.value.status == pkg.RPA_ERR_OOM
        used, limit = h.workspace_bytes()
        assert used <= limit == 64 * 1024
        h.set_workspace_limit(0)  # lift the cap: the same handle completes the call
        ec, _ = h.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="split")
        ref, _ = O.ec_rpa(s.R, s.eps_o, s.eps_v, x, w)
        assert abs(ec - ref) < 1e-6
        used, _ = h.workspace_bytes()
        assert used > 0
        # a cap at the bytes now held lets calls of the same shape run without growing
        h.set_workspace_limit(used)
        ec2, _ = h.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec="split")
        assert ec2 == ec


def test_upper_triangle_of_pi_is_never_read(pkg, handle):
    # Pi(u) arguments: only the lower triangle is read, so non-finite data above the diagonal (of
    # a device input that reaches the workspace through the lower-triangle copy, or of a host input
    # copied whole) must not raise RPA_ERR_NONFINITE
    import torch
    s, x, w = _small(13)
    pi = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
    ref = handle.ec_from_pi(pi, w)
    up = pi.copy()
    up[:, 40, 3] = np.nan  # pi[k, c, r] = entry (r, c): r = 3 < c = 40, above the diagonal
    ec, _ = handle.ec_from_pi(up, w)
    assert ec == ref[0]
    ec, _ = handle.ec_from_pi(torch.from_numpy(up).cuda(), w)
    assert ec == ref[0]
    low = pi.copy()
    low[2, 3, 40] = np.inf  # r = 40 > c = 3: read
    with pytest.raises(pkg.RPAError) as err:
        handle.ec_from_pi(torch.from_numpy(low).cuda(), w)
    assert err.value.status == pkg.RPA_ERR_NONFINITE


@pytest.mark.parametrize("prec", ["fp64", "split"])
def test_nonfinite_exchange_inputs_are_reported(pkg, handle, prec):
    # the exchange entry points do not screen R and U: a non-finite input shows in the energy, which
    # is reported as RPA_ERR_NONFINITE (not returned as NaN), and the handle stays usable
    rng = np.random.default_rng(5)
    nq, no, nv, nt = 77, 5, 19, 45
    R = rng.standard_normal((nq, no * nv)) * 0.1
    U = rng.standard_normal((no * nv, nt)) * 0.2
    A = -0.05 * rng.uniform(size=nt)
    good = handle.exchange_sosex(R, no, nv, U, A, alpha=2.0, prec=prec)
    bad = U.copy()
    bad[17, 3] = np.nan
    with pytest.raises(pkg.RPAError) as err:
        handle.exchange_sosex(R, no, nv, bad, A, alpha=2.0, prec=prec)
    assert err.value.status == pkg.RPA_ERR_NONFINITE
    assert handle.exchange_sosex(R, no, nv, U, A, alpha=2.0, prec=prec) == good


def test_nonfinite_pno_inputs_are_reported(pkg, handle):
    Z, Xa, Xi, eo, ev = O.make_thc_factors(120, 30, 4, 16, 41)
    rng = np.random.default_rng(141)
    U, _ = np.linalg.qr(rng.standard_normal((4 * 16, 24)))
    A = -0.2 * rng.uniform(size=24)
    Z = Z.copy()
    Z[7, 2] = np.inf
    with pytest.raises(pkg.RPAError) as err:
        handle.jctc2024(Z, Xi, Xa, U, A, cutoff_pno=1e-8)
    assert err.value.status == pkg.RPA_ERR_NONFINITE


def test_nonfinite_thc_and_projection_inputs_are_reported(pkg, handle):
    # array entry points that do not screen their inputs screen their output instead
    Z, Xa, Xi, eo, ev = O.make_thc_factors(90, 20, 3, 11, 43)
    good = handle.thc_r(Z, Xa, Xi)
    bad = Z.copy()
    bad[5, 4] = np.nan
    with pytest.raises(pkg.RPAError) as err:
        handle.thc_r(bad, Xa, Xi)
    assert err.value.status == pkg.RPA_ERR_NONFINITE
    G = np.linalg.qr(np.random.default_rng(9).standard_normal((20, 8)))[0]
    Rp = handle.project_basis(G, good)
    assert np.allclose(Rp, G.T @ good, rtol=1e-12, atol=1e-14)
    Gb = G.copy()
    Gb[3, 2] = np.inf
    with pytest.raises(pkg.RPAError) as err:
        handle.project_basis(Gb, good)
    assert err.value.status == pkg.RPA_ERR_NONFINITE


def test_nonfinite_t2_guess_vectors_are_reported(pkg, handle):
    s = O.make_system(60, 3, 10, 77, lam0=0.8)
    x, w = O.grid_for(s, 4)
    omega = np.random.default_rng(2).uniform(-0.5, 0.5, size=(3 * 10, 24))
    omega[4, 7] = np.nan
    with pytest.raises(pkg.RPAError) as err:
        handle.dring_t2(s.R, s.eps_o, s.eps_v, x, w, prec="fp64", guess=omega)
    assert err.value.status == pkg.RPA_ERR_NONFINITE
