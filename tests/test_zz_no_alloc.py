"""GPU test of rpa_b200_ec_from_pi_noalloc, the allocation-free entry point for
callers that cannot allocate GPU memory (their device memory belongs to a
pool or arena they cannot grow, or the footprint must not change while they
run).  It must give the same energies as rpa_b200_ec_from_pi, call after call
on the one shared scratch array, and refuse problems larger than that array.

This file is collected last so that a failure here, in a run that stops at
the first failure, comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from oracle import rpa_oracle as O

pytestmark = pytest.mark.gpu


def _noalloc(pkg, pi, weights, device=0, stream=None):
    lib = pkg.load_library()
    K, nq = int(pi.shape[0]), int(pi.shape[1])
    ec = ctypes.c_double()
    eu = np.zeros(K)
    if type(pi).__module__.startswith("torch"):
        ptr = pi.data_ptr()
    else:
        pi = np.ascontiguousarray(pi, dtype=np.float64)
        ptr = pi.ctypes.data
    w = np.ascontiguousarray(weights, dtype=np.float64)
    st = lib.rpa_b200_ec_from_pi_noalloc(device, stream, nq, K, ptr, nq, w.ctypes.data, ctypes.byref(ec),
                                         eu.ctypes.data)
    return st, ec.value, eu


def _case(seed, nq, no, nv, K):
    s = O.make_system(nq, no, nv, seed, decay=nq / 8.0, lam0=0.8)
    x, w = O.grid_for(s, K)
    return O.pi_matrices(s.R, s.eps_o, s.eps_v, x), w


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(pkg, handle):
    import torch
    # two different problems in a row: the second call must not see the first one's leftovers
    pi_a, w_a = _case(501, 400, 8, 72, 12)
    pi_b, w_b = _case(502, 200, 5, 37, 5)
    ref_a = handle.ec_from_pi(pi_a, w_a)
    ref_b = handle.ec_from_pi(pi_b, w_b)
    st, ec, eu = _noalloc(pkg, pi_a, w_a)                       # host input
    assert st == pkg.RPA_OK
    assert abs(ec - ref_a[0]) < 1e-11 and np.max(np.abs(eu - ref_a[1])) < 1e-10
    st, ec, eu = _noalloc(pkg, torch.from_numpy(pi_b).cuda(), w_b)  # device input
    assert st == pkg.RPA_OK
    assert abs(ec - ref_b[0]) < 1e-11 and np.max(np.abs(eu - ref_b[1])) < 1e-10


def test_noalloc_statuses_leave_no_stale_state(pkg, handle):
    import torch
    pi_a, w_a = _case(503, 300, 6, 50, 8)
    pi_b, w_b = _case(504, 200, 5, 37, 5)
    ref_a = handle.ec_from_pi(pi_a, w_a)
    ref_b = handle.ec_from_pi(pi_b, w_b)
    # pi[k, c, r] is entry (r, c) of the column-major Pi(u_k) the library reads (column c, row r)
    # NaN in the lower triangle (r >= c): reported, and the next (device-input, other NQ) call is clean
    bad = pi_a.copy()
    bad[3, 5, 17] = np.nan
    st, _, _ = _noalloc(pkg, bad, w_a)
    assert st == pkg.RPA_ERR_NONFINITE
    st, ec, _ = _noalloc(pkg, torch.from_numpy(pi_b).cuda(), w_b)
    assert st == pkg.RPA_OK and abs(ec - ref_b[0]) < 1e-11
    # NaN only above the diagonal is never read: a host call that copies it into the shared array and
    # the device-input call after it (which copies only the lower triangle over it) both succeed
    up = pi_a.copy()
    up[:, 17, 5] = np.nan
    st, ec, _ = _noalloc(pkg, up, w_a)
    assert st == pkg.RPA_OK and abs(ec - ref_a[0]) < 1e-11
    st, ec, _ = _noalloc(pkg, torch.from_numpy(pi_a).cuda(), w_a)
    assert st == pkg.RPA_OK and abs(ec - ref_a[0]) < 1e-11
    # 1 + Pi not positive definite: reported, and the next call is clean
    nspd = pi_b.copy()
    nspd[2] -= 3.0 * np.eye(pi_b.shape[1])
    st, _, _ = _noalloc(pkg, nspd, w_b)
    assert st == pkg.RPA_ERR_NOT_SPD
    st, ec, eu = _noalloc(pkg, pi_b, w_b)
    assert st == pkg.RPA_OK and abs(ec - ref_b[0]) < 1e-11 and np.max(np.abs(eu - ref_b[1])) < 1e-10


def test_noalloc_on_a_caller_stream(pkg, handle):
    import torch
    pi, w = _case(505, 256, 4, 60, 6)
    ref = handle.ec_from_pi(pi, w)
    s = torch.cuda.Stream()
    d = torch.from_numpy(pi).cuda()
    torch.cuda.current_stream().synchronize()
    for _ in range(2):
        st, ec, eu = _noalloc(pkg, d, w, stream=ctypes.c_void_p(s.cuda_stream))
        assert st == pkg.RPA_OK
        assert abs(ec - ref[0]) < 1e-11 and np.max(np.abs(eu - ref[1])) < 1e-10


def test_noalloc_rejects_bad_arguments(pkg):
    lib = pkg.load_library()
    ec = ctypes.c_double()
    w = np.ones(1)
    pi = np.zeros((1, 4, 4))
    # NQ beyond 2^20 (its size would wrap a 64-bit count) and a negative device are argument errors
    st = lib.rpa_b200_ec_from_pi_noalloc(0, None, 1 << 62, 4, pi.ctypes.data, 1 << 62, w.ctypes.data,
                                         ctypes.byref(ec), None)
    assert st == pkg.RPA_ERR_INVALID_ARG
    st = lib.rpa_b200_ec_from_pi_noalloc(-1, None, 4, 1, pi.ctypes.data, 4, w.ctypes.data, ctypes.byref(ec), None)
    assert st == pkg.RPA_ERR_INVALID_ARG


def test_noalloc_rejects_problems_beyond_its_scratch(pkg):
    # 1 x 2100^2 doubles exceed the 32 MiB array: refused before any GPU work
    pi = np.zeros((1, 4, 4))
    lib = pkg.load_library()
    ec = ctypes.c_double()
    w = np.ones(1)
    st = lib.rpa_b200_ec_from_pi_noalloc(0, None, 2100, 1, pi.ctypes.data, 2100, w.ctypes.data,
                                         ctypes.byref(ec), None)
    assert st == pkg.RPA_ERR_TOO_LARGE
    assert b"size limit" in lib.rpa_b200_status_string(st)
