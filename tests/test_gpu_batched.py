"""GPU tests of the batched many-instance energy (rpa_b200_ec_batched):
every instance must match the single-system entry point and the FP64
oracle, and a dimer of non-interacting monomers must give a vanishing
interaction energy (size consistency, rpa_Eint2Body src/rpa/rpa_driver.f90:381-386).

Tolerances: FP64 1e-10 Eh per instance; split-BF16 1e-6 Eh per instance and
1e-7 Eh on the interaction energy.
"""
import numpy as np
import pytest

from oracle import rpa_oracle as O

pytestmark = pytest.mark.gpu


def systems(seed=100, n=7):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        no = int(rng.integers(3, 9))
        nv = int(round(rng.uniform(8, 12) * no))
        nq = 4 * (no + nv)
        K = int(rng.choice([8, 12, 16]))
        s = O.make_system(nq, no, nv, seed + i, decay=nq / 6.0, lam0=0.8)
        x, w = O.casimir_polder(K, 0.5 + 0.1 * i)
        out.append((s.R, s.eps_o, s.eps_v, x, w))
    return out


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("split", 1e-6)])
def test_batched_matches_single_and_oracle(handle, prec, tol):
    sys_ = systems()
    ec, eus = handle.ec_batched(sys_, prec=prec)
    import torch
    for (R, eo, ev, x, w), e, eu in zip(sys_, ec, eus):
        # device R: the single call runs the same one-shot arithmetic as the batched launch
        # (host R is staged in pieces whose contributions are summed in FP64 instead)
        Rd = torch.from_numpy(np.ascontiguousarray(R.T)).cuda().T
        single, single_eu = handle.ec_rpa(Rd, eo, ev, x, w, prec=prec)
        assert abs(e - single) < 1e-12
        ref, _ = O.ec_rpa(R, eo, ev, x, w)
        assert abs(e - ref) < tol
        assert np.max(np.abs(eu - single_eu)) < 1e-11


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("split", 1e-7)])
def test_batched_dimer_size_consistency(handle, prec, tol):
    a = O.make_system(120, 4, 26, 201, decay=30.0, lam0=0.6)
    b = O.make_system(96, 3, 29, 202, decay=25.0, lam0=0.6)
    eo = np.concatenate([a.eps_o, b.eps_o])
    ev = np.concatenate([a.eps_v, b.eps_v])
    no, nv = len(eo), len(ev)
    R = np.zeros((a.nq + b.nq, no * nv))
    for (s, q0, i0, a0) in ((a, 0, 0, 0), (b, a.nq, a.no, a.nv)):
        Rr = s.R.reshape(s.nq, s.nv, s.no, order="F")
        for i in range(s.no):
            R[q0:q0 + s.nq, a0 + nv * (i0 + i): a0 + nv * (i0 + i) + s.nv] = Rr[:, :, i]
    x, w = O.casimir_polder(12, 0.6)
    ec, _ = handle.ec_batched([(R, eo, ev, x, w), (a.R, a.eps_o, a.eps_v, x, w), (b.R, b.eps_o, b.eps_v, x, w)],
                              prec=prec)
    assert abs(O.eint_2body(ec[0], ec[1], ec[2])) < tol


def test_batched_repeated_call_uses_cached_graph(handle):
    sys_ = systems(seed=300, n=5)
    a, _ = handle.ec_batched(sys_, prec="split")
    b, _ = handle.ec_batched(sys_, prec="split")
    assert np.array_equal(a, b)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("split", 1e-7)])
def test_mbe_driver_dimer_of_noninteracting_monomers(handle, prec, tol):
    # the MBE driver (Handle.mbe_energies): shared grid over the dimer and its monomers, batched energies, Eint;
    # two non-interacting monomers (block-diagonal R) must give Eint ~ 0 on the shared grid
    a = O.make_system(110, 4, 26, 301, decay=30.0, lam0=0.6)
    b = O.make_system(90, 3, 28, 302, decay=25.0, lam0=0.6)
    eo = np.concatenate([a.eps_o, b.eps_o])
    ev = np.concatenate([a.eps_v, b.eps_v])
    order_o, order_v = np.argsort(eo), np.argsort(ev)
    no, nv = len(eo), len(ev)
    R = np.zeros((a.nq + b.nq, no * nv))
    pos_o, pos_v = np.argsort(order_o), np.argsort(order_v)  # position of each orbital in the sorted lists
    for (s, q0, i0, a0) in ((a, 0, 0, 0), (b, a.nq, a.no, a.nv)):
        Rr = s.R.reshape(s.nq, s.nv, s.no, order="F")
        for i in range(s.no):
            for aa in range(s.nv):
                col = pos_v[a0 + aa] + nv * pos_o[i0 + i]
                R[q0:q0 + s.nq, col] = Rr[:, aa, i]
    subsystems = [(R, eo[order_o], ev[order_v]), (a.R, a.eps_o, a.eps_v), (b.R, b.eps_o, b.eps_v)]
    ec, eint, x, w = handle.mbe_energies(subsystems, 2, prec=prec, nfixed=12)
    assert abs(eint) < tol
    for (Rs, eos, evs), e in zip(subsystems, ec):
        ref, _ = O.ec_rpa(Rs, eos, evs, x, w)
        assert abs(e - ref) < (1e-10 if prec == "fp64" else 1e-6)


def _dimer(seed_a, seed_b, occ, virt):
    a = O.make_system(60, 4, 26, seed_a, occ_range=occ, virt_range=virt, decay=20.0, lam0=0.6)
    b = O.make_system(50, 3, 28, seed_b, occ_range=occ, virt_range=virt, decay=18.0, lam0=0.6)
    eo = np.concatenate([a.eps_o, b.eps_o])
    ev = np.concatenate([a.eps_v, b.eps_v])
    order_o, order_v = np.argsort(eo), np.argsort(ev)
    pos_o, pos_v = np.argsort(order_o), np.argsort(order_v)
    no, nv = len(eo), len(ev)
    R = np.zeros((a.nq + b.nq, no * nv))
    for (s, q0, i0, a0) in ((a, 0, 0, 0), (b, a.nq, a.no, a.nv)):
        Rr = s.R.reshape(s.nq, s.nv, s.no, order="F")
        for i in range(s.no):
            for aa in range(s.nv):
                R[q0:q0 + s.nq, pos_v[a0 + aa] + nv * pos_o[i0 + i]] = Rr[:, aa, i]
    return [(R, eo[order_o], ev[order_v]), (a.R, a.eps_o, a.eps_v), (b.R, b.eps_o, b.eps_v)]


@pytest.mark.parametrize("prec", ["fp64", "split"])
def test_batched_instances_beyond_16_frequencies(handle, prec):
    # up to 64 points per instance (the reference's limit): such instances run as groups of 16
    import torch
    sys_ = []
    for i, K in enumerate((40, 17, 12, 64)):
        s = O.make_system(96 + 16 * i, 3, 30, 500 + i, decay=20.0, lam0=0.7)
        x, w = O.casimir_polder(K, 0.6)
        sys_.append((s.R, s.eps_o, s.eps_v, x, w))
    ec, eus = handle.ec_batched(sys_, prec=prec)
    for (R, eo, ev, x, w), e, eu in zip(sys_, ec, eus):
        assert len(eu) == len(x)
        Rd = torch.from_numpy(np.ascontiguousarray(R.T)).cuda().T
        single, single_eu = handle.ec_rpa(Rd, eo, ev, x, w, prec=prec)
        assert abs(e - single) < 1e-12 and np.max(np.abs(eu - single_eu)) < 1e-11
        ref, _ = O.ec_rpa(R, eo, ev, x, w)
        assert abs(e - ref) < (1e-10 if prec == "fp64" else 1e-6)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("split", 1e-7)])
def test_mbe_driver_optimised_grid_beyond_16_points(handle, pkg, prec, tol):
    # nfixed = 0: the shared grid is optimised to the targets; this wide spectrum needs 23 points
    subsystems = _dimer(301, 302, (-3.0, -0.1), (0.02, 100.0))
    ec, eint, x, w = handle.mbe_energies(subsystems, 2, prec=prec)
    assert len(x) > 16
    assert abs(eint) < tol
    for (Rs, eos, evs), e in zip(subsystems, ec):
        ref, _ = O.ec_rpa(Rs, eos, evs, x, w)
        assert abs(e - ref) < (1e-10 if prec == "fp64" else 1e-6)


def test_mbe_driver_shared_pi_basis(handle):
    # basis="eigen": one compressed Pi basis from the whole system at the grid's lowest frequency,
    # shared by every subsystem (the reference's THC_ZgkPiU); the energies equal piu_basis +
    # project_basis + the single-system path done by hand
    import torch
    from tests.golden import pinned as P
    s = O.make_system(240, 8, 40, 611, decay=40.0, lam0=0.7)
    Rt = np.ascontiguousarray(s.R.T)
    subs = []
    for frags in P.subsystems(2):
        Rs, eos, evs = P.subsystem(Rt, s.eps_o, s.eps_v, frags, 2)
        subs.append((np.asfortranarray(Rs.T), eos, evs))
    ec, eint, x, w = handle.mbe_energies(subs, 2, prec="fp64", nfixed=10, basis="eigen", basis_target_error=1e-4)
    G, _, _ = handle.piu_basis(subs[0][0], subs[0][1], subs[0][2], float(x[0]), target_error=1e-4, basis="eigen")
    assert G.shape[1] < 240  # the basis is compressed
    for (Rs, eos, evs), e in zip(subs, ec):
        Rp = handle.project_basis(G, Rs)
        ref, _ = handle.ec_rpa(torch.from_numpy(np.ascontiguousarray(Rp.T)).cuda().T, eos, evs, x, w, prec="fp64")
        assert abs(e - ref) < 1e-12
    assert abs(eint - pkg_mbe(ec)) < 1e-14
    with pytest.raises(ValueError):  # subsystems over different Cholesky vectors cannot share a basis
        handle.mbe_energies(_dimer(301, 302, (-1.3, -0.4), (0.03, 4.0)), 2, nfixed=8, basis="eigen")


def pkg_mbe(ec):
    return O.eint_2body(ec[0], ec[1], ec[2])


def test_mbe_beyond_rpa_shares_the_t2_threshold(handle):
    # the whole system fixes the T2 cutoff threshold and every subsystem reuses it.  For two
    # non-interacting monomers the RPA interaction energy vanishes to rounding; the SOSEX one only
    # to the accuracy of the range finder's retained subspace (its Gram cutoff drops near-null
    # directions of I differently in the dimer and in the monomers: the oracle's range finder gives
    # -3.7e-7 Eh on this dimer, whose exchange energy is 3.2e-2 Eh)
    subs = _dimer(321, 322, (-1.3, -0.4), (0.03, 4.0))
    r = handle.mbe_beyond_rpa(subs, 2, prec="fp64", nfixed=10, cutoff_thresh=1e-4)
    assert r["common_thresh"] == 1e-4
    assert abs(r["eint"]) < 1e-11 and abs(r["ex_int"]) < 1e-4 * abs(r["ex"][0])
    # the dimer keeps the monomers' amplitudes (an eigenvalue at the threshold may fall either way)
    assert abs(r["nt"][0] - (r["nt"][1] + r["nt"][2])) <= 1
    # each subsystem's exchange energy is the plain T2 + SOSEX chain at the shared threshold
    x, w = r["freqs"], r["weights"]
    for (R, eo, ev), ex in zip(subs[1:], r["ex"][1:]):
        t2 = handle.dring_t2(R, eo, ev, x, w, prec="fp64", seed=0, common_thresh=r["common_thresh"])
        assert abs(handle.exchange_sosex(R, len(eo), len(ev), t2["U"], t2["A"], prec="fp64") - ex) < 1e-13
