"""CPU checks of the seeded synthetic workloads bench.py measures: shapes, seeding, the dimer /
trimer split and the algorithmic work the measurements divide by (no GPU needed)."""
import numpy as np


def test_mbe_512_batch_definition(pkg):
    from beyond_rpa_b200.workloads import mbe_specs
    sp = mbe_specs(512, seed=4000)  # the batch bench.py --workload mbe_512 runs
    assert len(sp) == 512 and sp == mbe_specs(512, seed=4000)
    for no, nv, nq, K in sp:
        assert 16 <= no <= 48 and 8 * no - 1 <= nv <= 12 * no + 1
        assert nq == 4 * (no + nv) and K in (8, 12, 16)
    pi = sum(K * nq * nq * no * nv for no, nv, nq, K in sp)  # lower-triangle SYRK flops
    ld = sum(K * nq ** 3 / 3 for no, nv, nq, K in sp)        # Cholesky flops
    assert abs(pi / 1.89e14 - 1) < 0.01 and abs(ld / 7.1e12 - 1) < 0.01


def test_mbe_batch_labels_and_shapes(pkg):
    from beyond_rpa_b200.workloads import make_mbe_batch, mbe_specs
    systems, kinds = make_mbe_batch(5, seed=0, device="cpu")
    assert kinds == ["dimer"] * 3 + ["trimer"] * 2  # round(0.6 * 5) dimers first
    for (R, eo, ev, x, w), (no, nv, nq, K) in zip(systems, mbe_specs(5, seed=0)):
        assert R.shape == (nq, no * nv) and len(eo) == no and len(ev) == nv and len(x) == len(w) == K
        assert eo.max() < ev.min()


def test_single_system_is_normalised(pkg, oracle):
    from beyond_rpa_b200.workloads import make_single_system
    s = make_single_system("water_dimer_twin", seed=0, device="cpu")
    assert s.R.shape == (400, 8 * 72) and len(s.freqs) == 12 and np.all(np.diff(s.freqs) > 0)
    # R is rescaled so that the largest eigenvalue of Pi(0) is 0.8 (power iteration: to ~2 %)
    lam = np.linalg.eigvalsh(oracle.pi_matrices(s.R.numpy(), s.eps_o, s.eps_v, np.zeros(1))[0]).max()
    assert abs(lam - 0.8) < 0.02


def test_pinned_mbe_sample_is_drawn_from_the_measured_batch(pkg):
    # the oracle-pinned fragments have the shapes, frequency counts and orbital energies of the
    # measured 512-fragment batch (only R is drawn with numpy instead of on the GPU)
    from beyond_rpa_b200.workloads import mbe_specs, orbital_energies
    from tests.golden import pinned as P
    assert P.mbe_specs() == mbe_specs(512, seed=4000)
    ids = P.mbe_sample_ids()
    assert len(ids) == 16 and sum(i < P.MBE_DIMERS for i in ids) == 8
    i = min(ids, key=lambda j: P.mbe_specs()[j][2])  # the smallest sampled fragment
    no, nv, nq, K = mbe_specs(512, seed=4000)[i]
    eo, ev = orbital_energies(no, nv, 4000 + 7919 * (i + 1), (-1.3, -0.4), (0.03, 4.0))
    Rt, peo, pev, pK = P.mbe_instance(i)
    assert np.array_equal(eo, peo) and np.array_equal(ev, pev) and pK == K and Rt.shape == (no * nv, nq)


def test_pinned_subsystems_partition_the_columns():
    from tests.golden import pinned as P
    rng = np.random.default_rng(3)
    no, nv, nq = 5, 7, 4
    Rt = rng.standard_normal((no * nv, nq))
    eo, ev = np.sort(rng.uniform(-1, -0.5, no)), np.sort(rng.uniform(0.5, 1, nv))
    for nfrag in (2, 3):
        subs = P.subsystems(nfrag)
        full, _, _ = P.subsystem(Rt, eo, ev, subs[0], nfrag)
        assert np.array_equal(full, Rt)
        singles = [P.subsystem(Rt, eo, ev, (f,), nfrag) for f in range(nfrag)]
        assert sum(s[0].shape[0] for s in singles) < Rt.shape[0]  # cross-fragment pairs belong to no monomer
        for Rs, eos, evs in singles:
            assert Rs.shape == (len(eos) * len(evs), nq)
            # column a + nv_s i of the subsystem is the supersystem column of the same orbitals
            i, a = len(eos) - 1, len(evs) - 1
            gi, ga = int(np.flatnonzero(eo == eos[i])[0]), int(np.flatnonzero(ev == evs[a])[0])
            assert np.array_equal(Rs[a + len(evs) * i], Rt[ga + nv * gi])
