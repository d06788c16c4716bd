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
