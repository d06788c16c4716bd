"""GPU tests of the FP64 log-det tile plans and the tile tuner, and of the
pipelined batched launch (the next batch's scale/split pass beside this
batch's log-det; log-det order buckets on parallel branches).

A plan changes only the blocking of the Cholesky, not its arithmetic per
element beyond summation order: energies under every plan agree with the
default plan to 1e-12 relative and with the FP64 oracle to 1e-10 Eh.
Batching changes no arithmetic at all: energies are bit-identical.
"""
import os

import numpy as np
import pytest

from oracle import rpa_oracle as O

pytestmark = pytest.mark.gpu

CANDIDATES = [(128, 64), (256, 64), (512, 64), (128, 128), (256, 128), (512, 128)]


def test_tuner_picks_a_candidate_and_stores_it(pkg):
    with pkg.Handle(0) as h:
        assert h.logdet_plan(600) == (256, 64)  # default before tuning
        best, ms = h.tune_logdet(600, 24)
        assert best in CANDIDATES
        assert set(ms) == set(CANDIDATES) and all(t > 0 for t in ms.values())
        assert min(ms, key=ms.get) == best
        assert h.logdet_plan(600) == best
        assert h.logdet_plan(513) == best and h.logdet_plan(768) == best  # same bucket of 256 orders
        assert h.logdet_plan(900) == (256, 64)  # another bucket is untouched


def test_set_logdet_plan_validates(pkg):
    with pkg.Handle(0) as h:
        h.set_logdet_plan(1000, 512, 128)
        assert h.logdet_plan(1000) == (512, 128)
        for nb2, tile in ((192, 64), (256, 96), (0, 64), (1024, 64)):
            with pytest.raises(pkg.RPAError):
                h.set_logdet_plan(1000, nb2, tile)
        assert h.logdet_plan(1000) == (512, 128)


@pytest.mark.parametrize("prec", ["fp64", "split"])
def test_every_plan_gives_the_same_energy(pkg, prec):
    # NQ = 700 crosses two 256-column outer blocks and a ragged last panel under every plan
    s = O.make_system(700, 6, 60, 31, decay=110.0, lam0=0.8)
    x, w = O.casimir_polder(10, 0.7)
    ref, _ = O.ec_rpa(s.R, s.eps_o, s.eps_v, x, w)
    energies = {}
    with pkg.Handle(0) as h:
        h.set_autotune(False)
        for nb2, tile in CANDIDATES:
            h.set_logdet_plan(700, nb2, tile)
            ec, _ = h.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec=prec)
            energies[(nb2, tile)] = ec
            (eb,), _ = h.ec_batched([(s.R, s.eps_o, s.eps_v, x, w)], prec=prec)
            if prec == "fp64":
                assert abs(ec - ref) < 1e-10
                assert abs(eb - ref) < 1e-10
            else:
                assert abs(ec - ref) < 1e-6
                assert abs(eb - ref) < 1e-6
    base = energies[(256, 64)]
    for plan, ec in energies.items():
        assert abs(ec - base) <= 1e-12 * abs(base), plan


def _fragments(seed=300, n=9):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        no = int(rng.integers(3, 10))
        nv = int(round(rng.uniform(8, 12) * no))
        nq = 4 * (no + nv)  # 176 .. 520: three order buckets
        K = int(rng.choice([8, 12]))
        s = O.make_system(nq, no, nv, seed + i, decay=nq / 6.0, lam0=0.8)
        x, w = O.casimir_polder(K, 0.5 + 0.05 * i)
        out.append((s.R, s.eps_o, s.eps_v, x, w))
    return out


@pytest.mark.parametrize("prec", ["fp64", "split"])
def test_pipelined_batches_are_bit_identical(pkg, prec, monkeypatch):
    sys_ = _fragments()
    with pkg.Handle(0) as h:
        h.set_autotune(False)
        one, eu1 = h.ec_batched(sys_, prec=prec)
    # a 24 MB budget splits the fragments into several batches (pipelined graph)
    monkeypatch.setenv("RPA_B200_BATCH_BYTES", str(24 << 20))
    with pkg.Handle(0) as h:
        h.set_autotune(False)
        many, eu2 = h.ec_batched(sys_, prec=prec)
        again, _ = h.ec_batched(sys_, prec=prec)  # cached graph
    assert np.array_equal(one, many) and np.array_equal(many, again)
    for a, b in zip(eu1, eu2):
        assert np.array_equal(a, b)
    for (R, eo, ev, x, w), e in zip(sys_, many):
        ref, _ = O.ec_rpa(R, eo, ev, x, w)
        assert abs(e - ref) < (1e-10 if prec == "fp64" else 1e-6)


def test_batched_autotune_tunes_each_bucket_once(pkg):
    sys_ = _fragments(seed=400, n=6)
    orders = sorted({int(R.shape[0]) for R, *_ in sys_})
    with pkg.Handle(0) as h:
        h.set_autotune(False)
        off, _ = h.ec_batched(sys_, prec="split")
        assert all(h.logdet_plan(n) == (256, 64) for n in orders)
    with pkg.Handle(0) as h:
        on, _ = h.ec_batched(sys_, prec="split")
        plans = {n: h.logdet_plan(n) for n in orders}
        assert all(p in CANDIDATES for p in plans.values())
        n_first = h.launches()
        again, _ = h.ec_batched(sys_, prec="split")
        assert h.launches() < n_first  # no tuning the second time
        assert np.array_equal(on, again)
    for a, b in zip(on, off):
        assert abs(a - b) <= 1e-12 * abs(b)


@pytest.mark.parametrize("prec", ["fp64", "split"])
def test_lookahead_schedule_is_bit_identical(pkg, prec, monkeypatch):
    # the lookahead splits each trailing update into two launches over disjoint columns: every
    # element takes the same products in the same order, so energies must not move at all
    s = O.make_system(1100, 6, 60, 41, decay=180.0, lam0=0.8)  # five 256-column outer blocks
    x, w = O.casimir_polder(8, 0.7)
    sys_ = _fragments(seed=500, n=5) + [(s.R, s.eps_o, s.eps_v, x, w)]
    out = {}
    for la in ("0", "1"):
        monkeypatch.setenv("RPA_B200_LOOKAHEAD", la)
        with pkg.Handle(0) as h:
            h.set_autotune(False)
            ec, eu = h.ec_rpa(s.R, s.eps_o, s.eps_v, x, w, prec=prec)
            eb, _ = h.ec_batched(sys_, prec=prec)
            out[la] = (ec, eu, eb)
    assert out["0"][0] == out["1"][0]
    assert np.array_equal(out["0"][1], out["1"][1])
    assert np.array_equal(out["0"][2], out["1"][2])
    ref, _ = O.ec_rpa(s.R, s.eps_o, s.eps_v, x, w)
    assert abs(out["1"][0] - ref) < (1e-10 if prec == "fp64" else 1e-6)


@pytest.mark.parametrize("digits", ["7", "8"])
def test_int8_trailing_updates_match_the_dmma_log_det(pkg, monkeypatch, digits):
    # opt-in int8 tensor-core trailing updates (digit planes, exact integer products, FP64
    # recombination): E(u) equal to the DMMA updates' to 1e-13 relative, for the lookahead and the
    # plain schedule (which are bit-identical to each other), with a ragged last panel (order 1100)
    import torch
    s = O.make_system(1100, 10, 90, 77, decay=140.0, lam0=0.8)
    x, w = O.grid_for(s, 6)
    with pkg.Handle(0) as h0:
        pi = torch.from_numpy(h0.pi_u(s.R, s.eps_o, s.eps_v, x, prec="fp64")).cuda()
        h0.set_autotune(False)
        _, ref = h0.ec_from_pi(pi, w)
    out = []
    for la in ("1", "0"):
        monkeypatch.setenv("RPA_B200_OZAKI_SLICES", digits)
        monkeypatch.setenv("RPA_B200_LOOKAHEAD", la)
        with pkg.Handle(0) as h:
            h.set_autotune(False)
            _, eu = h.ec_from_pi(pi, w)
        out.append(eu)
        assert np.max(np.abs(eu - ref) / np.abs(ref)) < 1e-13
    assert np.array_equal(out[0], out[1])
