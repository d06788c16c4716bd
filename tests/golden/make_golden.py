"""Generate the committed golden fixtures of the oracle.

    python tests/golden/make_golden.py

The reference (Fortran 2008 + MKL + coarrays) cannot be compiled or run in
this environment and ships no outputs of its own, so these fixtures are
outputs of the oracle restatement (oracle/rpa_oracle.py), which the identity
tests in tests/test_oracle.py pin.  They freeze the oracle's numbers so that
both the oracle and the GPU path are checked against the same values.
Inputs are regenerated from their seeds (make_system is deterministic); a
checksum of R guards against silent generator changes.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import rpa_oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent

# name: (NQ, NOcc, NVirt, seed, kwargs, K or None (= optimise))
CASES = {
    # seeded twin of the water-dimer case: 10 occupied (2 frozen core), 72 virtual, NQ = 400, 12 points;
    # R rescaled so that lambda_max(Pi(0)) = 0.8 (a physical coupling strength)
    "water_dimer_twin": (400, 8, 72, 1234, dict(decay=50.0, ncore_orbs=2, lam0=0.8), 12),
    # ragged sizes: NQ not a multiple of any tile, nov = 185
    "ragged": (200, 5, 37, 7, dict(decay=40.0, lam0=0.6), 5),
    # tiny case with committed inputs
    "tiny": (40, 3, 10, 99, dict(decay=15.0, lam0=0.5), None),
    # large-gap system scaled as the single-system workload (smaller)
    "scaled_c2": (512, 16, 128, 2024, dict(occ_range=(-1.2, -0.3), virt_range=(0.02, 5.0), decay=64.0,
                                          scale=0.05, lam0=0.8), 16),
}


def system(name):
    nq, no, nv, seed, kw, K = CASES[name]
    s = O.make_system(nq, no, nv, seed, **kw)
    x, w = O.grid_for(s, K)
    return s, x, w


def main():
    meta = {}
    for name in CASES:
        s, x, w = system(name)
        pi = O.pi_matrices(s.R, s.eps_o, s.eps_v, x)
        ec, eu = O.ec_rpa_analytic(pi, w)
        rec = dict(NQ=s.nq, NOcc=s.no, NVirt=s.nv, freqs=x.tolist(), weights=w.tolist(), Ec=ec, Eu=eu.tolist(),
                   R_sum=float(s.R.sum()), R_sumsq=float((s.R ** 2).sum()),
                   pi_trace=[float(np.trace(p)) for p in pi], eps_o=s.eps_o.tolist(), eps_v=s.eps_v.tolist())
        if name == "tiny":
            rec["R"] = s.R.tolist()
            rec["pi"] = pi.tolist()
        meta[name] = rec
        print(f"{name}: NQ={s.nq} no={s.no} nv={s.nv} K={len(x)} Ec={ec:.12f}")
    (OUT / "oracle_golden.json").write_text(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
