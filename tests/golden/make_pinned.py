"""Oracle fixtures at the benchmarked configurations (pinned_golden.json).

    python tests/golden/make_pinned.py [single_4096] [adjoint_2560] [mbe_sample]

Runs the oracle (oracle/rpa_oracle.py, numpy + LAPACK) on the seeded inputs of
tests/golden/pinned.py and stores, per case, the rescale factor of R, the frequency grid, the
energies and (for the adjoint case) gradient samples and norms.  The inputs are rebuilt from
their seeds by the GPU tests; an R checksum guards against a changed generator.  Each case takes
one to a few minutes on 8 cores; a named subset updates only those entries.
"""
from __future__ import annotations

import json
import math
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import rpa_oracle as O  # noqa: E402
from tests.golden import pinned as P  # noqa: E402

OUT = Path(__file__).resolve().parent / "pinned_golden.json"


def rescale_factor(R, eo, ev, lam0=0.8):
    return math.sqrt(lam0 / O.lambda_max_pi0(R, O.dai(eo, ev)))


def checksum(Rt):
    return {"sum": float(Rt.sum(dtype=np.float64)), "sumsq": float(np.einsum("ij,ij->", Rt, Rt))}


def grid(eo, ev, K):
    s = O.RPASystem(R=np.zeros((1, len(eo) * len(ev))), eps_o=eo, eps_v=ev)
    return O.grid_for(s, K)


def make_single(name):
    K = P.SINGLE[name][3]
    Rt, eo, ev = P.single_system(name)
    f = rescale_factor(Rt.T, eo, ev)
    Rt *= f
    x, w = grid(eo, ev, K)
    t = time.time()
    pi = O.pi_matrices(Rt.T, eo, ev, x)
    ec, eu = O.ec_rpa_analytic(pi, w)
    # the same energy with a Cholesky log-det (LAPACK dpotrf): at these orders QR and Cholesky
    # differ by FP64 rounding (~1e-10 relative), which bounds how closely any FP64 path can agree
    ec_chol, eu_chol = O.ec_rpa_analytic(pi, w, logdet=O.logdet_cholesky)
    rec = dict(factor=f, freqs=x.tolist(), weights=w.tolist(), Ec=ec, Eu=eu.tolist(), Ec_cholesky=ec_chol,
               Eu_cholesky=eu_chol.tolist(), R=checksum(Rt), pi_trace=[math.fsum(np.diag(p).tolist()) for p in pi])
    print(f"{name}: Ec = {ec:.15f}, Cholesky log-det {ec_chol:.15f} ({time.time() - t:.0f} s)", flush=True)
    return rec


def make_adjoint(name):
    rec = make_single(name)
    Rt, eo, ev = P.single_system(name, rec["factor"])
    x, w = np.array(rec["freqs"]), np.array(rec["weights"])
    t = time.time()
    dR, do, dv = O.ec_grad(Rt.T, eo, ev, x, w)
    rng = np.random.default_rng(7)
    q = rng.integers(0, Rt.shape[1], 4096)
    ai = rng.integers(0, Rt.shape[0], 4096)
    rec.update(grad=dict(q=q.tolist(), ai=ai.tolist(), dR=dR[q, ai].tolist(), dR_max=float(np.max(np.abs(dR))),
                         dR_norm=float(np.linalg.norm(dR)), deps_o=do.tolist(), deps_v=dv.tolist()))
    print(f"{name}: gradient ({time.time() - t:.0f} s), max |dR| = {rec['grad']['dR_max']:.3e}", flush=True)
    return rec


def make_mbe_sample():
    out = {}
    for i in P.mbe_sample_ids():
        t = time.time()
        Rt, eo, ev, K = P.mbe_instance(i)
        f = rescale_factor(Rt.T, eo, ev)
        Rt *= f
        x, w = grid(eo, ev, K)
        nfrag = P.fragments(i)
        energies, energies_chol = [], []
        for frags in P.subsystems(nfrag):
            Rs, eos, evs = P.subsystem(Rt, eo, ev, frags, nfrag)
            pi = O.pi_matrices(Rs.T, eos, evs, x)
            energies.append(O.ec_rpa_analytic(pi, w)[0])
            energies_chol.append(O.ec_rpa_analytic(pi, w, logdet=O.logdet_cholesky)[0])
        eint = O.mbe_energy(nfrag, np.array(energies))
        out[str(i)] = dict(factor=f, freqs=x.tolist(), weights=w.tolist(), nfrag=nfrag, energies=energies,
                           Eint=eint, energies_cholesky=energies_chol,
                           Eint_cholesky=O.mbe_energy(nfrag, np.array(energies_chol)), R=checksum(Rt))
        print(f"mbe {i}: NQ={Rt.shape[1]} nov={Rt.shape[0]} K={K} frags={nfrag} Eint={eint:.3e} "
              f"({time.time() - t:.0f} s)", flush=True)
    return out


def main(names):
    data = json.loads(OUT.read_text()) if OUT.exists() else {}
    for name in names:
        if name == "single_4096":
            data[name] = make_single(name)
        elif name == "adjoint_2560":
            data[name] = make_adjoint(name)
        elif name == "mbe_sample":
            data[name] = make_mbe_sample()
        else:
            raise SystemExit(f"unknown case {name}")
        OUT.write_text(json.dumps(data, indent=1))


if __name__ == "__main__":
    main(sys.argv[1:] or ["single_4096", "adjoint_2560", "mbe_sample"])
