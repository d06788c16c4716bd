"""Seeded numpy inputs of the benchmarked configurations.

The fixtures in pinned_golden.json hold the oracle's energies (and gradient samples) for the
inputs these functions make; tests/test_gpu_pinned.py and bench.py regenerate the same inputs
bit for bit (numpy's PCG64 stream and its normal sampler are deterministic for a given seed) and
run the library on them.  Only scalars, samples and checksums are committed: the inputs
themselves (up to 2.15 GB) are rebuilt from their seeds.

Shapes and distributions are the workloads' (NQ, NOcc, NVirt, K; occupied energies uniform,
virtual energies log-uniform, R(Q, ai) ~ N(0, 1) * scale * exp(-Q / decay), rescaled so that the
largest eigenvalue of Pi(0) is 0.8).  The rescale factor comes from the oracle's power iteration
when the fixture is made and is stored with it, so regenerating an input needs no iteration.
"""
from __future__ import annotations

import math

import numpy as np

# single systems: name -> (NQ, NOcc, NVirt, K, occ range, virt range, decay, scale, seed)
SINGLE = {
    # the single-system split-BF16 vs FP64 workload (NQ = 4096, NOcc = 64, NVirt = 1024, 16 points)
    "single_4096": (4096, 64, 1024, 16, (-1.2, -0.3), (0.02, 5.0), 512.0, 0.05, 4096),
    # the adjoint workload (NQ = 2560, NOcc = 48, NVirt = 640, 16 points)
    "adjoint_2560": (2560, 48, 640, 16, (-1.3, -0.4), (0.03, 4.0), 320.0, 1.0, 2560),
}

# many-body-expansion sample: instance ids of the 512-fragment batch (the first 307 are dimers)
MBE_N_INST = 512
MBE_DIMERS = 307
MBE_SAMPLE_SEED = 512


def orbital_energies(no, nv, seed, occ_range, virt_range):
    rng = np.random.default_rng(seed)
    eo = np.sort(rng.uniform(occ_range[0], occ_range[1], no))
    ev = np.sort(np.exp(rng.uniform(math.log(virt_range[0]), math.log(virt_range[1]), nv)))
    return eo, ev


def raw_vectors(nq, nov, seed, scale, decay):
    """Rt (nov, nq), C order: R = Rt.T is the column-major (NQ, nov) matrix with ld = NQ."""
    rng = np.random.default_rng(seed)
    Rt = rng.standard_normal((nov, nq))
    Rt *= (scale * np.exp(-np.arange(nq) / decay))[None, :]
    return Rt


def single_system(name, factor=None, variant=0):
    """(Rt, eps_o, eps_v) of a single-system workload; Rt is multiplied by `factor` when given.
    variant > 0 draws another system of the same shape (other seeds; not pinned by a fixture)."""
    nq, no, nv, _, occ, virt, decay, scale, seed = SINGLE[name]
    seed += 100003 * variant
    eo, ev = orbital_energies(no, nv, seed, occ, virt)
    Rt = raw_vectors(nq, no * nv, seed + 1, scale, decay)
    if factor is not None:
        Rt *= factor
    return Rt, eo, ev


def mbe_sample_ids():
    """8 dimers and 8 trimers of the 512-fragment batch."""
    rng = np.random.default_rng(MBE_SAMPLE_SEED)
    dimers = sorted(int(i) for i in rng.choice(MBE_DIMERS, 8, replace=False))
    trimers = sorted(int(i) for i in rng.choice(np.arange(MBE_DIMERS, MBE_N_INST), 8, replace=False))
    return dimers + trimers


MBE_SEED = 4000  # the seed of the measured 512-fragment batch


def mbe_specs(n_inst=MBE_N_INST, seed=MBE_SEED):
    """(NOcc, NVirt, NQ, K) of every fragment of the many-body-expansion batch (the workload's)."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n_inst):
        no = int(rng.integers(16, 49))
        nv = int(round(rng.uniform(8.0, 12.0) * no))
        specs.append((no, nv, 4 * (no + nv), int(rng.choice([8, 12, 16]))))
    return specs


def mbe_instance(i, factor=None, seed=MBE_SEED):
    """(Rt, eps_o, eps_v, K) of instance i: its shape and orbital energies are the batch's; R is
    drawn with numpy from seed 1000003 + i."""
    no, nv, nq, K = mbe_specs(MBE_N_INST, seed)[i]
    eo, ev = orbital_energies(no, nv, seed + 7919 * (i + 1), (-1.3, -0.4), (0.03, 4.0))
    Rt = raw_vectors(nq, no * nv, 1000003 + i, 1.0, nq / 8.0)
    if factor is not None:
        Rt *= factor
    return Rt, eo, ev, K


def fragments(i):
    """Number of fragments of instance i (2 for a dimer, 3 for a trimer)."""
    return 2 if i < MBE_DIMERS else 3


# subsystems in the order of the many-body-expansion energy entry point: total, A, B[, C, AB, BC, AC]
def subsystems(nfrag):
    if nfrag == 2:
        return [(0, 1), (0,), (1,)]
    return [(0, 1, 2), (0,), (1,), (2,), (0, 1), (1, 2), (0, 2)]


def subsystem(Rt, eo, ev, frags, nfrag):
    """Fragment f owns the occupied and virtual orbitals whose index is f modulo nfrag; a
    subsystem keeps every Cholesky vector (the supersystem's basis, as the reference's MBE
    driver shares it) and the ai columns of its orbitals, in ai = a + NVirt i order.  Returns
    (Rt_sub (nov_sub, NQ), eps_o_sub, eps_v_sub)."""
    no, nv = len(eo), len(ev)
    occ = [i for i in range(no) if i % nfrag in frags]
    vir = [a for a in range(nv) if a % nfrag in frags]
    cols = np.array([a + nv * i for i in occ for a in vir], dtype=np.int64)
    return np.ascontiguousarray(Rt[cols]), eo[occ], ev[vir]
