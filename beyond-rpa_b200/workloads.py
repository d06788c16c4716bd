"""Seeded synthetic RPA inputs with the shapes of the measured workloads.

There is no network and no SCF/Cholesky stack here, so inputs are synthetic:
occupied energies ~ U[occ_range], virtual energies log-uniform in virt_range,
R(Q, ai) ~ N(0,1) * scale * exp(-Q/decay), rescaled so that the largest
eigenvalue of Pi(0) equals `lam0` (a physical coupling strength).
R is generated on the GPU (torch) as a column-major (NQ, nov) view.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# name -> (NQ, NOcc, NVirt, K, generator kwargs)
SINGLE_SYSTEM = {
    # single-system split-BF16 vs FP64 workload: N_occ=64, N_virt=1024, NQ=4096, 16 points
    "single_4096": (4096, 64, 1024, 16, dict(occ_range=(-1.2, -0.3), virt_range=(0.02, 5.0), decay=512.0,
                                             scale=0.05, lam0=0.8)),
    # a quarter-size single system (NQ = 2048, nov = 16384): profiling case that fits an ncu capture
    "single_2048": (2048, 32, 512, 16, dict(occ_range=(-1.2, -0.3), virt_range=(0.02, 5.0), decay=256.0,
                                            scale=0.05, lam0=0.8)),
    # seeded twin of the water dimer (10 occ incl. 2 core, 72 virt, NQ = 400, 12 points)
    "water_dimer_twin": (400, 8, 72, 12, dict(occ_range=(-1.3, -0.4), virt_range=(0.03, 4.0), decay=50.0,
                                              scale=1.0, lam0=0.8)),
    # adjoint workload shapes
    "adjoint_2560": (2560, 48, 640, 16, dict(occ_range=(-1.3, -0.4), virt_range=(0.03, 4.0), decay=320.0,
                                             scale=1.0, lam0=0.8)),
    # CC path (direct-ring T2 + SOSEX + MBPT3 exchange) shapes, one scaled-down large case each
    "cc_1024": (1024, 32, 256, 12, dict(occ_range=(-1.3, -0.4), virt_range=(0.03, 4.0), decay=128.0,
                                        scale=1.0, lam0=0.8)),
    "cc_2048": (2048, 48, 512, 12, dict(occ_range=(-1.3, -0.4), virt_range=(0.03, 4.0), decay=256.0,
                                        scale=1.0, lam0=0.8)),
    # beyond-RPA large case shapes
    "large_8192": (8192, 128, 2048, 20, dict(occ_range=(-1.3, -0.4), virt_range=(0.03, 4.0), decay=1024.0,
                                             scale=1.0, lam0=0.8)),
}


@dataclass
class SyntheticSystem:
    R: object            # torch (NQ, nov) column-major view on the device, or numpy
    eps_o: np.ndarray
    eps_v: np.ndarray
    freqs: np.ndarray
    weights: np.ndarray

    @property
    def nq(self):
        return int(self.R.shape[0])


def orbital_energies(no, nv, seed, occ_range, virt_range):
    rng = np.random.default_rng(seed)
    eo = np.sort(rng.uniform(occ_range[0], occ_range[1], no))
    ev = np.sort(np.exp(rng.uniform(math.log(virt_range[0]), math.log(virt_range[1]), nv)))
    return eo, ev


def lambda_max_pi0(R, d, alpha=4.0, iters=40, seed=0):
    """Largest eigenvalue of Pi(0) = alpha R diag(1/D) R^T (power iteration, torch)."""
    import torch
    g = torch.Generator(device=R.device).manual_seed(seed)
    v = torch.randn(R.shape[0], generator=g, device=R.device, dtype=R.dtype)
    lam = 0.0
    for _ in range(iters):
        w = alpha * (R @ ((R.T @ v) / d))
        lam = float(torch.linalg.norm(w))
        v = w / lam
    return lam


def make_single_system(name="single_4096", seed=0, device="cuda", K=None):
    """Build one synthetic system on `device` with its optimised frequency grid."""
    import torch
    from . import freq_grid
    nq, no, nv, k_default, kw = SINGLE_SYSTEM[name]
    K = K or k_default
    eo, ev = orbital_energies(no, nv, seed, kw["occ_range"], kw["virt_range"])
    nov = no * nv
    g = torch.Generator(device=device).manual_seed(seed + 1)
    Rt = torch.randn((nov, nq), generator=g, device=device, dtype=torch.float64)  # (ai, Q) rows -> R = Rt.T
    Rt *= kw["scale"] * torch.exp(-torch.arange(nq, device=device, dtype=torch.float64) / kw["decay"])[None, :]
    R = Rt.T
    d = torch.from_numpy((ev[:, None] - eo[None, :]).reshape(-1, order="F")).to(device)
    lam = lambda_max_pi0(R, d)
    Rt *= math.sqrt(kw["lam0"] / lam)
    x, w = freq_grid(np.concatenate([eo, ev]), no, nv, nfixed=K)
    return SyntheticSystem(R=R, eps_o=eo, eps_v=ev, freqs=x, weights=w)


def mbe_specs(n_inst=512, seed=0):
    """(NOcc, NVirt, NQ, K) of every fragment of the many-body-expansion batch."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n_inst):
        no = int(rng.integers(16, 49))
        nv = int(round(rng.uniform(8.0, 12.0) * no))
        specs.append((no, nv, 4 * (no + nv), int(rng.choice([8, 12, 16]))))
    return specs


def make_mbe_batch(n_inst=512, seed=0, device="cuda", dimer_frac=0.6, only=None):
    """Many-body-expansion fragment batch: n_inst instances (dimer_frac dimers, the
    rest trimers) with NOcc ~ U{16..48}, NVirt = round(U[8,12] NOcc),
    NQ = 4 (NOcc + NVirt), K in {8, 12, 16}; each drawn like the water-dimer
    twin (occ U[-1.3,-0.4], virt log-U[0.03,4], R ~ N(0,1) exp(-Q/(NQ/8)),
    lambda_max(Pi(0)) = 0.8) from seed + instance id.  `only` restricts the
    materialised instances to a subset of ids (a rank's share).  Returns a
    list of (R, eps_o, eps_v, freqs, weights) and the dimer/trimer labels."""
    import torch
    from . import freq_grid
    specs = mbe_specs(n_inst, seed)
    ids = range(n_inst) if only is None else only
    out, kinds = [], []
    for i in ids:
        no, nv, nq, K = specs[i]
        eo, ev = orbital_energies(no, nv, seed + 7919 * (i + 1), (-1.3, -0.4), (0.03, 4.0))
        g = torch.Generator(device=device).manual_seed(seed + i + 1)
        Rt = torch.randn((no * nv, nq), generator=g, device=device, dtype=torch.float64)
        Rt *= torch.exp(-torch.arange(nq, device=device, dtype=torch.float64) / (nq / 8.0))[None, :]
        d = torch.from_numpy((ev[:, None] - eo[None, :]).reshape(-1, order="F")).to(device)
        lam = lambda_max_pi0(Rt.T, d, iters=25)
        Rt *= math.sqrt(0.8 / lam)
        x, w = freq_grid(np.concatenate([eo, ev]), no, nv, nfixed=K)
        out.append((Rt.T, eo, ev, x, w))
        kinds.append("dimer" if i < int(round(dimer_frac * n_inst)) else "trimer")
    return out, kinds
