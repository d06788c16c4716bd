"""Multi-GPU plumbing, one process per GPU.

* Independent systems (many-body-expansion fragments): dealt out to ranks by
  cost, each rank runs rpa_b200_ec_batched on its share, the energies are
  gathered once at the end; no data-path collective.
* One system over N GPUs: the ai columns are split over the ranks as the
  reference splits them over coarray images (rpa_OVSubsets,
  src/rpa/rpa_core_MO.f90:304-344, co_sum of Pi); here the partial Pi_k are
  reduce-scattered over the frequency index so the log-dets are distributed too.

Timings are reduced with MAX over ranks.
"""
from __future__ import annotations

import heapq

import numpy as np

import torch
import torch.distributed as dist


def instance_cost(nq, nov, nfreqs):
    """Work of one energy: Pi build (NQ^2 nov K) + log-det (NQ^3/3 K)."""
    return float(nq) * nq * nov * nfreqs + float(nq) ** 3 / 3.0 * nfreqs


def shard(costs, rank, world):
    """Indices owned by `rank`: longest-processing-time-first greedy over the
    costs (deterministic; ties broken by index), returned in ascending order."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    owner = [0] * len(costs)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + costs[i], r))
    return [i for i in range(len(costs)) if owner[i] == rank]


def max_over_ranks(x, device="cpu"):
    """MAX of a scalar over all ranks (identity without a process group)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_energies(local_ids, local_values, n_total, device="cpu"):
    """Full energy vector on every rank from each rank's (ids, values): one
    SUM all-reduce of a zero-padded vector (each id is owned by exactly one rank)."""
    t = torch.zeros(n_total, dtype=torch.float64, device=device)
    if len(local_ids):
        t[torch.as_tensor(list(local_ids), dtype=torch.long, device=device)] = torch.as_tensor(
            list(local_values), dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


# ----------------------------------------------------------------------------- one system over N GPUs
# The reference splits one system's ai range over coarray images (rpa_OVSubsets,
# src/rpa/rpa_core_MO.f90:304-344) and co_sums the partial Pi (rpa_GPiUG_MO,
# src/rpa/rpa_core_MO.f90:347-406).  Here each rank builds the partial Pi_k of an equal,
# contiguous ai-column range; one reduce-scatter over the frequency index leaves each rank
# the full Pi_k of K/N frequencies, whose log-dets it computes; one scalar all-reduce
# assembles E_c.  Pi and the log-det are both distributed.

def column_range(nov, rank, world):
    """Contiguous ai columns [c0, c1) of `rank` (equal split of nov)."""
    return nov * rank // world, nov * (rank + 1) // world


def column_pieces(c0, c1, nvirt):
    """Split the ai columns [c0, c1) (ai = a + NVirt i) into sub-instances, each a block of
    whole or partial occupied orbitals: list of (i0, i1, a0, a1, col0, col1) meaning
    occupied i0..i1-1 with virtual a0..a1-1, R columns col0..col1-1."""
    out = []
    c = c0
    while c < c1:
        i, a = divmod(c, nvirt)
        if a != 0 or c1 - c < nvirt:          # partial occupied block
            a1 = min(nvirt, a + (c1 - c))
            out.append((i, i + 1, a, a1, c, c + (a1 - a)))
            c += a1 - a
        else:                                  # run of whole occupied blocks
            i1 = i + (c1 - c) // nvirt
            out.append((i, i1, 0, nvirt, c, i1 * nvirt))
            c = i1 * nvirt
    return out


def _world(group):
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def partial_pi(pi_fn, R, eps_o, eps_v, freqs, rank, world, device="cuda"):
    """This rank's partial Pi_k (sum over its ai columns), zero-padded to a multiple of world
    frequencies: (ceil(K / world) * world, NQ, NQ).  pi_fn(R_cols, eps_o_slice, eps_v_slice,
    freqs, out) fills out (K, NQ, NQ) with the Pi_k of those columns."""
    nq = int(R.shape[0])
    no, nv, K = len(eps_o), len(eps_v), len(freqs)
    Kl = -(-K // world)
    pi = torch.zeros((Kl * world, nq, nq), dtype=torch.float64, device=device)
    c0, c1 = column_range(no * nv, rank, world)
    tmp = None
    for (i0, i1, a0, a1, col0, col1) in column_pieces(c0, c1, nv):
        if tmp is None:
            tmp = torch.empty((K, nq, nq), dtype=torch.float64, device=device)
        pi_fn(R[:, col0:col1], eps_o[i0:i1], eps_v[a0:a1], freqs, tmp)
        pi[:K] += tmp
    return pi


def energy_of_chunk(ec_fn, pi_chunk, weights, rank, world, K, device="cuda"):
    """E(u) of this rank's frequencies (rank*Kl .. rank*Kl+Kl-1, padding excluded) from the
    full Pi_k of those frequencies; returns a (Kl*world + 1) vector holding them and, last,
    their partial E_c (zeros elsewhere), ready for a SUM over ranks."""
    Kl = pi_chunk.shape[0]
    out = torch.zeros(Kl * world + 1, dtype=torch.float64, device=device)
    k0 = rank * Kl
    nreal = max(0, min(K, k0 + Kl) - k0)
    if nreal:
        w = np.asarray(weights, dtype=np.float64)[k0:k0 + nreal]
        ec_part, eu_part = ec_fn(pi_chunk[:nreal], w)
        out[k0:k0 + nreal] = torch.as_tensor(np.asarray(eu_part, dtype=np.float64), device=device)
        out[-1] = float(ec_part)
    return out


def ec_rpa_ai_split(pi_fn, ec_fn, R, eps_o, eps_v, freqs, weights, group=None, device="cuda"):
    """RPA E_c of one system whose ai columns are split over the ranks of `group`:
    partial Pi_k per rank, one reduce-scatter over frequencies, log-dets of the rank's
    frequencies, one SUM all-reduce.  Returns (E_c, E(u) of all K) on every rank.
    ec_fn(pi (k, NQ, NQ), weights (k)) returns (E_c, E(u)) of those frequencies."""
    rank, world = _world(group)
    K = len(freqs)
    pi = partial_pi(pi_fn, R, eps_o, eps_v, freqs, rank, world, device)
    Kl = pi.shape[0] // world
    if world > 1:
        mine = torch.empty((Kl,) + tuple(pi.shape[1:]), dtype=torch.float64, device=device)
        dist.reduce_scatter_tensor(mine, pi, op=dist.ReduceOp.SUM, group=group)
    else:
        mine = pi
    del pi
    vec = energy_of_chunk(ec_fn, mine, weights, rank, world, K, device)
    if world > 1:
        dist.all_reduce(vec, op=dist.ReduceOp.SUM, group=group)
    vec = vec.cpu().numpy()
    return float(vec[-1]), vec[:K]


def emulate_ai_split(pi_fn, ec_fn, R, eps_o, eps_v, freqs, weights, world, device="cuda"):
    """The ai-split path of `world` ranks run one after another in one process (the
    reduce-scatter becomes a sum of the ranks' partial Pi): for testing on one GPU."""
    K = len(freqs)
    total = None
    for r in range(world):
        p = partial_pi(pi_fn, R, eps_o, eps_v, freqs, r, world, device)
        total = p if total is None else total + p
    Kl = total.shape[0] // world
    vec = None
    for r in range(world):
        v = energy_of_chunk(ec_fn, total[r * Kl:(r + 1) * Kl], weights, r, world, K, device)
        vec = v if vec is None else vec + v
    vec = vec.cpu().numpy()
    return float(vec[-1]), vec[:K]
