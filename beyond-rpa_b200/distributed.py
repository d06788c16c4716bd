"""Multi-GPU plumbing of the batched path: one process per GPU, no data-path
collective.  Independent systems (many-body-expansion fragments) are dealt
out to ranks by cost; each rank runs rpa_b200_ec_batched on its share; the
energies are gathered once at the end and timings are reduced with MAX.

The reference distributes work over Fortran coarray images (the virtual-index
split of rpa_OVSubsets, src/rpa/rpa_core_MO.f90:304-344, with co_sum of Pi);
whole fragments need no reduction of Pi at all, so none is done here.
"""
from __future__ import annotations

import heapq

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
