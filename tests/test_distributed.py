"""World-size-2 gloo tests (CPU) of the multi-rank host logic of the batched
path: cost-balanced sharding, max-over-ranks timing and the energy gather."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT / "tests"))
    import conftest
    pkg = conftest.load_package()
    import importlib
    D = importlib.import_module("beyond_rpa_b200.distributed")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    rng = np.random.default_rng(0)
    costs = [D.instance_cost(int(rng.integers(700, 2300)), int(rng.integers(2000, 25000)), int(rng.choice([8, 12, 16])))
             for _ in range(40)]
    mine = D.shard(costs, rank, world)
    t = D.max_over_ranks(1.0 + rank)
    ec = D.gather_energies(mine, [-(i + 1) * 0.001 for i in mine], len(costs))
    q.put((rank, mine, t, ec.tolist(), sum(costs[i] for i in mine)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shard_timing_and_gather():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    owned = sorted(res[0][1] + res[1][1])
    assert owned == list(range(40))                       # every instance exactly once
    assert set(res[0][1]).isdisjoint(res[1][1])
    loads = [r[4] for r in res]
    assert max(loads) / min(loads) < 1.1                   # cost-balanced
    assert res[0][2] == res[1][2] == 2.0                   # max over ranks
    expect = [-(i + 1) * 0.001 for i in range(40)]
    assert np.allclose(res[0][3], expect) and np.allclose(res[1][3], expect)


def test_single_process_fallbacks():
    sys.path.insert(0, str(ROOT / "tests"))
    import conftest
    conftest.load_package()
    import importlib
    D = importlib.import_module("beyond_rpa_b200.distributed")
    assert D.shard([3.0, 1.0, 2.0], 0, 1) == [0, 1, 2]
    assert D.max_over_ranks(4.5) == 4.5
    assert np.allclose(D.gather_energies([0, 2], [1.0, 3.0], 3), [1.0, 0.0, 3.0])


# ----------------------------------------------------------------------------- one system split over ranks

def test_column_pieces_cover_each_column_once():
    sys.path.insert(0, str(ROOT / "tests"))
    import conftest
    conftest.load_package()
    import importlib
    D = importlib.import_module("beyond_rpa_b200.distributed")
    rng = np.random.default_rng(5)
    for _ in range(300):
        nv = int(rng.integers(1, 9))
        no = int(rng.integers(1, 7))
        world = int(rng.integers(1, 6))
        nov = no * nv
        seen = []
        for r in range(world):
            c0, c1 = D.column_range(nov, r, world)
            for (i0, i1, a0, a1, col0, col1) in D.column_pieces(c0, c1, nv):
                cols = [a + nv * i for i in range(i0, i1) for a in range(a0, a1)]
                assert cols == list(range(col0, col1))       # one contiguous block of R
                assert c0 <= col0 and col1 <= c1
                seen += cols
        assert sorted(seen) == list(range(nov))


def _split_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT / "tests"))
    sys.path.insert(0, str(ROOT))
    import conftest
    conftest.load_package()
    import importlib
    D = importlib.import_module("beyond_rpa_b200.distributed")
    from oracle import rpa_oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    s = O.make_system(50, 5, 13, 17, decay=12.0, lam0=0.7)
    x, w = O.grid_for(s, 7)                       # K = 7: padded to a multiple of world

    def pi_fn(Rc, eo, ev, fr, out):
        out.copy_(torch.from_numpy(O.pi_matrices(np.asarray(Rc), eo, ev, fr)))

    def ec_fn(pi, wk):
        return O.ec_rpa_analytic(pi.numpy(), wk)

    ec, eu = D.ec_rpa_ai_split(pi_fn, ec_fn, torch.from_numpy(s.R), s.eps_o, s.eps_v, x, w, device="cpu")
    q.put((rank, ec, list(eu)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ai_split_energy_equals_whole_system(world):
    sys.path.insert(0, str(ROOT))
    from oracle import rpa_oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    s = O.make_system(50, 5, 13, 17, decay=12.0, lam0=0.7)
    x, w = O.grid_for(s, 7)
    ref, ref_eu = O.ec_rpa(s.R, s.eps_o, s.eps_v, x, w)
    for _, ec, eu in res:
        assert abs(ec - ref) < 1e-12 and np.max(np.abs(np.array(eu) - ref_eu)) < 1e-12
