"""Sharded sweep host logic on CPU: sector assignment, and two gloo ranks reproducing the
single-process sweep exactly (the oracle stands in for the per-sector GPU evaluation)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from ftlm_extended_hubbard_b200 import HubbardParams
from ftlm_extended_hubbard_b200.sharding import assign_sectors, sector_costs, sharded_sweep

LAT = (3, 2, 1.0, -0.35, 5.75, 0.9, 0.0, 0.0)
R, M, SEED = 4, 20, 7
T = np.array([0.2, 0.5, 1.0, 2.0])
MU = np.array([-1.0, 0.5, 2.0, 4.0])


def test_assignment_covers_every_sector_once_and_balances():
    for n, world in [(8, 2), (12, 4), (16, 8), (6, 3)]:
        costs = sector_costs(n, 32, 100)
        parts = assign_sectors(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range((n + 1) ** 2))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-9
        assert parts == assign_sectors(costs, world)  # deterministic


def _oracle_eval(nu, nd, bts):
    import oracle as O
    s = O.OracleSector(*LAT, nu, nd)
    return s.ftlm(bts, R, M, SEED, mode=1, nthreads=1)


def _oracle_reduce(lnz_s, e_s, N, bts, mus, n):
    import oracle as O
    return O.gc_reduce(lnz_s, e_s, N, bts, mus, n)


def _worker(rank, world, port, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = HubbardParams(*LAT)
        lz, es, N, (g, nav, eav), mine = sharded_sweep(p, R, M, SEED, T, MU, evaluate=_oracle_eval,
                                                         reduce=_oracle_reduce)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), lz=lz, es=es, g=g, nav=nav, mine=np.array(mine))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_reproduce_the_single_process_sweep(tmp_path):
    import oracle as O
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    lz1, es1, N1, dims, (g1, n1, e1) = O.oracle_sweep(*LAT, R, M, SEED, 1.0 / T, MU, mode=1)
    mines = []
    for r in range(world):
        d = np.load(tmp_path / f"r{r}.npz")
        np.testing.assert_array_equal(d["lz"], lz1)
        np.testing.assert_array_equal(d["es"], es1)
        np.testing.assert_array_equal(d["g"], g1)
        np.testing.assert_array_equal(d["nav"], n1)
        mines.append(set(d["mine"].tolist()))
    assert not (mines[0] & mines[1]) and len(mines[0] | mines[1]) == lz1.shape[0]
