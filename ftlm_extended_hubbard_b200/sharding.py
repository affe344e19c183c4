"""Grand-canonical sweep sharded over ranks (one process per GPU, torch.distributed).

Sectors are independent units: a rank runs whole (N_up, N_dn) sectors and no vector ever crosses
ranks.  The only exchange is one all_reduce (sum) of the per-sector FP64 table [n_sec][2][n_T]
(ln Z_s and E_s; zeros where a rank did not run the sector), after which every rank holds the full
table and forms the (T, mu) grid.  Sectors are assigned by longest-processing-time-first on a cost
model (state count x chains x steps, plus a fixed per-step launch cost), deterministic for a given
(lattice, R, M, world size).  Reference: the sector loop of benchmarks/bench_ftlm_nmu_rect.cpp:138-219.
"""
from __future__ import annotations

from math import comb
from typing import Callable, Optional, Sequence

import numpy as np
import torch
import torch.distributed as dist

# Fixed cost of one chain step in state-equivalents (kernel launches and the per-step host sync).
STEP_OVERHEAD_STATES = 20000


def sector_costs(n_sites: int, R: int, M: int) -> list[float]:
    out = []
    for nu in range(n_sites + 1):
        for nd in range(n_sites + 1):
            dim = comb(n_sites, nu) * comb(n_sites, nd)
            steps = min(M, 2 * dim) * R
            out.append(float(steps) * (dim + STEP_OVERHEAD_STATES))
    return out


def assign_sectors(costs: Sequence[float], world: int) -> list[list[int]]:
    """LPT: sectors by descending cost (index breaks ties), each to the least-loaded rank
    (lowest rank breaks ties).  Returns the sector indices of every rank, ascending."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def _gpu_evaluate(p, R, M, seed, method, start):
    from .api import Sector

    def ev(nu, nd, bts):
        s = Sector(p, nu, nd)
        if method == "batched":
            return s.batched_ftlm(bts, R, M, seed)
        return s.ftlm(bts, R, M, seed, start=start)
    return ev


def _gpu_reduce(lnz_s, e_s, N, bts, mus, n_sites):
    import ctypes as C

    from ._lib import call
    g = [np.zeros((bts.size, mus.size)) for _ in range(3)]
    Ni = np.ascontiguousarray(N, np.int32)
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    call("ftlm_gpu_gc_reduce", P(lnz_s), P(e_s), P(Ni), Ni.size, P(bts), bts.size, P(mus), mus.size, n_sites,
         P(g[0]), P(g[1]), P(g[2]))
    return tuple(g)


def sharded_sweep(p, R: int, M: int, seed: int, temperatures, mus, method: str = "batched",
                  start: str = "philox", group=None,
                  evaluate: Optional[Callable] = None, reduce: Optional[Callable] = None):
    """Every sector of lattice p on this rank's share, then the full (T, mu) grid on every rank.

    evaluate(nu, nd, betas) -> (lnz[n_T], e[n_T]) and reduce(lnz_s, e_s, N, betas, mus, n_sites) ->
    (lnz_gc, n_avg, e_avg) default to the GPU library.  Returns (lnz_s, e_s, N, (lnz_gc, n_avg, e_avg),
    this rank's sector indices)."""
    n = p.Lx * p.Ly
    bts = np.ascontiguousarray(1.0 / np.atleast_1d(np.asarray(temperatures, np.float64)))
    mus = np.ascontiguousarray(np.atleast_1d(np.asarray(mus, np.float64)))
    rank, world = 0, 1
    if dist.is_available() and dist.is_initialized():
        rank, world = dist.get_rank(group), dist.get_world_size(group)
    mine = assign_sectors(sector_costs(n, R, M), world)[rank]
    ev = evaluate or _gpu_evaluate(p, R, M, seed, method, start)
    nsec = (n + 1) ** 2
    table = np.zeros((nsec, 2, bts.size))
    for idx in mine:
        nu, nd = divmod(idx, n + 1)
        lz, e = ev(nu, nd, bts)
        table[idx, 0] = lz
        table[idx, 1] = e
    if world > 1:
        backend = dist.get_backend(group)
        dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        t = torch.from_numpy(table).to(dev)
        # -inf (empty sectors) cannot be summed: ship exp-free placeholders and a mask
        finite = torch.isfinite(t)
        t = torch.where(finite, t, torch.zeros_like(t))
        owned = torch.zeros(nsec, dtype=torch.float64, device=dev)
        owned[list(mine)] = 1.0
        bad = (~finite).to(torch.float64)
        dist.all_reduce(t, group=group)
        dist.all_reduce(bad, group=group)
        dist.all_reduce(owned, group=group)
        if not bool(torch.all(owned == 1.0)):
            raise RuntimeError("sector assignment does not cover every sector exactly once")
        t = torch.where(bad > 0, torch.full_like(t, -float("inf")), t)
        table = t.cpu().numpy()
        table[:, 1][~np.isfinite(table[:, 1])] = 0.0
    lnz_s = np.ascontiguousarray(table[:, 0])
    e_s = np.ascontiguousarray(table[:, 1])
    N = np.array([nu + nd for nu in range(n + 1) for nd in range(n + 1)], np.int32)
    red = reduce or _gpu_reduce
    return lnz_s, e_s, N, red(lnz_s, e_s, N, bts, mus, n), mine
