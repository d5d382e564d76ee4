"""Ensemble partition over ranks: LPT bin packing on the members' cell
counts (every member once, balanced) and the final gather of per-member
records, on two gloo ranks on the host."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cms2d_b200 import cases
from cms2d_b200.partition import gather_results, lpt


def test_lpt_assigns_every_member_once_and_balances():
    specs = cases.ensemble_specs(64, seed=23)
    sizes = [s["nx"] * s["ny"] for s in specs]
    for nparts in (1, 2, 3, 4, 8):
        parts = lpt(sizes, nparts)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(64))
        loads = [sum(sizes[k] for k in p) for p in parts]
        lower = max(sum(sizes) / nparts, max(sizes))  # no partition beats this
        assert max(loads) <= 4.0 / 3.0 * lower + max(sizes), (nparts, loads)
        assert lpt(sizes, nparts) == parts  # deterministic
    # the greedy rule by hand: 5 -> part 0, 4 -> 1, 3 -> 1 (4 < 5), 3 -> 0 (5 < 7), 3 -> 1 (7 < 8)
    assert lpt([5, 4, 3, 3, 3], 2) == [[0, 3], [1, 2, 4]]


def test_ensemble_specs_match_built_members():
    specs = cases.ensemble_specs(6, seed=5, nmin=2000, nmax=6000)
    built = cases.ensemble_basins(6, seed=5, nmin=2000, nmax=6000, members=[1, 4])
    for c, k in zip(built, (1, 4)):
        assert c.name == specs[k]["name"] and c.grid.ncells == specs[k]["nx"] * specs[k]["ny"]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = cases.ensemble_specs(16, seed=3, nmin=1000, nmax=4000)
        parts = lpt([s["nx"] * s["ny"] for s in specs], world)
        mine = parts[rank]
        # a real member record: the basin's cells and mean bed, built on this rank only
        local = {k: {"rank": rank, "cells": c.grid.ncells, "zb_mean": float(np.mean(c.zb[: c.grid.ncells]))}
                 for k, c in zip(mine, cases.ensemble_basins(16, seed=3, nmin=1000, nmax=4000, members=mine))}
        got = gather_results(local)
        q.put((rank, mine, got))
    finally:
        dist.destroy_process_group()


def test_partition_and_gather_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    (r0, m0, g0), (r1, m1, g1) = out
    assert sorted(m0 + m1) == list(range(16)) and not set(m0) & set(m1)
    assert g0 == g1 and sorted(g0) == list(range(16))
    specs = cases.ensemble_specs(16, seed=3, nmin=1000, nmax=4000)
    for k, rec in g0.items():
        assert rec["rank"] == (0 if k in m0 else 1)
        assert rec["cells"] == specs[k]["nx"] * specs[k]["ny"]
