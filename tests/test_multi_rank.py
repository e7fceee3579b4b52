"""The N > 1 path on CPU: world_size-2 gloo ranks take their shard from the library's split
(mcs_shard, host code), solve it (a stand-in solver that stamps each record with its point,
so that any loss or misplacement shows), gather the records on rank 0 and take the max of
their timings -- rank 0 must hold every point's record in input order.
"""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def fake_solve(points, idx):
    """Result records that identify their point: alim = S / 1000, trials = the index."""
    from mcs import _abi as A

    r = np.zeros(len(idx), dtype=A.RESULT_DTYPE)
    r["alim"] = points["S"][idx] / 1000.0
    r["trials"] = idx
    r["status"] = 0
    return r


def _worker(rank, world, port, outdir):
    sys.path.insert(0, str(ROOT / "machinig-sim_b200"))
    import torch.distributed as dist
    from datetime import timedelta

    from mcs import dist as D
    from mcs import workloads as W

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    wl = W.hetero(n=97)
    mine = D.library_shards(wl, world)[rank]
    res = fake_solve(wl.points, mine)
    full = D.gather_results(mine, res, wl.n, dist)
    t = D.max_over_ranks(float(rank + 1), dist)
    if rank == 0:
        np.save(os.path.join(outdir, "gathered.npy"), full)
        np.save(os.path.join(outdir, "tmax.npy"), np.array([t]))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_balances_cost():
    from mcs import dist as D

    cost = np.array([10, 1, 1, 1, 1, 1, 1, 1, 1, 1, 9], dtype=float)
    parts = D.shard(cost, 2)
    loads = [cost[p].sum() for p in parts]
    assert sorted(np.concatenate(parts).tolist()) == list(range(len(cost)))
    assert abs(loads[0] - loads[1]) <= 1


def test_cost_estimate_tracks_steps_per_tooth():
    from mcs import dist as D
    from mcs import workloads as W

    wl = W.sweep(n_speeds=64)
    c = D.cost_estimate(wl)
    # lower speed -> longer tooth period -> more steps per tooth
    assert c[0] > c[-1]


def test_library_split_is_balanced_and_complete():
    """mcs_shard: every point in exactly one shard, deterministic, and a longest-first
    greedy split: no shard's load exceeds the lightest by more than one point's cost."""
    import mcs
    from mcs import workloads as W

    wl = W.hetero(n=500, first_seed=123)
    for world in (1, 2, 3, 8):
        of, cost = mcs.shard(wl.setups, wl.modals, wl.points, wl.opts, world)
        assert of.min() >= 0 and of.max() < world and len(of) == wl.n
        loads = np.array([cost[of == r].sum() for r in range(world)])
        assert loads.max() - loads.min() <= cost.max() + 1e-9 * loads.max()
        of2, _ = mcs.shard(wl.setups, wl.modals, wl.points, wl.opts, world)
        assert np.array_equal(of, of2)
    # the cost follows the work: a slow speed of the sweep costs more than a fast one
    sw = W.sweep(n_speeds=64)
    _, c = mcs.shard(sw.setups, sw.modals, sw.points, sw.opts, 2)
    assert c[0] > c[-1]


def test_two_rank_gloo_gather_restores_input_order(tmp_path):
    world = 2
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    gathered = np.load(tmp_path / "gathered.npy")
    assert float(np.load(tmp_path / "tmax.npy")[0]) == 2.0

    from mcs import workloads as W

    wl = W.hetero(n=97)
    ref = fake_solve(wl.points, np.arange(wl.n))
    assert gathered.tobytes() == ref.tobytes()
