"""The N > 1 path on CPU: world_size-2 gloo ranks shard a batch, solve their shard (with the
oracle standing in for the device), gather the records on rank 0 and take the max of
their timings -- the result must equal the single-process solve."""
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


def _worker(rank, world, port, outdir):
    sys.path.insert(0, str(ROOT / "machinig-sim_b200"))
    sys.path.insert(0, str(ROOT / "oracle"))
    import torch.distributed as dist
    from datetime import timedelta

    import pyoracle as O
    from mcs import _abi as A
    from mcs import dist as D
    from mcs import workloads as W

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    wl = W.hetero(n=24)
    wl.opts.revs = 10
    wl.opts.iters = 3
    parts = D.shard(D.cost_estimate(wl), world)
    mine = parts[rank]
    setups = [A.Setup.from_buffer_copy(r.tobytes()) for r in wl.setups]
    modals = [A.Modal.from_buffer_copy(r.tobytes()) for r in wl.modals]
    pts = wl.points[mine]
    P = (A.Point * len(pts)).from_buffer_copy(pts.tobytes())
    res, _ = O.solve_batch(setups, modals, P, wl.opts, nthreads=1)
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


def test_two_rank_gloo_solve_matches_single_process(tmp_path, oracle):
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

    from mcs import _abi as A
    from mcs import workloads as W

    wl = W.hetero(n=24)
    wl.opts.revs = 10
    wl.opts.iters = 3
    setups = [A.Setup.from_buffer_copy(r.tobytes()) for r in wl.setups]
    modals = [A.Modal.from_buffer_copy(r.tobytes()) for r in wl.modals]
    P = (A.Point * wl.n).from_buffer_copy(wl.points.tobytes())
    ref, _ = oracle.solve_batch(setups, modals, P, wl.opts, nthreads=1)
    assert gathered.tobytes() == ref.tobytes()
