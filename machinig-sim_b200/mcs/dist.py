"""Multi-GPU: one process per GPU, points sharded with no exchange on the data path.

Every boundary point is independent, so N GPUs split a batch into cost-balanced shards
(largest first, each point to the least-loaded rank), solve their shard on their own
device and meet only to gather the small result records (48-56 bytes per point) and to
take the max of their timings.  torch.distributed is the plumbing (NCCL on GPUs, gloo on
CPU); there is no collective inside any kernel.
"""
from __future__ import annotations

import heapq

import numpy as np

from . import _abi as A


def cost_estimate(workload) -> np.ndarray:
    """Relative cost of each point: steps per trial ~ steps_per_tooth * N; steps per tooth
    follows the reference rule max(48, ceil(Ttooth * fTop * 24)) (cutting.js:50)."""
    st = workload.setups[workload.points["setup"]]
    md = workload.modals[workload.points["modal"]]
    N = st["tool"]["N"].astype(np.float64)
    S = np.maximum(100.0, workload.points["S"])
    fx = np.max(np.where(np.arange(A.MAX_MODES)[None, :] < md["nx"][:, None],
                         md["x"]["fn"], 0.0), axis=1)
    fy = np.max(np.where(np.arange(A.MAX_MODES)[None, :] < md["ny"][:, None],
                         md["y"]["fn"], 0.0), axis=1)
    ftop = np.maximum(fx, fy)
    spt = workload.opts.steps_per_tooth or 0
    spt = np.full(len(S), float(spt)) if spt else np.maximum(48.0, np.ceil(60 / (S * N) * ftop * 24))
    return spt * N * N


def shard(cost: np.ndarray, world: int) -> list[np.ndarray]:
    """Greedy longest-processing-time partition of point indices into `world` shards."""
    order = np.argsort(-np.asarray(cost), kind="stable")
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(int(i))
        heapq.heappush(heap, (load + float(cost[i]), r))
    return [np.sort(np.array(p, dtype=np.int64)) for p in parts]


def library_shards(workload, world: int) -> list[np.ndarray]:
    """The library's split (mcs_shard, the one mcs_solve_multi uses): point indices of each
    of `world` shards, from the FP64 preparation's cost of every point (host only)."""
    from ._lib import shard as lib_shard

    of, _ = lib_shard(workload.setups, workload.modals, workload.points, workload.opts, world)
    return [np.flatnonzero(of == r) for r in range(world)]


def gather_results(local_idx: np.ndarray, local_res: np.ndarray, n_total: int, dist,
                   group=None) -> np.ndarray | None:
    """Rank 0 receives every shard's result records in the original point order."""
    payload = (np.asarray(local_idx), np.asarray(local_res))
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    objs = [None] * world if rank == 0 else None
    dist.gather_object(payload, objs, dst=0, group=group)
    if rank != 0:
        return None
    out = np.zeros(n_total, dtype=local_res.dtype)
    for idx, res in objs:
        out[idx] = res
    return out


def max_over_ranks(x: float, dist, device=None) -> float:
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
