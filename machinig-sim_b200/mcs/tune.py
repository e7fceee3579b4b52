"""The schedule autotuner: picks max_buckets for a batch and remembers the choice.

A solve's points are grouped into shared-memory size classes ("buckets"), each run as its
own persistent grid on its own stream.  More classes waste less shared memory per warp
(more resident warps) but split the device into more, smaller grids; the best count
depends on the spread of the batch's steps per revolution and slice counts.  Results do not
depend on the schedule, only the time does.

`autotune` times the candidates through `mcs_tune` on a seeded sample of the batch (at
most `sample` points, spread over the batch's cost range), stores the winner under a
signature of the batch in a JSON cache next to the package and returns it.  A later call
with a batch of the same signature reads the cache.
"""
from __future__ import annotations

import hashlib
import json
import os
import threading
from pathlib import Path

import numpy as np

from . import _abi as A
from ._lib import Context

CACHE = Path(__file__).resolve().parent.parent / "tune_cache.json"
CANDIDATES = (3, 4, 6, 8, 12, 16, 24, 32)
_LOCK = threading.Lock()


def signature(setups, modals, points, opts: A.Opts, device_name: str = "") -> str:
    """A key for batches that schedule alike: size (to a power of two), precision, force
    law, and a digest of the speeds, tooth counts and mode counts."""
    pts = A.as_records(points, A.POINT_DTYPE)
    st = A.as_records(setups, A.SETUP_DTYPE)
    md = A.as_records(modals, A.MODAL_DTYPE)
    n = len(pts)
    S = np.sort(pts["S"].astype(np.float64)) if n else np.zeros(1)
    q = np.quantile(S, [0.0, 0.1, 0.5, 0.9, 1.0]).round(-1)
    teeth = np.bincount(st["tool"]["N"][pts["setup"]], minlength=9)[:9] if n else np.zeros(9)
    modes = np.bincount(md["nx"][pts["modal"]], minlength=5)[:5] if n else np.zeros(5)
    h = hashlib.sha1()
    h.update(q.tobytes())
    h.update((teeth / max(1, n)).round(2).tobytes())
    h.update((modes / max(1, n)).round(2).tobytes())
    return (f"{device_name}|n2^{int(np.ceil(np.log2(max(n, 1))))}|p{opts.precision}"
            f"|nl{opts.nonlinear}|s{opts.slices}|r{opts.revs}|{h.hexdigest()[:12]}")


def load_cache(path: Path = CACHE) -> dict:
    try:
        return json.loads(Path(path).read_text())
    except (OSError, ValueError):
        return {}


def store(key: str, entry: dict, path: Path = CACHE) -> None:
    with _LOCK:
        c = load_cache(path)
        c[key] = entry
        tmp = Path(path).with_suffix(f".{os.getpid()}.tmp")
        tmp.write_text(json.dumps(c, indent=1, sort_keys=True))
        tmp.replace(path)


def sample_points(points, k: int, seed: int = 7) -> np.ndarray:
    """k points spread over the batch: every (n/k)-th of a seeded permutation."""
    pts = A.as_records(points, A.POINT_DTYPE)
    if len(pts) <= k:
        return pts
    perm = np.random.default_rng(seed).permutation(len(pts))
    return pts[np.sort(perm[:k])]


def autotune(ctx: Context, setups, modals, points, opts: A.Opts, *, candidates=CANDIDATES,
             sample: int = 8192, cache: Path | None = CACHE, device_name: str = "",
             refresh: bool = False) -> tuple[int, dict]:
    """(max_buckets, record) for the batch; the record holds the timings and the key."""
    key = signature(setups, modals, points, opts, device_name)
    if cache is not None and not refresh:
        hit = load_cache(cache).get(key)
        if hit is not None and hit.get("best") in range(1, A.MAX_BUCKETS + 1):
            return int(hit["best"]), dict(hit, cached=True)
    pts = sample_points(points, sample)
    best, ms = ctx.tune(setups, modals, pts, opts, candidates)
    rec = {"key": key, "best": best, "ms": {str(k): v for k, v in ms.items()},
           "sample_points": int(len(pts)), "cached": False}
    if cache is not None:
        store(key, {k: v for k, v in rec.items() if k != "cached"}, cache)
    return best, rec
