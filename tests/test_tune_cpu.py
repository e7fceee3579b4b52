"""The schedule autotuner's host logic: batch signatures, sampling and the cache."""
from __future__ import annotations

import numpy as np


def test_signature_is_stable_and_tells_batches_apart():
    from mcs import _abi as A
    from mcs import tune as T
    from mcs import workloads as W

    a, b = W.hetero(n=1024), W.hetero(n=1024)
    ka = T.signature(a.setups, a.modals, a.points, a.opts, "dev")
    assert ka == T.signature(b.setups, b.modals, b.points, b.opts, "dev")
    s = W.sweep()
    assert ka != T.signature(s.setups, s.modals, s.points, s.opts, "dev")
    o64 = A.make_opts(precision="fp64")
    assert T.signature(a.setups, a.modals, a.points, a.opts) != T.signature(
        a.setups, a.modals, a.points, o64)
    assert ka != T.signature(a.setups, a.modals, a.points, a.opts, "other")


def test_sample_spreads_over_the_batch():
    from mcs import tune as T
    from mcs import workloads as W

    wl = W.sweep()
    s = T.sample_points(wl.points, 512)
    assert len(s) == 512
    assert np.all(np.diff(s["S"]) > 0)  # order kept
    assert s["S"].min() < 3300 and s["S"].max() > 29000
    assert len(T.sample_points(wl.points[:100], 512)) == 100


def test_cache_round_trip(tmp_path):
    from mcs import tune as T

    path = tmp_path / "cache.json"
    assert T.load_cache(path) == {}
    T.store("k1", {"best": 16, "ms": {"8": 2.0, "16": 1.5}}, path)
    T.store("k2", {"best": 4}, path)
    c = T.load_cache(path)
    assert c["k1"]["best"] == 16 and c["k2"]["best"] == 4
    path.write_text("not json")
    assert T.load_cache(path) == {}


def test_opts_carry_the_schedule():
    from mcs import _abi as A

    assert A.make_opts().max_buckets == 0
    assert A.make_opts(maxBuckets=12).max_buckets == 12
    assert A.OPTS_DTYPE.itemsize == __import__("ctypes").sizeof(A.Opts)


def test_old_option_records_read_with_defaults():
    """Option records stored before the schedule fields existed read them as 0."""
    import ctypes as C

    from mcs import _abi as A

    o = A.make_opts(maxBuckets=0)
    old = np.frombuffer(bytes(o), dtype=np.uint8)[:56].copy()  # the 56-byte layout
    r = A.opts_from_record(old)
    assert r.max_buckets == 0 and r.serial_trials == 0 and r.a_max == o.a_max
    assert r.coop_warps == 0 and r.coop_points == 0
    assert C.sizeof(A.Opts) == 72
    assert A.make_opts(serialTrials=True).serial_trials == 1
    assert A.make_opts(coopWarps=3, coopPoints=40).coop_points == 40
