"""The register-capped solve kernel for FP64 linear buckets computes what the default one
does: byte-identical results, only more warps resident per SM."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_capped_kernel_matches_default(ctx):
    """2048 high speeds of the sweep in one size class (small tables and rings: a bucket
    bound by its total work, where the library picks the capped kernel) against the same
    batch led by one multi-warp point, beside which the other points keep the default
    kernel."""
    from mcs import _abi as A
    from mcs import workloads as W

    wl = W.sweep(n_speeds=4096)
    sub = wl.subset(np.arange(2048, 4096))  # 16,500-30,000 rpm
    o = A.Opts.from_buffer_copy(bytes(sub.opts))
    o.precision = A.FP64
    o.revs = 20
    o.max_buckets = 1
    dense = ctx.plan(sub.setups, sub.modals, sub.points, o)
    dense.execute()
    a = dense.results()
    info_a = dense.info()
    dense.close()
    h = A.Opts.from_buffer_copy(bytes(o))
    h.coop_warps = 8
    h.coop_points = 1
    plain = ctx.plan(sub.setups, sub.modals, sub.points, h)
    plain.execute()
    b = plain.results()
    info_b = plain.info()
    plain.close()
    print(f"capped: {info_a['blocks']} blocks, {info_a['warps_per_sm']} warps/SM; "
          f"default: {info_b['blocks']} blocks, {info_b['warps_per_sm']} warps/SM")
    # more blocks resident in the capped plan (12 warps per SM against the default's 8)
    assert info_a["coop_points"] == 0 and info_b["coop_points"] == 1
    assert info_a["blocks"] > info_b["blocks"]
    assert a.tobytes() == b.tobytes()
