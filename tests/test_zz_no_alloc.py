"""The allocation-free solve (mcs_solve_noalloc), for callers that must not allocate GPU
memory -- code running while a CUDA graph is being built, real-time loops that cannot
afford the device-wide synchronisation of cudaMalloc/cudaFree, hosts whose device memory
belongs to another allocator.  Its scratch lives in a preallocated area shared by all
calls, so the test makes two calls in a row with different inputs (the second must not
see the first's leftovers) and compares each with mcs_solve through the C ABI.

This file is collected last so that a failure here does not hide any other test's.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

DEPTH_RTOL = 0.02  # the parity tests' critical-depth tolerance
NOALLOC_MAX_POINTS = 1024  # MCS_NOALLOC_MAX_POINTS of include/mcs.h


def _solve(ctx, fn_name, g, opts):
    from mcs import _abi as A
    from mcs import _lib

    setups = np.ascontiguousarray(g["setups"])
    modals = np.ascontiguousarray(g["modals"])
    points = np.ascontiguousarray(g["points"])
    out = np.zeros(len(points), dtype=A.RESULT_DTYPE)
    fn = getattr(ctx._L, fn_name)
    st = fn(ctx._h, C.c_void_p(setups.ctypes.data), len(setups),
            C.c_void_p(modals.ctypes.data), len(modals), C.c_void_p(points.ctypes.data),
            len(points), C.byref(opts), C.c_void_p(out.ctypes.data))
    return st, out, _lib.last_error()


def _opts(g, **kw):
    from mcs import _abi as A

    o = A.opts_from_record(g["opts"])
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _check_same(ref, got):
    assert np.array_equal(got["status"], ref["status"])
    rel = np.abs(got["alim"] / ref["alim"] - 1)
    assert np.all(rel <= DEPTH_RTOL), rel.max()
    assert np.array_equal(got["trials"], ref["trials"])
    assert np.array_equal(got["open"], ref["open"])


def test_noalloc_matches_solve_on_two_calls_in_a_row(ctx):
    small = load_golden("small")
    sweep = load_golden("sweep")
    o1 = _opts(small, revs=20)
    o2 = _opts(sweep, revs=20)
    # first call: the 64-speed sweep
    st, a, msg = _solve(ctx, "mcs_solve_noalloc", small, o1)
    assert st == 0, msg
    st, ref_a, msg = _solve(ctx, "mcs_solve", small, o1)
    assert st == 0, msg
    _check_same(ref_a, a)
    # second call right after, different points, process damping, more modes
    st, b, msg = _solve(ctx, "mcs_solve_noalloc", sweep, o2)
    assert st == 0, msg
    st, ref_b, msg = _solve(ctx, "mcs_solve", sweep, o2)
    assert st == 0, msg
    _check_same(ref_b, b)
    # and the first batch once more, now over the second call's leftovers
    st, a2, msg = _solve(ctx, "mcs_solve_noalloc", small, o1)
    assert st == 0, msg
    _check_same(ref_a, a2)


def test_noalloc_rejects_batches_beyond_its_scratch(ctx):
    from mcs import _abi as A
    from mcs import workloads as W

    wl = W.sweep(n_speeds=NOALLOC_MAX_POINTS + 1)
    g = {"setups": wl.setups, "modals": wl.modals, "points": wl.points,
         "opts": A.opts_record(wl.opts)}
    st, _, msg = _solve(ctx, "mcs_solve_noalloc", g, wl.opts)
    assert st == A.MCS_ERR_ARG
    assert "1024" in msg and "scratch" in msg
