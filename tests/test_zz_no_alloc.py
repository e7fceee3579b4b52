"""The allocation-free solve (mcs_solve_noalloc), for callers that must not allocate GPU
memory: real-time loops where cudaMalloc/cudaFree may synchronise the whole device, and
host applications whose device memory is already claimed by their own allocator or held
to a fixed budget.  Its scratch lives in a preallocated area shared by all calls, so the
test makes calls in a row with different inputs (a call must not see the previous one's
leftovers) and compares each with mcs_solve through the C ABI, byte for byte: both run the
same deterministic kernels on the same inputs.  It also checks that repeated calls leave
the device's free memory unchanged.

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
    assert np.array_equal(got["trials"], ref["trials"])
    assert np.array_equal(got["open"], ref["open"])
    rel = np.abs(got["alim"] / ref["alim"] - 1)
    assert np.all(rel <= DEPTH_RTOL), rel.max()
    # the same kernels on the same inputs: every field of every record is identical
    assert got.tobytes() == ref.tobytes()


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


def test_noalloc_leaves_device_memory_unchanged(ctx):
    """After a first call (which looks the scratch area up and loads its kernel), further
    calls on the same inputs do not change the device's free memory."""
    import torch

    g = load_golden("small")
    o = _opts(g, revs=10)
    st, ref, msg = _solve(ctx, "mcs_solve_noalloc", g, o)
    assert st == 0, msg
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        st, got, msg = _solve(ctx, "mcs_solve_noalloc", g, o)
        assert st == 0, msg
        assert got.tobytes() == ref.tobytes()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"free device memory moved by {free0 - free1} bytes"
