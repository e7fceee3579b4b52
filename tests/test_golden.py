"""The committed golden fixtures are the oracle's output: re-running the oracle on a few of
their points reproduces results and trial traces bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden


def oracle_run(oracle, g, idx):
    from mcs import _abi as A

    setups = [A.Setup.from_buffer_copy(r.tobytes()) for r in g["setups"]]
    modals = [A.Modal.from_buffer_copy(r.tobytes()) for r in g["modals"]]
    pts = g["points"][idx]
    P = (A.Point * len(pts)).from_buffer_copy(pts.tobytes())
    opts = A.opts_from_record(g["opts"])
    return oracle.solve_batch(setups, modals, P, opts, nthreads=0, traces=True)


@pytest.mark.parametrize("name,idx", [("small", [0, 37]), ("edge", list(range(11))),
                                      ("sweep", [0, 128]), ("hetero", [0, 1, 2, 3])])
def test_fixture_reproduces(oracle, name, idx):
    g = load_golden(name)
    res, tr = oracle_run(oracle, g, idx)
    ref = g["results"][idx]
    assert res.tobytes() == ref.tobytes()
    assert tr.tobytes() == g["traces"][idx].tobytes()


def test_fixtures_cover_their_workloads():
    from mcs import workloads as W

    sw = load_golden("sweep")
    full = W.sweep()
    assert np.array_equal(sw["index"], full.meta["fp64_subset"])
    assert sw["points"]["S"].tobytes() == full.points["S"][sw["index"]].tobytes()
    het = load_golden("hetero")
    hw = W.hetero()
    assert het["setups"].tobytes() == hw.setups[het["index"]].tobytes()
    for name in ("small", "edge", "sweep", "hetero"):
        g = load_golden(name)
        assert g["sens_flip"].shape == (len(g["sens_levels"]),) + g["traces"].shape
        assert g["sens_levels"][0] == 1e-7
