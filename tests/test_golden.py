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


def _within(alim, ref_alim, opn, ref_open, tol=0.02):
    both = (opn == 1) & (ref_open == 1)
    rel = np.where(both, 0.0, np.abs(alim / ref_alim - 1))
    return rel <= tol


def test_self_agreement_fixture_reproduces(oracle):
    """self_agreement.npz is the oracle's timeDomainLimit under scaled feeds: recomputing
    two of its points gives the same bits."""
    from mcs import _abi as A

    s = load_golden("self_agreement")
    g = load_golden("sweep")
    idx = [0, 117]
    setups = g["setups"].copy()
    setups["fz"] *= 1 + s["levels"][0]
    S = [A.Setup.from_buffer_copy(r.tobytes()) for r in setups]
    M = [A.Modal.from_buffer_copy(r.tobytes()) for r in g["modals"]]
    pts = g["points"][idx]
    P = (A.Point * len(pts)).from_buffer_copy(pts.tobytes())
    res, _ = oracle.solve_batch(S, M, P, A.opts_from_record(g["opts"]), nthreads=0)
    assert res["alim"].tobytes() == s["sweep_alim"][0][idx].tobytes()


@pytest.mark.parametrize("name", ["sweep", "hetero"])
def test_reference_disagrees_with_itself_under_a_1e6_feed_change(name):
    """The FP64 reference's own critical depths are ill-conditioned near chaotic chatter:
    scaling the feed by 1 +- 1e-6 (about what the rounding of an FP32 trajectory amounts
    to) moves more than 1 % of the limits by more than 2 %.  This is why FP32 integration
    cannot meet a 2 %-on-99 % bar against FP64 on these workloads, and why the parity tests
    hold FP32 to the reference's own agreement under that change."""
    s = load_golden("self_agreement")
    g = load_golden(name)
    ref = g["results"]
    for k, eps in enumerate(s["levels"]):
        ok = _within(s[f"{name}_alim"][k], ref["alim"], s[f"{name}_open"][k], ref["open"])
        print(f"{name}: feed x (1 + {eps:g}): {ok.sum()}/{len(ok)} within 2 % of the reference")
        if abs(eps) == 1e-6:
            assert ok.mean() < 0.99
