"""The Node-API addon glue (machinig-sim_b200/node/mcs_napi.c), built against a stand-in
Node-API runtime (tests/napi/fake_napi.c) because no JavaScript engine exists in this
image.  The CPU test checks argument handling and that, without a device, every
computation throws MCS_ERR_CUDA (no fallback); the GPU test checks the results against
the oracle and the reference's published numbers."""
from __future__ import annotations

import json
import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
NODE = ROOT / "machinig-sim_b200" / "node"
FAKE = ROOT / "tests" / "napi"


@pytest.fixture(scope="module")
def driver(tmp_path_factory, mcs_lib):
    exe = tmp_path_factory.mktemp("napi") / "driver"
    lib = ROOT / "machinig-sim_b200"
    subprocess.run(["gcc", "-std=gnu11", "-Wall", "-Wextra", "-Werror", "-O1",
                    "-o", str(exe), str(FAKE / "driver.c"), str(FAKE / "fake_napi.c"),
                    str(NODE / "mcs_napi.c"), f"-L{lib}", "-lmcs", f"-Wl,-rpath,{lib}",
                    "-lpthread", "-lm"], check=True)
    return exe


def run(driver, oracle) -> dict:
    tm = oracle.tool_model(10, 30, 50000)
    out = subprocess.run([str(driver), repr(tm["k"]), repr(tm["fn"])], capture_output=True,
                         text=True, timeout=600, env=dict(os.environ))
    assert out.returncode == 0, out.stderr
    return {d["case"]: d for d in map(json.loads, out.stdout.splitlines())}


def test_addon_arguments_and_no_fallback(driver, oracle):
    import torch

    res = run(driver, oracle)
    assert res["missing_args"]["threw"] == "MCS_ERR_ARG"
    assert res["bad_tool"]["threw"] == "MCS_ERR_ARG"
    assert res["bad_modal"]["threw"] == "MCS_ERR_ARG"
    if not torch.cuda.is_available():
        for case in ("tdl_defaults_fp64", "tdl_D_runout", "tdl_open", "chatter_shallow",
                     "chatter_deep", "sweep", "lobes"):
            assert res[case].get("threw") == "MCS_ERR_CUDA" or \
                res[case].get("rejected") == "MCS_ERR_CUDA", res[case]


@pytest.mark.gpu
def test_addon_results_on_the_gpu(driver, oracle):
    import math

    res = run(driver, oracle)
    tm = oracle.tool_model(10, 30, 50000)
    modal = {"k": tm["k"], "fn": tm["fn"], "zeta": 0.04}
    mat = dict(Ktc=2100, Krc=850, Kte=35, Kre=45, mc=0.14, Ci=1.5e5)
    tool = dict(N=3, R=5, helixDeg=30, type="flat", fluteLen=25)
    arc = [math.pi / 2, math.pi]
    # the reference's published 0.94 mm at its defaults (FP64 integration)
    d = res["tdl_defaults_fp64"]
    assert f"{d['alim']:.2f}" == "0.94" and d["lo"] < d["alim"] < d["hi"]
    ref = oracle.timeDomainLimit(tool, modal, mat, 8000, arc, 0.05)
    assert d["alim"] == pytest.approx(ref["alim"], rel=1e-12)
    # D instead of R, runout in um (ignored by chatterAt)
    r = oracle.timeDomainLimit(tool, modal, mat, 8000, arc, 0.05, {"revs": 30, "iters": 6})
    assert res["tdl_D_runout"]["alim"] == pytest.approx(r["alim"], rel=0.05)
    assert res["tdl_open"] == {"case": "tdl_open", "alim": 0.3, "hi_inf": 1}
    assert res["chatter_shallow"]["chatter"] == 0 and res["chatter_deep"]["chatter"] == 1
    sw = res["sweep"]
    assert sw["state"] == 1 and sw["S"] == [6000, 9000, 13000]
    for S, a in zip(sw["S"], sw["alim"]):
        want = oracle.timeDomainLimit(tool, modal, mat, S, arc, 0.05, {"revs": 30, "iters": 6})
        assert a == pytest.approx(want["alim"], rel=0.05)
    p = dict(modal, N=3, Ktc=2100, Krc=850, phiSt=arc[0], phiEx=arc[1], lobes=30,
             rpmMin=2000, rpmMax=40000)
    lobes = oracle.stabilityLobes(p)
    for rpm, a in zip((2500, 8000), res["lobes"]["alim"]):
        assert a == pytest.approx(oracle.alimAt(lobes, rpm), rel=1e-10)
