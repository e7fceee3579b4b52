"""The C ABI surface without a GPU: struct layouts of include/mcs.h against the ctypes and
numpy mirrors (compiled with gcc), every declared entry point exported by libmcs.so,
argument errors reported before any device work, the reference defaults."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "mcs.h"

STRUCTS = ["mcs_mode", "mcs_modal", "mcs_tool", "mcs_material", "mcs_setup", "mcs_point",
           "mcs_opts", "mcs_result", "mcs_trial", "mcs_trial_result", "mcs_lobe_query",
           "mcs_plan_info", "mcs_train_opts", "mcs_guide_opts", "mcs_guide_info"]


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(mcs_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def c_sizes(tmp_path_factory):
    d = tmp_path_factory.mktemp("abi")
    src = d / "sizes.c"
    fields = {"mcs_opts": ["a_max", "iters", "chatter_idx", "precision"],
              "mcs_result": ["alim", "open", "evals", "engaged"],
              "mcs_setup": ["tool", "mat", "arc_st", "fz"],
              "mcs_modal": ["nx", "x", "y"],
              "mcs_lobe_query": ["Ktc", "rpm_max", "modal"],
              "mcs_plan_info": ["n_points", "h2d_bytes", "d2h_bytes"],
              "mcs_train_opts": ["lr", "seed", "keep_best"],
              "mcs_guide_opts": ["z", "refine", "mode", "levels", "skip_top"],
              "mcs_guide_info": ["mu", "sigma", "path", "rounds"]}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(){"]
    for s in STRUCTS:
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
    for s, fs in fields.items():
        for f in fs:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = d / "sizes"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return dict((k, int(v)) for k, v in (ln.split() for ln in out.splitlines()))


def test_struct_layouts(c_sizes):
    from mcs import _abi as A

    pairs = {"mcs_mode": A.Mode, "mcs_modal": A.Modal, "mcs_tool": A.Tool,
             "mcs_material": A.Material, "mcs_setup": A.Setup, "mcs_point": A.Point,
             "mcs_opts": A.Opts, "mcs_result": A.Result, "mcs_trial": A.Trial,
             "mcs_trial_result": A.TrialResult, "mcs_lobe_query": A.LobeQuery,
             "mcs_plan_info": A.PlanInfo, "mcs_train_opts": A.TrainOpts,
             "mcs_guide_opts": A.GuideOpts, "mcs_guide_info": A.GuideInfo}
    for name, ct in pairs.items():
        assert c_sizes[name] == C.sizeof(ct), name
    dtypes = {"mcs_modal": A.MODAL_DTYPE, "mcs_setup": A.SETUP_DTYPE, "mcs_point": A.POINT_DTYPE,
              "mcs_opts": A.OPTS_DTYPE, "mcs_result": A.RESULT_DTYPE,
              "mcs_trial": A.TRIAL_DTYPE, "mcs_trial_result": A.TRIAL_RESULT_DTYPE}
    for name, dt in dtypes.items():
        assert c_sizes[name] == dt.itemsize, name
    for key, off in c_sizes.items():
        if "." not in key:
            continue
        s, f = key.split(".")
        ct = pairs[s]
        assert getattr(ct, f).offset == off, key


def test_library_exports_every_declared_function(mcs_lib):
    names = declared_functions()
    assert len(names) >= 18
    from mcs import _lib

    assert sorted(_lib.EXPORTS) == names
    for n in names:
        assert hasattr(mcs_lib, n), n
    nm = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True,
                        text=True, check=True).stdout
    exported = set(re.findall(r"\bT (mcs_\w+)$", nm, re.M))
    assert set(names) <= exported


def test_library_has_no_host_fallback(mcs_lib):
    """libmcs.so links the CUDA runtime and carries sm_100a code; no oracle symbols."""
    from mcs import _lib

    nm = subprocess.run(["nm", "-D", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    assert "or_engine" not in nm and "or_solve" not in nm
    ldd = subprocess.run(["ldd", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    assert "liboracle" not in ldd


def test_default_opts_are_the_reference_defaults(mcs_lib):
    from mcs import _abi as A, _lib

    o = _lib.default_opts()
    # stabtd.js:14,24 and :10
    assert (o.a_min, o.a_max, o.iters, o.revs, o.nonlinear) == (0.05, 20.0, 8, 120, 1)
    assert o.chatter_idx == 0.45 and o.honor_runout == 0
    assert bytes(A.make_opts()) == bytes(o)


def test_argument_errors_without_a_device(mcs_lib):
    from mcs import _abi as A, _lib

    L = mcs_lib
    o = A.make_opts()
    out = (A.Result * 1)()
    st = L.mcs_solve(None, None, 0, None, 0, None, 0, C.byref(o), out)
    assert st == A.MCS_ERR_ARG
    assert "ctx" in _lib.last_error()
    h = C.c_void_p()
    st = L.mcs_create(C.byref(h), -1)
    assert st in (A.MCS_ERR_ARG, A.MCS_ERR_CUDA)
    assert _lib.last_error()


def test_create_fails_cleanly_without_a_device(mcs_lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import mcs

    with pytest.raises(mcs.MCSError) as e:
        mcs.Context(0)
    assert e.value.status == 2  # MCS_ERR_CUDA: no fallback to the host


def test_modal_conversion_follows_modeset():
    """frf.js modeSet: x = modesX or the single mode, y = modesY or x."""
    from mcs import _abi as A

    m = A.make_modal({"k": 1e4, "fn": 1000, "zeta": 0.02})
    assert (m.nx, m.ny) == (1, 0) and m.x[0].k == 1e4
    m = A.make_modal({"k": 0, "fn": 0, "zeta": 0,
                      "modesX": [{"k": 1, "fn": 2, "zeta": 0.1}, {"k": 3, "fn": 4, "zeta": 0.2}]})
    assert (m.nx, m.ny) == (2, 0)
    with pytest.raises(ValueError):
        A.make_modal({"modesX": [{"k": 1, "fn": 1, "zeta": 0}] * 5})


def test_tool_conversion_units():
    """Tool runout arrives in micrometres (stabtd.js:12) and reaches the engine in mm."""
    from mcs import _abi as A

    t = A.make_tool({"N": 3, "R": 5, "helixDeg": 30, "type": "ball", "fluteLen": 25,
                     "runout": 5})
    assert t.runout == pytest.approx(0.005) and t.type == A.TOOL_BALL
    assert A.make_tool({"N": 2, "D": 6}).R == 3.0


def test_precision_option():
    from mcs import _abi as A

    assert A.make_opts().precision == A.FP64  # the reference's arithmetic by default
    assert A.make_opts(precision="fp32").precision == A.FP32
    assert A.make_opts(precision="fp64").precision == A.FP64
    with pytest.raises(ValueError):
        A.make_opts(precision="fp16")
