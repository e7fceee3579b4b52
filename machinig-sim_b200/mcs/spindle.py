"""Speed-dependent tool-tip dynamics for lobe sweeps: the reference's spindle model.

The reference's lobe sweep gives every speed its own modal set: main.js:495-496 builds the
Worker's points as {S, modal: sim.modalNow(S)}, and modalNow (sim.js:229-233) applies
modesAt (spindle.js:64-85) with the compliance chain of the active tool (sim.js:235-241).
This module builds the same chain and calls the library's mcs_modes_at for the modes:

    sp = Spindle.from_tool({"D": 10, "stickout": 30, "kSpindle": 5e4}, modal)
    sp.modal_now(15000)            # {k, fn, zeta, modesX, modesY} like sim.modalNow(S)
    pts = sweep_points(sp)         # the 18 log-spaced speeds of main.js:494 with their modes
    timeDomainLimits(tool, mat, arc, fz, pts)            # the Worker sweep on the GPU

toolModel (tool.js:16-32, the uniform carbide cantilever) gives the tool's own stiffness
and modal mass; measured FRFs at several speeds (cfg.modal.speedFrfs) replace the model.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Any, Mapping, Sequence

import numpy as np

from . import _abi as A
from ._lib import _ptr, check, load

E_CARBIDE = 600000.0    # MPa (tool.js:4)
RHO_CARBIDE = 14500.0   # kg/m^3 (tool.js:5)
SOFT_DEFAULT = {"drop": 0.25, "Sref": 30000.0}  # spindle.js:15
LOBE_RANGE = (4000.0, 30000.0)                  # main.js:876


def tool_model(tool: Mapping[str, Any]) -> dict:
    """The uniform cantilever tool (tool.js:16-32): tool stiffness kTool and tip stiffness k
    [N/mm] in series with the spindle, first natural frequency fn [Hz], tip modal mass mEff
    [kg] (the tool's participating mass plus mHolder, 50 g by default)."""
    D, L, kSp = float(tool["D"]), float(tool["stickout"]), float(tool["kSpindle"])
    De = 0.8 * D
    I = math.pi * De ** 4 / 64
    kTool = 3 * E_CARBIDE * I / L ** 3
    kTotal = 1 / (1 / kTool + 1 / kSp)
    EI = E_CARBIDE * 1e6 * I * 1e-12
    rhoA = RHO_CARBIDE * math.pi * (De * 1e-3) ** 2 / 4
    wTool = 1.875 ** 2 * math.sqrt(EI / rhoA) / (L * 1e-3) ** 2
    mEff = kTool * 1e3 / wTool ** 2 + float(tool.get("mHolder", 0.05))
    fn = math.sqrt(kTotal * 1e3 / mEff) / (2 * math.pi)
    return {"kTool": kTool, "k": kTotal, "fn": fn, "mEff": mEff, "De": De, "I": I}


def _speed_frf(e: Mapping[str, Any]) -> A.SpeedFrf:
    f = A.SpeedFrf()
    f.S = float(e["S"])
    m = {"modesX": e["modesX"], "modesY": e.get("modesY") or None}
    if not m["modesY"]:
        m.pop("modesY")
    f.modes = A.make_modal(m)
    return f


class Spindle:
    """A modal set at rest plus the speed model of spindle.js (all FP64, on the host)."""

    def __init__(self, modal: Mapping[str, Any], *, kTool: float = 0.0, kSp: float = 0.0,
                 soft: Mapping[str, Any] | None = None, two_dof: Mapping[str, Any] | None = None,
                 speed_frfs: Sequence[Mapping[str, Any]] = ()):
        soft = SOFT_DEFAULT if soft is None else soft
        sp = A.Spindle()
        sp.rest = A.make_modal(modal)
        sp.drop = float(soft.get("drop", 0.0) or 0.0)
        sp.s_ref = float(soft.get("Sref", 30000.0) or 30000.0)
        sp.k_tool = float(kTool)
        sp.k_sp = float(kSp)
        if two_dof:
            sp.two_dof = 1
            sp.m_tool = float(two_dof["mTool"])
            sp.m_sp = float(two_dof["mSp"])
            sp.z_tool = float(two_dof.get("zTool", modal["zeta"]))
            sp.z_sp = float(two_dof.get("zSp", 0.05))
        self.modal = dict(modal)
        self.record = sp
        self.frfs = [_speed_frf(e) for e in speed_frfs]

    @classmethod
    def from_tool(cls, tool: Mapping[str, Any], modal: Mapping[str, Any], *,
                  soft: Mapping[str, Any] | None = None,
                  spindle_mode: Mapping[str, Any] | None = None) -> "Spindle":
        """The Simulator's chain (sim.js:235-241): the tool's bending stiffness on the spindle
        spring kSpindle; with modal["auto"] the rest mode is the tool model's (k, fn rounded,
        sim.js:221); spindle_mode {on, fn, zeta} adds the spindle/holder mode."""
        tm = tool_model(tool)
        modal = dict(modal)
        if modal.get("auto"):
            modal["k"] = float(math.floor(tm["k"] + 0.5))  # Math.round
            modal["fn"] = float(math.floor(tm["fn"] + 0.5))
        kSp = float(tool["kSpindle"])
        two = None
        if spindle_mode and spindle_mode.get("on"):
            two = {"mTool": tm["mEff"],
                   "mSp": kSp * 1e3 / (2 * math.pi * (spindle_mode.get("fn") or 1200)) ** 2,
                   "zSp": spindle_mode.get("zeta", 0.05), "zTool": modal["zeta"]}
        return cls(modal, kTool=tm["kTool"], kSp=kSp, soft=soft,
                   two_dof=two if modal.get("auto") else None,
                   speed_frfs=modal.get("speedFrfs") or ())

    def modes_at(self, speeds) -> np.ndarray:
        """MODAL_DTYPE records of the modal set at each speed (mcs_modes_at)."""
        S = np.ascontiguousarray(np.atleast_1d(speeds), dtype=np.float64)
        out = np.zeros(max(1, len(S)), dtype=A.MODAL_DTYPE)
        F = A.array_of(A.SpeedFrf, self.frfs)
        check(load().mcs_modes_at(C.byref(self.record), C.cast(F, C.c_void_p), len(self.frfs),
                                  _ptr(S), len(S), _ptr(out)))
        return out[: len(S)]

    def modal_now(self, S: float) -> dict:
        """The modal object of sim.modalNow(S): the rest {k, fn, zeta} plus modesX/modesY."""
        return self._as_modal(self.modes_at([S])[0])

    def _as_modal(self, m) -> dict:
        mx = [{"k": float(r["k"]), "fn": float(r["fn"]), "zeta": float(r["zeta"])}
              for r in m["x"][: m["nx"]]]
        my = [{"k": float(r["k"]), "fn": float(r["fn"]), "zeta": float(r["zeta"])}
              for r in m["y"][: m["ny"]]]
        return {"k": self.modal["k"], "fn": self.modal["fn"], "zeta": self.modal["zeta"],
                "modesX": mx, "modesY": my}


def lobe_speeds(r0: float = LOBE_RANGE[0], r1: float = LOBE_RANGE[1], n: int = 18):
    """The time-domain lobe curve's speeds (main.js:494): S = round(r0 (r1/r0)^(i/(n-1)))."""
    return [float(math.floor(r0 * (r1 / r0) ** (i / (n - 1)) + 0.5)) for i in range(n)]


def sweep_points(spindle: Spindle, speeds=None) -> list[dict]:
    """The Worker's points [{S, modal}] with each speed's own modes (main.js:495-496)."""
    speeds = lobe_speeds() if speeds is None else list(speeds)
    recs = spindle.modes_at(speeds)
    return [{"S": float(S), "modal": spindle._as_modal(r)} for S, r in zip(speeds, recs)]
