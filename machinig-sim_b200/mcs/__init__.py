"""mcs -- B200 time-domain chatter stability (host layer over libmcs.so).

The functions mirror the reference's JavaScript API for this path:

  timeDomainLimit, chatterAt          src/stabtd.js:14-32
  timeDomainLimits (the Worker sweep) src/stabworker.js:6-14
  StabWorker (the message protocol)   src/stabworker.js:1-15
  lobeLimit (stabilityLobes + alimAt) src/sld.js:23-76
  spindle.Spindle (modesAt)           src/spindle.js:64-85, sim.modalNow (sim.js:229-233)

Surrogate (an MLP trained on the solver's own limits) guides the bisection of
Context.solve_guided and guided plans; mcs.surrogate trains and stores one.

All compute runs in the CUDA library; a missing library or device raises.
"""
from ._abi import (CHATTER_IDX, DEFAULTS, make_material, make_modal, make_opts, make_setup,
                   make_tool)
from ._lib import (Context, Job, MCSError, Plan, Surrogate, default_context, shard, solve_multi,
                   default_guide_opts, default_train_opts, load)
from .sld import alimAt, compositeLobes, lobeLimit, lobeLimits
from .spindle import Spindle, lobe_speeds, sweep_points, tool_model
from .stabtd import chatterAt, chatterIndex, timeDomainLimit, timeDomainLimits
from .worker import StabWorker

__all__ = [
    "CHATTER_IDX", "DEFAULTS", "Context", "Job", "MCSError", "Plan", "Spindle", "StabWorker",
    "Surrogate", "alimAt", "shard", "solve_multi", "compositeLobes", "lobe_speeds", "sweep_points", "tool_model",
    "chatterAt", "chatterIndex", "default_context", "default_guide_opts",
    "default_train_opts", "load", "lobeLimit", "lobeLimits",
    "make_material", "make_modal", "make_opts", "make_setup", "make_tool", "timeDomainLimit",
    "timeDomainLimits",
]
