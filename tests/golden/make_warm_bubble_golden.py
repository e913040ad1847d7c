"""Generate ``warm_bubble_2d_500s.json``: the oracle's 2-D Skamarock warm bubble
(the reference's own idealized case, ``ic_generators/idealized.py:195-276``)
run 5000 steps (500 s) and diagnosed with the reference's gate diagnostics
(``idealized.py:660-773``).  Takes about 9 minutes on one CPU core.

    python tests/golden/make_warm_bubble_golden.py
"""

from __future__ import annotations

import json
import os
import sys
from types import SimpleNamespace

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import dycore as D  # noqa: E402
from wrf_gpu_b200 import cases  # noqa: E402

# The reference's own recorded gate values for this case at 500 s
# (proofs/v040/idealized_no_regression_report.json, reference run on GPU).
REFERENCE_RECORDED = {"source": "proofs/v040/idealized_no_regression_report.json (reference run on GPU, reference v0.4.0)",
                      "max_abs_w": 11.680187856366487, "thermal_rise": 1924.3475674060383,
                      "theta_prime_max": 1.9200603163244523, "relative_mass_drift": 0.0}


def diagnose(case, state):
    """The reference's snapshot diagnostics (idealized.py:660-705, 751-773)."""
    x_m, z_m = case.notes["x_m"], case.notes["z_m"]
    tp = state.theta[:, 0, :] - 300.0
    wf = state.w[:, 0, :]
    wm = 0.5 * (wf[:-1] + wf[1:])
    wp = np.maximum(tp, 0.0)
    tot = float(np.sum(wp))
    return {"theta_prime_max": float(tp.max()), "max_abs_w": float(np.abs(wm).max()),
            "center_z": float(np.sum(wp * z_m[:, None]) / tot), "center_x": float(np.sum(wp * x_m[None, :]) / tot),
            "mass": float(np.sum(state.mu_total))}


def main(steps: int = 5000, out: str | None = None):
    case = cases.warm_bubble_2d()
    nl = D.Namelist(metrics=case.metrics, **case.controls)
    carry = SimpleNamespace(state=D.copy_state(case.state), mudf=case.mudf.copy())
    d0 = diagnose(case, carry.state)
    for i in range(steps):
        carry = D.rk_scan_step(carry, nl, lead_seconds=i * nl.dt_s)
    d = diagnose(case, carry.state)
    res = {"steps": steps, "theta_prime_max": d["theta_prime_max"], "max_abs_w": d["max_abs_w"],
           "thermal_rise": d["center_z"] - d0["center_z"], "horizontal_drift": abs(d["center_x"] - 10000.0),
           "relative_mass_drift": abs(d["mass"] - d0["mass"]) / d0["mass"],
           "reference_recorded": REFERENCE_RECORDED}
    path = out or os.path.join(os.path.dirname(os.path.abspath(__file__)), "warm_bubble_2d_500s.json")
    with open(path, "w") as f:
        json.dump(res, f, indent=1)
    return res


if __name__ == "__main__":
    print(main())
