"""Generate ``warm_bubble_3d_60steps.npz``: the oracle's 3-D dry warm bubble
(64 x 64 x 40, dx = dy = 1 km, dt = 6 s, 6 acoustic substeps, doubly
periodic) advanced 60 RK3 steps (360 s), stored as the central x-z cross
sections (j = ny/2) of every prognostic field plus per-field max-abs and L2
norms of the full 3-D fields.  The GPU drift test compares the CUDA step's
60-step trajectory with these.  Takes about one minute on one CPU core.

    python tests/golden/make_drift60_golden.py
"""

from __future__ import annotations

import os
import sys
from types import SimpleNamespace

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import dycore as D  # noqa: E402
from wrf_gpu_b200 import cases  # noqa: E402

NSTEPS = 60
FIELDS = ("u", "v", "w", "theta", "p_perturbation", "ph_perturbation", "mu_perturbation")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "warm_bubble_3d_60steps.npz")


def summarize(state, jc):
    out = {}
    for f in FIELDS:
        a = np.asarray(getattr(state, f))
        out[f + "_xz"] = a[:, jc, :] if a.ndim == 3 else a[jc, :]
        out[f + "_maxabs"] = np.array(float(np.abs(a).max()))
        out[f + "_l2"] = np.array(float(np.sqrt(np.mean(a * a))))
    return out


def main():
    case = cases.warm_bubble_3d(64, 64, 40)
    nl = D.Namelist(metrics=case.metrics, **case.controls)
    carry = SimpleNamespace(state=D.copy_state(case.state), mudf=case.mudf.copy())
    for n in range(NSTEPS):
        out = D.rk_scan_step(carry, nl, lead_seconds=n * nl.dt_s)
        carry = SimpleNamespace(state=out.state, mudf=out.mudf)
    np.savez_compressed(OUT, nsteps=np.array(NSTEPS), jc=np.array(case.ny // 2), **summarize(carry.state, case.ny // 2))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
