"""The end-of-step lateral boundary pass on the GPU
(``wrfgpu_apply_lateral_boundaries`` / ``dycore.apply_lateral_boundaries``)
against the oracle's restatement of apply_lateral_boundaries
(coupling/boundary_apply.py:170-326): a perturbed state and drifting random
strips at a lead between two strip times, the full pass (specified and
nested geopotential) and the specified cadence's ring-0 pass."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import dycore as D
from tests import parity_util as P
from wrf_gpu_b200 import cases, dycore

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "theta", "qv", "qc", "qr", "qi", "qs", "qg", "p_total", "p_perturbation", "ph_total",
          "ph_perturbation", "mu_total", "mu_perturbation")


def _state(seed=8):
    case = cases.real_like_moist(30, 22, 10, hmax=800.0, specified=True, bdy_noise=True)
    s = D.copy_state(case.state)
    rng = np.random.default_rng(seed)
    for f, sc in (("u", 0.5), ("v", 0.5), ("w", 0.1), ("theta", 0.3), ("p_perturbation", 30.0),
                  ("ph_perturbation", 5.0)):
        setattr(s, f, getattr(s, f) + sc * rng.standard_normal(getattr(s, f).shape))
    s.mu_perturbation = s.mu_perturbation + 20.0 * rng.standard_normal(s.mu_perturbation.shape)
    return case, P.attach_lbc_leaves(s, rng)


@pytest.mark.parametrize("geo,spec_only", [(True, False), (False, False), (True, True)])
def test_boundary_pass_matches_oracle(cuda_ready, geo, spec_only):
    case, s = _state()
    nl = SimpleNamespace(update_cadence_s=3600.0, spec_zone=1, relax_zone=4, force_geopotential=geo)
    want = D.apply_lateral_boundaries(s, 1800.0, 6.0, nl, dry_spec_only=spec_only)
    st = dycore.State.from_host(s, device="cuda")
    cfg = dycore.BoundaryConfig(force_geopotential=geo)
    got = dycore.apply_lateral_boundaries(st, 1800.0, 6.0, cfg, dry_spec_only=spec_only)
    torch.cuda.synchronize()
    for f in FIELDS:
        err = P.rel_err(getattr(got, f).cpu().numpy(), getattr(want, f))
        assert err <= 1.0e-14, (f, err)
    if not spec_only:
        assert float(got.qv.min()) >= 0.0
        assert float((got.theta - st.theta).abs()[:, 2, 5:-5].max()) > 0.0  # the relax zone moved
    del case
