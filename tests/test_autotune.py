"""The launch-shape autotuner (pytential_b200.autotune): every candidate shape gives
the same apply (to the summation order), the chosen shapes stay in the plan, and the
tuned apply still matches the checker."""

import numpy as np
import pytest
import torch

from pytential_b200 import abi

from helpers import oracle_for, relerr, workload

pytestmark = pytest.mark.gpu


def test_tuning_roundtrip_and_validation():
    from pytential_b200.autotune import get_tuning, set_tuning
    from pytential_b200.fmm import QBXApply
    from pytential_b200 import native
    wl = workload("h3d-CF-small")
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs)
    assert all(v == 0 for v in get_tuning(ap.plan).values())
    set_tuning(ap.plan, {"m2qbxl_densities": 4, "m2l_densities": 1, "p2e_densities": 8,
                         "l2qbxl_densities": 1, "tsqbx_densities": 16})
    assert get_tuning(ap.plan)["p2e_densities"] == 8
    with pytest.raises(native.QBXFMMError) as ei:
        set_tuning(ap.plan, {"m2l_densities": 2})          # not a shape
    assert ei.value.code == abi.QBXFMM_ERR_ARG


@pytest.mark.parametrize("name", ["h3d-CF-small", "h3d-CF-p15"])
def test_every_shape_gives_the_same_apply(name):
    from pytential_b200.autotune import KNOBS, autotune, set_tuning
    from pytential_b200.fmm import QBXApply
    wl = workload(name)
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs)
    dens = torch.from_numpy(wl.density).cuda()
    base = ap(dens).cpu().numpy()
    for knob, (_, cands, mixed_only) in KNOBS.items():
        for c in cands:
            if c in mixed_only:
                continue
            set_tuning(ap.plan, {knob: c})
            assert relerr(ap(dens).cpu().numpy(), base) < 1e-13, (knob, c)
    set_tuning(ap.plan, {})
    res = autotune(ap, reps=2)
    got = ap(dens).cpu().numpy()
    ref = oracle_for(wl).apply(wl.tree_strengths())
    assert relerr(got, ref) < 5e-12
    assert set(res["choice"]) == set(KNOBS)
    assert all(np.isfinite(list(v.values())).all() for v in res["ms"].values())
