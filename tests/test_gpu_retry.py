"""The single-period retries (surfdisp.cpp:94-109) on the GPU against the
oracle: on columns of the 256x256x64 model where the continuation from the
previous period fails (Love mode 0 at long periods), the same slots are
retried, the retries find the same roots (|dc| <= 1e-6 km/s against the
oracle's FP64 search) and nothing is left without a root.  The GPU runs the
retry scans 32 grid points at a time per warp, so this is also the check
that the cooperative scan ends in the sequential scan's cell."""
import numpy as np
import pytest

import oracle_lib as O
from jdsurfg_b200 import Engine, ST_RETRIED, synth

pytestmark = pytest.mark.gpu


def test_retried_slots_match_oracle():
    full = synth.make_config("large", seed=2024)
    case = synth.subset_columns(full, np.arange(0, 65536, 16))  # 4096 columns across the grid
    ref = O.get_2d_map(case, refine=1)
    eng = Engine(device=0)
    eng.setup(case)
    g = eng.get_2d_map(case["vs"], case["vp"], case["rho"], nx=case["nx"], ny=case["ny"])
    eng.close()
    nret = int((ref["status"] == ST_RETRIED).sum())
    print(f"{nret} retried slots of {ref['status'].size}")
    assert nret > 20
    assert np.array_equal(g["status"], ref["status"])
    ok = ref["status"] != 1
    assert np.abs(g["vc"] - ref["vc"])[ok].max() <= 1e-6
    assert np.abs(g["vout"] - ref["vout"])[ok].max() <= 1e-6
