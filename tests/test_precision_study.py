"""The precision study's machinery on the small scene (the ice block, 64,000
points, wind), against the FP64 oracle.  The full study (the ice block and the
1M-point ridging scene at 1, 100 and 1000 steps) is tests/precision_study.py.

Tolerances: FP64 on the GPU within 1e-9 cells and 1e-9 relative velocity;
the FP32-state variants within 1e-5 relative velocity after one step and
1e-4 cells / 1e-3 relative velocity after 20 steps; momentum and kinetic
energy within 1e-4; mass exact (no point is disabled in this scene).
"""
import pytest

import precision_study as ps

pytestmark = pytest.mark.gpu


def test_precision_study_ice_block_short():
    from icempm_2d_sp_b200 import capi
    capi.load()
    if capi.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    rows = ps.run(["ice_block"], [1, 20])
    assert len(rows) == 6
    for r in rows:
        assert r["device_errors"] == 0 and r["mass"] == 0.0 and r["flags"] == 0, r
        assert r["mom"] <= 1e-4 and r["ke"] <= 1e-4, r
        if r["variant"] == "fp64":
            assert r["pos_max"] < 1e-9 and r["vel_max"] < 1e-9, r
        elif r["steps"] == 1:
            assert r["vel_max"] <= 1e-5 and r["pos_max"] <= 1e-5, r
        else:
            assert r["vel_max"] <= 1e-3 and r["pos_max"] <= 1e-4, r
