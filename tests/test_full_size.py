"""Parity at the benchmark's full sizes.

The floe field (4096x2048 grid, 23.0M points, Voronoi floes, Rankine wind,
extended forcing) and a 16M-point compressive ridging scene (8192x2048
grid, 16.0M points, every point crushed so the return map runs) are advanced
10 sub-steps by the chosen form (fixed-point P2G, FP32 state) and by the FP64
oracle on the host cores, on the same seeded inputs.

Tolerances (those of the multi-step parity tests for FP32 state): world
position within 1e-4 cells, velocity within 1e-3 of the largest speed,
|dFe| within 1e-5, at most 1 % of the points with a different flag word or
cell; identical device error bits; total mass to 1e-12 and momentum and
kinetic energy to 1e-4.  A second run gives a bit-identical state (the
fixed-point sums do not depend on the order of the atomics).
"""
import hashlib

import numpy as np
import pytest

from icempm_2d_sp_b200 import scenes
from icempm_2d_sp_b200.params import Options
from parity_util import errors, aggregates

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
STEPS = 10


@pytest.fixture(scope="module")
def capi():
    from icempm_2d_sp_b200 import capi as C
    C.load()
    if C.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    return C


def _gpu(capi, sc, opts):
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=opts) as ctx:
        ctx.upload(sc.soa, sc.n)
        ctx.step(STEPS, 0)
        out, m = ctx.download(np.zeros_like(sc.soa))
        err, dis = ctx.status()
    assert m == sc.n
    return out, err, dis


def _digest(soa, n):
    return hashlib.sha256(np.ascontiguousarray(soa[:, :n]).tobytes()).hexdigest()


@pytest.mark.parametrize("which", ["floe_field_23M", "ridging_16M"])
def test_full_size_against_fp64_oracle(capi, which):
    import oracle
    if which == "floe_field_23M":
        sc = scenes.floe_field()
    else:
        sc = scenes.ridging(gx=8192, gy=2048, cells_x=4000, cells_y=1000, h=1.0, dt=1e-4, speed=2.0)
    opts = Options.default()
    for f, _ in Options._fields_:
        setattr(opts, f, getattr(sc.options, f))
    out, err, dis = _gpu(capi, sc, opts)
    d1 = _digest(out, sc.n)
    out2, _, _ = _gpu(capi, sc, opts)
    assert _digest(out2, sc.n) == d1
    del out2

    ref = sc.soa.copy()
    grid = oracle.new_grid(sc.prms, current=sc.current)
    rerr, rdis = oracle.run_steps(sc.prms, ref, sc.n, grid, sc.status, STEPS, 0, opts=sc.options)
    del grid
    assert err == rerr
    assert abs(dis - rdis) <= max(1, sc.n // 100)
    e = errors(out, ref, sc.n, sc.prms.cellsize)
    assert e["pid_equal"] and e["thickness_equal"]
    assert e["flags_mismatch"] <= sc.n // 100 and e["cell_mismatch"] <= sc.n // 100, e
    assert e["pos_cells"] <= 1e-4 and e["vel_rel"] <= 1e-3 and e["fe_abs"] <= 1e-5, e
    a, b = aggregates(out, sc.n, sc.prms), aggregates(ref, sc.n, sc.prms)
    assert abs(a["mass"] - b["mass"]) <= 1e-12 * b["mass"]
    assert np.hypot(a["px"] - b["px"], a["py"] - b["py"]) <= 1e-4 * np.hypot(b["px"], b["py"]), (a, b)
    assert abs(a["ke"] - b["ke"]) <= 1e-4 * b["ke"], (a, b)
    print(f"\n{which}: n={sc.n} {e}")
