"""GPU parity of the CUDA step (through the C ABI) against the reference.

Expected values come from the golden fixtures (produced by the reference's own
kernels compiled on the host, tests/golden/make_golden.py) and, for scenes
without a fixture, from the FP64 oracle that those fixtures pin.

Tolerances (relative unless stated; errors are defined in parity_util.errors):
  * FP64 variant: 1e-9 after up to 60 steps (1e-4 on the chaotic
    disable_then_sort fixture, whose own FP64 roundoff grows to ~1e-6).
  * FP32 state (fixed-point and FP32-atomic variants), one step:
    world position and velocity <= 1e-5, |dFe| <= 1e-6 absolute,
    identical flags and cell keys.
  * FP32 state, 10-60 steps: position <= 1e-4 cells, velocity <= 1e-3,
    |dFe| <= 1e-5, at most 1% of points with a different crushed latch
    (the chaotic disable_then_sort fixture: integer outcomes within 2%,
    floats loosely, see the test).
  * 1000 steps: total momentum and kinetic energy within 1e-4 (fixed-point
    and FP64; 1e-3 for plain FP32 atomics).
"""
import os

import numpy as np
import pytest

from icempm_2d_sp_b200 import scenes, hssoa as H
from icempm_2d_sp_b200.params import (SimParams, Options, VARIANTS, IDX_UTILITY, IDX_CELL, IDX_POINT,
                                      IDX_VELX, STATUS_CRUSHED, STATUS_DISABLED, FORCING_EXTENDED,
                                      WIND_UNIFORM, ERR_POINT_VEL_NAN, ERR_POINT_LEFT_AREA,
                                      ERR_GRID_P2G_NAN_VEL)
from parity_util import errors, aggregates

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def capi():
    from icempm_2d_sp_b200 import capi as C
    C.load()
    if C.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    return C


def load_fixture(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z, SimParams.from_buffer_copy(z["prms"].tobytes())


def run_gpu(capi, prms, status, current, soa_in, n, nsteps, first_step, variant, opts=None, **kw):
    o = opts if opts is not None else Options.default(variant=variant, **kw)
    if opts is not None:
        o.variant = VARIANTS[variant]
    with capi.Context(prms, status, current, capacity=soa_in.shape[1], options=o) as ctx:
        ctx.upload(soa_in, n)
        ctx.step(nsteps, first_step)
        out, m = ctx.download(np.zeros_like(soa_in))
        err, dis = ctx.status()
    assert m == n
    return out, err, dis


@pytest.mark.parametrize("variant", ["fixed", "fp32", "fp64", "textbook"])
def test_one_step_golden(capi, variant):
    z, prms = load_fixture("random_1step")
    n = int(z["n"])
    out, err, dis = run_gpu(capi, prms, z["status"], z["current"], z["soa_in"], n, 1, 0, variant)
    e = errors(out, z["soa_out"], n, prms.cellsize)
    assert err == int(z["err"]) and dis == int(z["disabled"])
    assert e["pid_equal"] and e["thickness_equal"]
    assert e["flags_mismatch"] == 0 and e["cell_mismatch"] == 0
    if variant == "fp64":
        assert e["pos_cells"] < 1e-12 and e["vel_rel"] < 1e-10 and e["fe_abs"] < 1e-12, e
        assert e["bp_rel"] < 1e-9 and e["jp_rel"] < 1e-12 and e["pq_rel"] < 1e-9, e
    else:
        assert e["pos_rel"] <= 1e-5 and e["pos_cells"] <= 1e-5 and e["vel_rel"] <= 1e-5, e
        assert e["fe_abs"] <= 1e-6 and e["jp_rel"] <= 1e-6, e
        assert e["bp_rel"] <= 1e-4 and e["pq_rel"] <= 1e-3, e


MULTI = ["random_10step", "random_plastic_20step", "ridging_60step", "disable_then_sort"]


@pytest.mark.parametrize("variant", ["fixed", "fp32", "fp64", "textbook"])
@pytest.mark.parametrize("name", MULTI)
def test_multi_step_golden(capi, name, variant):
    z, prms = load_fixture(name)
    n = int(z["n"])
    out, err, dis = run_gpu(capi, prms, z["status"], z["current"], z["soa_in"], n, int(z["nsteps"]),
                            int(z["first_step"]), variant)
    e = errors(out, z["soa_out"], n, prms.cellsize)
    assert err == int(z["err"])
    assert e["pid_equal"] and e["thickness_equal"]
    if variant == "fp64":
        tol = 1e-4 if name == "disable_then_sort" else 1e-9
        assert dis == int(z["disabled"]) and e["flags_mismatch"] == 0 and e["cell_mismatch"] == 0, e
        assert e["pos_cells"] < tol and e["vel_rel"] < tol and e["fe_abs"] < tol, e
    elif name == "disable_then_sort":
        # 30 m/s in a 20x16 grid next to the velocity clamp: the FP64 oracle's own
        # summation-order roundoff grows ~1e9x in 40 steps, so FP32 state is
        # checked on the integer outcomes and only loosely on the floats
        assert abs(dis - int(z["disabled"])) <= max(1, n // 50), (dis, int(z["disabled"]))
        assert e["cell_mismatch"] <= max(1, n // 50), e
        assert e["pos_cells"] <= 5e-3 and e["vel_rel"] <= 0.1 and e["fe_abs"] <= 1e-2, e
    else:
        assert abs(dis - int(z["disabled"])) <= max(1, n // 100), (dis, int(z["disabled"]))
        assert e["flags_mismatch"] <= max(1, n // 100) and e["cell_mismatch"] <= max(1, n // 100), e
        assert e["pos_cells"] <= 1e-4 and e["vel_rel"] <= 1e-3 and e["fe_abs"] <= 1e-5, e


def test_fixed_point_is_deterministic(capi):
    sc = scenes.random_state(seed=21, gx=96, gy=64, fill=0.8, crushed_frac=0.7, strain=5e-3)
    outs = []
    for _ in range(2):
        out, err, dis = run_gpu(capi, sc.prms, sc.status, sc.current, sc.soa, sc.n, 40, 0, "fixed")
        outs.append(out)
    assert np.array_equal(outs[0].view(np.uint64), outs[1].view(np.uint64))


def test_upload_download_roundtrip(capi):
    sc = scenes.random_state(seed=22, crushed_frac=0.5, strain=1e-3)
    for variant in ("fp64", "fixed"):
        with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.soa.shape[1],
                          options=Options.default(variant=variant)) as ctx:
            ctx.upload(sc.soa, sc.n)
            out, m = ctx.download(np.zeros_like(sc.soa))
        assert m == sc.n
        assert np.array_equal(out[:3, :m].view(np.uint64), sc.soa[:3, :m].view(np.uint64))
        assert np.array_equal(out[18, :m], sc.soa[18, :m])
        if variant == "fp64":
            assert np.array_equal(out[:, :m], sc.soa[:, :m])
        else:
            rel = np.abs(out[3:18, :m] - sc.soa[3:18, :m]) / np.maximum(np.abs(sc.soa[3:18, :m]), 1e-30)
            assert (rel <= 2 ** -23).all() or np.abs(out[3:18, :m] - sc.soa[3:18, :m]).max() < 1e-6


def _oracle_run(sc, nsteps, first_step=0, opts=None):
    import oracle
    soa = sc.soa.copy()
    grid = oracle.new_grid(sc.prms, current=sc.current)
    err, dis = oracle.run_steps(sc.prms, soa, sc.n, grid, sc.status, nsteps, first_step, opts=opts)
    return soa, grid, err, dis


@pytest.mark.parametrize("variant", ["fixed", "fp64"])
def test_extended_forcing_vs_oracle(capi, variant):
    sc = scenes.random_state(seed=23, crushed_frac=0.3, strain=2e-3, forcing=FORCING_EXTENDED)
    ref, _, rerr, rdis = _oracle_run(sc, 20, 0, opts=sc.options)
    out, err, dis = run_gpu(capi, sc.prms, sc.status, sc.current, sc.soa, sc.n, 20, 0, variant, opts=sc.options)
    e = errors(out, ref, sc.n, sc.prms.cellsize)
    assert err == rerr
    tol = 1e-9 if variant == "fp64" else 1e-3
    assert e["pos_cells"] < tol and e["vel_rel"] < tol, e


@pytest.mark.parametrize("variant", ["fixed", "fp64"])
def test_boundary_forces_vs_oracle(capi, variant):
    sc = scenes.ridging(seed=24, gx=64, gy=32, cells_x=40, cells_y=20)
    ref, grid, _, _ = _oracle_run(sc, 30)
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n,
                      options=Options.default(variant=variant)) as ctx:
        ctx.upload(sc.soa, sc.n)
        ctx.clear_force_accumulator()
        ctx.step(30, 0)
        f = ctx.boundary_forces(30)
    G = sc.grid_nodes
    fref = np.concatenate([grid[7], grid[8]]) / (30 * sc.prms.InitialTimeStep)
    scale = np.abs(fref).max()
    assert scale > 0
    tol = 1e-9 if variant == "fp64" else 2e-3
    assert np.abs(f - fref).max() <= tol * scale


def test_sort_compact_matches_reference(capi):
    z, prms = load_fixture("disable_then_sort")
    n = int(z["n"])
    with capi.Context(prms, z["status"], z["current"], capacity=n, options=Options.default(variant="fp64")) as ctx:
        ctx.upload(z["soa_in"], n)
        ctx.step(int(z["nsteps"]), int(z["first_step"]))
        err, dis = ctx.status()
        assert dis == int(z["disabled"])
        ctx.sort_compact()
        out, m = ctx.download(np.zeros_like(z["soa_in"]))
        assert ctx.status()[1] == 0
    ref = z["sorted_soa"]
    assert m == int(z["sorted_n"])
    ky = H.cell_index(out, m, prms.GridYTotal)
    kr = H.cell_index(ref, m, prms.GridYTotal)
    assert np.array_equal(ky, kr)
    oy = np.lexsort((H.get_u32(out, IDX_POINT, m), ky))
    orr = np.lexsort((H.get_u32(ref, IDX_POINT, m), kr))
    a, b = out[:, :m][:, oy], ref[:, :m][:, orr]
    assert np.array_equal(a[:3].view(np.uint64), b[:3].view(np.uint64))
    assert np.abs(a[3:] - b[3:]).max() <= 1e-4 * np.abs(b[3:]).max()


def test_error_bits_for_nan_and_left_area(capi):
    sc = scenes.random_state(seed=25, crushed_frac=0.0, strain=1e-4)
    soa = sc.soa.copy()
    soa[IDX_VELX, 3] = np.nan                       # NaN velocity: flagged by P2G and G2P
    cells = H.get_u32(soa, IDX_CELL, sc.n).copy()
    cells[7] = (cells[7] & 0xffff0000) | 0          # x cell 0: outside [1, gx-2]
    H.set_u32(soa, IDX_CELL, cells, sc.n)
    import oracle
    ref = soa.copy()
    grid = oracle.new_grid(sc.prms, current=sc.current)
    rerr, _ = oracle.run_steps(sc.prms, ref, sc.n, grid, sc.status, 1, 0)
    assert rerr & ERR_POINT_VEL_NAN and rerr & ERR_POINT_LEFT_AREA
    got = {v: run_gpu(capi, sc.prms, sc.status, sc.current, soa, sc.n, 1, 0, v)[1] for v in VARIANTS}
    # floating-point accumulators carry the NaN into the grid and back to the
    # points, raising the same bits as the reference
    assert (got["fp32"] & 0x7ff) == (rerr & 0x7ff), (hex(got["fp32"]), hex(rerr))
    assert (got["fp64"] & 0x7ff) == (rerr & 0x7ff), (hex(got["fp64"]), hex(rerr))
    # int64 accumulators cannot hold a NaN: the fixed-point variant raises the
    # P2G NaN bit (so the run stops, as Model::Step does on any error bit) and
    # the out-of-area bit, but not the grid/point bits downstream of the NaN
    assert got["fixed"] & ERR_POINT_LEFT_AREA and got["fixed"] & ERR_GRID_P2G_NAN_VEL, hex(got["fixed"])
    assert (got["fixed"] & ~rerr & 0x7ff) == 0, (hex(got["fixed"]), hex(rerr))


@pytest.fixture(scope="module")
def ridging_1000():
    """The precision study's ridging scene (1024x512 grid, 1,000,000 crushed
    points driven at 2 m/s against the x = 0 wall) after 1000 sub-steps of the
    FP64 oracle (about 20 s on 16 host cores)."""
    sc = scenes.ridging()
    ref, _, rerr, rdis = _oracle_run(sc, 1000)
    return sc, ref, rerr


@pytest.mark.slow
@pytest.mark.parametrize("variant", ["fixed", "fp32", "fp64", "textbook"])
def test_1000_steps_aggregates(capi, ridging_1000, variant):
    """Momentum and kinetic energy within 1e-4 of the FP64 oracle after 1000
    sub-steps of fully plastic ridging (plasticity active everywhere), mass
    exact.  The scene is the million-point one the 1e-4 bar is stated for:
    on small scenes one plastic event of one particle moves these aggregates
    by ~1e-4 (seed sweeps of 7,680- and 38,400-point scenes put single FP32
    runs of every variant at up to 1.2e-4 in kinetic energy)."""
    sc, ref, rerr = ridging_1000
    out, err, dis = run_gpu(capi, sc.prms, sc.status, sc.current, sc.soa, sc.n, 1000, 0, variant)
    a, b = aggregates(out, sc.n, sc.prms), aggregates(ref, sc.n, sc.prms)
    assert err == rerr
    assert abs(a["mass"] - b["mass"]) <= 1e-12 * b["mass"]
    tol = 1e-4
    pref = np.hypot(b["px"], b["py"])
    assert np.hypot(a["px"] - b["px"], a["py"] - b["py"]) <= tol * pref, (a, b)
    assert abs(a["ke"] - b["ke"]) <= tol * b["ke"], (a, b)


@pytest.mark.slow
def test_ice_block_1000_steps(capi):
    sc = scenes.ice_block()
    ref, _, rerr, _ = _oracle_run(sc, 1000)
    out, err, dis = run_gpu(capi, sc.prms, sc.status, sc.current, sc.soa, sc.n, 1000, 0, "fixed")
    a, b = aggregates(out, sc.n, sc.prms), aggregates(ref, sc.n, sc.prms)
    assert err == rerr == 0
    assert np.hypot(a["px"] - b["px"], a["py"] - b["py"]) <= 1e-4 * np.hypot(b["px"], b["py"]), (a, b)
    assert abs(a["ke"] - b["ke"]) <= 1e-4 * b["ke"], (a, b)
    e = errors(out, ref, sc.n, sc.prms.cellsize)
    assert e["vel_rel"] <= 1e-4 and e["pos_cells"] <= 1e-5, e
