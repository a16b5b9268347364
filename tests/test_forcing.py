"""Time-varying current and wind (icempm_set_flow_frames / set_wind_frames /
set_forcing_time, icempm_2d_sp_b200/forcing.py) against the CPU restatement
oracle/forcing_reference.py, and the static current import against
WindAndCurrentInterpolator::ReadStaticFlowData
(simulation/data_manager/windandcurrentinterpolator.cpp:20-63).

Tolerances: the device tables equal the restatement bit for bit (same float64
operations, same rounding to the state type); a run with blended current
frames is bit-identical to a run given the host-blended field through
icempm_set_current (fixed-point variant); a run with uniform wind frames
matches the analytic uniform wind within FP32-state tolerance (the bilinear
weights of one cell sum to 1 only up to rounding).
"""
import numpy as np
import pytest

from icempm_2d_sp_b200 import forcing as F, scenes
from icempm_2d_sp_b200.params import SimParams, Options, FORCING_EXTENDED, WIND_UNIFORM
from oracle import forcing_reference as R


def test_flow_field_from_image_follows_reference_indexing():
    p = SimParams.reset()
    p.InitializationImageSizeX, p.InitializationImageSizeY = 11, 9
    p.GridXTotal, p.GridYTotal = 6, 5
    p.ModeledRegionOffsetX, p.ModeledRegionOffsetY = 3, 2
    rng = np.random.default_rng(0)
    img = rng.normal(size=(9, 11, 2)).astype(np.float32)
    got = F.flow_field_from_image(img, p)
    flat = img.reshape(-1, 2)
    ref = np.zeros(2 * 30)
    for i in range(6):
        for j in range(5):
            idx = (i + 3) + (j + 2) * 11
            ref[j + i * 5] = flat[idx, 0]
            ref[30 + j + i * 5] = flat[idx, 1]
    assert np.array_equal(got, ref)
    with pytest.raises(ValueError):
        F.flow_field_from_image(img[:, :10], p)
    p.ModeledRegionOffsetX = 6
    with pytest.raises(ValueError):
        F.flow_field_from_image(img, p)


class FakeCtx:
    G = 4

    def __init__(self):
        self.calls = []

    def set_flow_frames(self, a, b):
        self.calls.append(("flow", float(a[0]), float(b[0])))

    def set_wind_frames(self, w, cell, x0, y0):
        self.calls.append(("wind", float(w[0, 0, 0]), float(w[0, 0, 2]), cell))

    def set_forcing_time(self, tc, tw):
        self.calls.append(("time", round(tc, 12), round(tw, 12)))


def test_interpolator_brackets_and_uploads():
    ctx = FakeCtx()
    wac = F.WindAndCurrentInterpolator(ctx)
    wac.set_current_series([0.0, 10.0, 30.0], [np.full(8, v) for v in (1.0, 2.0, 3.0)])
    wac.set_wind_series([5.0, 15.0], [np.full((2, 3, 2), v, np.float32) for v in (7.0, 9.0)], cell=50.0)
    assert wac.SetTime(0.0)                       # first call uploads both series
    assert ctx.calls == [("flow", 1.0, 2.0), ("wind", 7.0, 9.0, 50.0), ("time", 0.0, 0.0)]
    ctx.calls.clear()
    assert not wac.SetTime(7.5)                   # same brackets: weights only
    assert ctx.calls == [("time", 0.75, 0.25)]
    ctx.calls.clear()
    assert wac.SetTime(20.0)                      # current moves to (10, 30); wind past its last frame
    assert ctx.calls == [("flow", 2.0, 3.0), ("time", 0.5, 1.0)]
    ctx.calls.clear()
    assert not wac.SetTime(99.0)
    assert ctx.calls == [("time", 1.0, 1.0)]
    with pytest.raises(ValueError):
        wac.set_current_series([0.0, 0.0], [np.zeros(8), np.zeros(8)])
    with pytest.raises(ValueError):
        wac.set_current_series([0.0], [np.zeros(7)])
    one = F.WindAndCurrentInterpolator(FakeCtx())
    one.set_current_series([3.0], [np.zeros(8)])
    one.SetTime(100.0)
    assert one.ctx.calls == [("flow", 0.0, 0.0), ("time", 0.0, 0.0)]


def test_restatement_bilinear_and_clamp():
    """A wind field linear in x and y is reproduced by the bilinear weights;
    positions outside the grid take the edge; tw blends the two frames."""
    rows, cols, cell, x0, y0 = 4, 5, 10.0, -5.0, 3.0
    r, c = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
    Xs, Ys = x0 + c * cell, y0 + r * cell
    w = np.zeros((rows, cols, 4), np.float32)
    w[..., 0], w[..., 1] = 0.5 * Xs + 0.25 * Ys, -Ys
    w[..., 2], w[..., 3] = 2.0, 4.0
    X = np.array([0.0, 7.5, 12.25, 30.0])
    Y = np.array([5.0, 10.0, 20.5, 33.0])
    ux, uy = R.wind_at(w, cell, x0, y0, X, Y, 0.0)
    assert np.allclose(ux, 0.5 * X + 0.25 * Y, rtol=1e-12) and np.allclose(uy, -Y, rtol=1e-12)
    ux, uy = R.wind_at(w, cell, x0, y0, np.array([-100.0, 1e4]), np.array([-100.0, 1e4]), 0.0)
    assert ux[0] == w[0, 0, 0] and ux[1] == w[-1, -1, 0]
    ux, uy = R.wind_at(w, cell, x0, y0, X, Y, 0.25)
    assert np.allclose(ux, 0.75 * (0.5 * X + 0.25 * Y) + 0.25 * 2.0, rtol=1e-12)
    ux1, _ = R.wind_at(w[:1, :1], cell, x0, y0, X, Y, 0.0)   # a single sample is uniform
    assert np.all(ux1 == w[0, 0, 0])


# ----------------------------------------------------------------- GPU

@pytest.fixture(scope="module")
def capi():
    from icempm_2d_sp_b200 import capi as C
    C.load()
    if C.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    return C


def _frames(sc, seed):
    rng = np.random.default_rng(seed)
    G = sc.prms.GridXTotal * sc.prms.GridYTotal
    a = rng.normal(0, 0.2, 2 * G)
    b = rng.normal(0, 0.2, 2 * G)
    w = rng.normal(0, 10, (7, 9, 4)).astype(np.float32)
    return a, b, w


@pytest.mark.gpu
@pytest.mark.parametrize("variant,real", [("fixed", np.float32), ("fp64", np.float64)])
def test_device_tables_match_restatement(capi, variant, real):
    sc = scenes.ridging(gx=256, gy=128, cells_x=60, cells_y=50)
    o = Options.default(variant=variant, forcing=FORCING_EXTENDED)
    a, b, w = _frames(sc, 1)
    p = sc.prms
    cell, x0, y0 = 41.0, -30.0, 12.5
    with capi.Context(p, sc.status, sc.current, capacity=sc.n, options=o) as ctx:
        with pytest.raises(capi.IcempmError):
            ctx.set_forcing_time(0.5)                          # no frames yet
        ctx.set_flow_frames(a, b)
        ctx.set_wind_frames(w, cell, x0, y0)
        with pytest.raises(capi.IcempmError):
            ctx.set_forcing_time(1.5)
        with pytest.raises(capi.IcempmError):
            ctx.set_wind_frames(np.zeros((0, 3, 4), np.float32), cell)
        for tc, tw in ((0.0, 0.0), (0.37, 0.81), (1.0, 1.0)):
            ctx.set_forcing_time(tc, tw)
            cur, st = ctx.get_forcing()
            rc, rs = R.forcing_tables(p.GridXTotal, p.GridYTotal, p.cellsize, o.air_density * o.air_drag_coeff,
                                      a, b, tc, w, cell, x0, y0, tw, real=real)
            assert np.array_equal(cur, rc), (tc, tw)
            assert np.array_equal(st, rs), (tc, tw)
        ctx.set_wind_frames(None)                              # only the current blends now
        ctx.set_forcing_time(0.5)
        cur, st2 = ctx.get_forcing()
        assert np.array_equal(cur, R.forcing_tables(p.GridXTotal, p.GridYTotal, p.cellsize, 0.0, a, b, 0.5,
                                                    real=real)[0])
        assert np.array_equal(st2, st)                         # the last wind stress stays


@pytest.mark.gpu
def test_blended_current_run_equals_host_blend(capi):
    """Compat forcing: frames blended on the device and the host-blended field
    through icempm_set_current give bit-identical runs."""
    sc = scenes.ridging(gx=256, gy=128, cells_x=120, cells_y=100, speed=2.0)
    a, b, _ = _frames(sc, 2)
    a[: a.size // 2] -= 2.0
    b[: b.size // 2] -= 1.0
    o = Options.default()
    out = []
    for mode in ("frames", "host"):
        with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o) as ctx:
            ctx.upload(sc.soa, sc.n)
            ctx.step(5, 0)
            if mode == "frames":
                ctx.set_flow_frames(a, b)
                ctx.set_forcing_time(0.37)
            else:
                ctx.set_current(R.blend_current(a, b, 0.37))
            ctx.step(10, 5)
            s, n = ctx.download(np.zeros_like(sc.soa))
            assert ctx.status()[0] == 0
            out.append(s[:, :n].copy())
    assert np.array_equal(out[0].view(np.uint64), out[1].view(np.uint64))


@pytest.mark.gpu
def test_uniform_wind_frames_match_analytic_wind(capi):
    """Extended forcing: wind frames a = 0, b = (15, -5) m/s everywhere at
    tw = 1, switched on after 5 steps, against a context given the same
    5-step state and the options' uniform wind of (15, -5) (both scatter the
    next step from the stored state: the forcing change drops the step the
    fused kernel had already scattered)."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from parity_util import errors
    sc = scenes.ridging(gx=256, gy=128, cells_x=120, cells_y=100, speed=0.5, forcing=FORCING_EXTENDED)
    w = np.zeros((3, 4, 4), np.float32)
    w[..., 2], w[..., 3] = 15.0, -5.0
    o0 = Options.default(forcing=FORCING_EXTENDED)
    o2 = Options.default(forcing=FORCING_EXTENDED, wind_kind=WIND_UNIFORM, wind_u=15.0, wind_v=-5.0)
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o0) as ctx:
        ctx.upload(sc.soa, sc.n)
        ctx.step(5, 0)
        mid, nm = ctx.download(np.zeros_like(sc.soa))
        assert not ctx.get_forcing()[1].any()
        ctx.set_wind_frames(w, cell=100.0)
        ctx.set_forcing_time(0.0, 1.0)
        _, st = ctx.get_forcing()
        ctx.step(15, 5)
        got, n = ctx.download(np.zeros_like(sc.soa))
        assert ctx.status()[0] == 0
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o2) as ctx:
        _, st_ref = ctx.get_forcing()
        ctx.upload(mid, nm)
        ctx.step(15, 5)
        ref, nr = ctx.download(np.zeros_like(sc.soa))
    assert np.abs(st - st_ref).max() <= 1e-6 * np.abs(st_ref).max()
    e = errors(got, ref, n, sc.prms.cellsize)
    assert e["pos_cells"] <= 1e-5 and e["vel_rel"] <= 1e-4 and e["fe_abs"] <= 1e-6, e
    v0 = np.hypot(mid[8, :nm], mid[9, :nm]).mean()
    assert abs(np.hypot(got[8, :n], got[9, :n]).mean() - v0) > 1e-4   # the wind acted
