"""Asynchronous point download (icempm_download_points_async /
icempm_download_wait) and the device-side boundary forces.

Bit-exact: a download started before more sub-steps are enqueued holds the
state at the moment it was started; it equals the synchronous download of an
identical run (fixed-point variant, deterministic); an upload issued while a
copy is outstanding does not overwrite what the copy reads; the forces
written into a caller's buffer equal the default path.
"""
import numpy as np
import pytest

from icempm_2d_sp_b200 import scenes, capi as C
from icempm_2d_sp_b200.params import Options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    C.load()
    if C.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    return C


def test_async_download_overlapping_steps(capi):
    sc = scenes.ridging(gx=256, gy=128, cells_x=120, cells_y=100, speed=2.0)
    o = Options.default()
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o) as ref:
        ref.upload(sc.soa, sc.n)
        ref.step(10, 0)
        r10, _ = ref.download(np.zeros_like(sc.soa))
        ref.step(10, 10)
        r20, _ = ref.download(np.zeros_like(sc.soa))
    buf = [np.zeros_like(sc.soa), np.zeros_like(sc.soa)]
    for b in buf:
        capi.host_register(b)
    try:
        with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o) as ctx:
            ctx.upload(sc.soa, sc.n)
            ctx.step(10, 0)
            assert ctx.download_async(buf[0]) == sc.n
            ctx.step(10, 10)                       # overlaps the copy
            ctx.download_wait()
            assert ctx.download_async(buf[1]) == sc.n
            ctx.download_wait()
            ctx.download_wait()                    # nothing outstanding: returns at once
            assert np.array_equal(buf[0].view(np.uint64), r10.view(np.uint64))
            assert np.array_equal(buf[1].view(np.uint64), r20.view(np.uint64))
            # an upload while a copy is outstanding waits for it on the device
            other = sc.soa.copy()
            other[8] += 1.0
            ctx.download_async(buf[0])
            ctx.upload(other, sc.n)
            ctx.download_wait()
            assert np.array_equal(buf[0].view(np.uint64), r20.view(np.uint64))
            back, _ = ctx.download(np.zeros_like(sc.soa))
            assert np.abs(back[8, :sc.n] - other[8, :sc.n]).max() < 1e-6 * np.abs(other[8, :sc.n]).max()
            with pytest.raises(ValueError):
                ctx.download_async(np.zeros((18, sc.n)))
            with pytest.raises(capi.IcempmError):
                ctx.download_async(np.zeros((19, sc.n - 1)))
    finally:
        for b in buf:
            capi.host_unregister(b)


def test_forces_into_caller_buffer(capi):
    sc = scenes.ridging(gx=256, gy=128, cells_x=120, cells_y=100, speed=2.0)
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=Options.default()) as ctx:
        ctx.upload(sc.soa, sc.n)
        ctx.clear_force_accumulator()
        ctx.step(20, 0)
        f1 = ctx.boundary_forces(20)
        out = np.full(2 * ctx.G, np.nan)
        f2 = ctx.boundary_forces(20, out)
        f4 = ctx.boundary_forces(10)
        assert f2 is out and np.array_equal(f1, f2)
        assert np.abs(f1).max() > 0                         # the wall took load
        assert np.array_equal(f4, (f1 * (20 * sc.prms.InitialTimeStep)) / (10 * sc.prms.InitialTimeStep)) or \
            np.abs(f4 - 2 * f1).max() <= 1e-15 * np.abs(f1).max()
        with pytest.raises(ValueError):
            ctx.boundary_forces(20, np.zeros(2 * ctx.G - 1))
