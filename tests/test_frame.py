"""Saved-frame grid arrays (icempm_prepare_frame) against the reference's own
SnapshotManager::PrepareFrameArrays (the golden fixture frame_ridging, made by
tests/golden/make_golden.py from the reference function compiled by
oracle/refbuild/build_ref.py) and against the CPU restatement
(oracle/frame_reference.py), which the same fixture pins.

Tolerances: the ten channels within 1e-4 of each channel's largest magnitude
(FP32 sums in another order), Jpinv (an average of values near 1, minus 1)
within 2e-6 absolute; mass mask and points per cell identical except
nodes whose density sits within 1e-5 of the 0.1 threshold; colour within one
unit (truncation after FP32 blending); region forces within 1e-4 relative.
The restatement (float64 sums) against the reference (float32 sums in point
order): channels within 1e-5 of the channel's largest magnitude.
"""
import os

import numpy as np
import pytest

from icempm_2d_sp_b200 import scenes, hssoa as H
from icempm_2d_sp_b200.params import Options, SimParams, IDX_UTILITY, STATUS_DISABLED
from oracle import frame_reference as fr

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "frame_ridging.npz")
CHANNELS = ("density", "mass", "vx", "vy", "Jpinv", "P", "Q", "r", "g", "b")


def _golden():
    z = np.load(GOLDEN)
    return z, SimParams.from_buffer_copy(z["prms"].tobytes())


def _compare(got, z, tol_rel, jp_abs, forces=True):
    for k in CHANNELS:
        ref = z["out_" + k].astype(np.float64)
        tol = jp_abs if k == "Jpinv" else tol_rel * max(np.abs(ref).max(), 1e-30)
        g = got[k] if k in got else got["point_density"]     # the C ABI's name of the density channel
        assert np.abs(np.asarray(g, np.float64) - ref).max() <= tol, k
    dens = z["out_density"].astype(np.float64)
    border = np.abs(dens - 0.1) < 1e-5
    assert np.array_equal(np.asarray(got["mass_mask"])[~border], z["out_mass_mask"][~border])
    assert np.array_equal(np.asarray(got["count"]), z["out_count"])
    assert np.abs(np.asarray(got["rgb"]).astype(int) - z["out_rgb"].astype(int)).max() <= 1
    if forces:
        rf = z["out_forces_per_region"].astype(np.float64).reshape(-1)
        gf = np.asarray(got["forces_per_region"], np.float64).reshape(-1)
        assert np.abs(gf - rf).max() <= tol_rel * max(np.abs(rf).max(), 1e-30)


def test_restatement_matches_reference_golden():
    """The CPU restatement reproduces the reference function's own output."""
    z, prms = _golden()
    n = int(z["n"])
    assert int(z["out_mass_mask"].sum()) > 0 and np.abs(z["out_forces_per_region"]).max() > 0
    out = fr.prepare_frame(prms, z["soa"], n, z["status"], z["forces"], z["colors"])
    _compare(out, z, 1e-5, 1e-6)


@pytest.mark.gpu
def test_frame_arrays_match_reference_golden():
    """icempm_prepare_frame on the fixture's point state (uploaded through the
    C ABI, no sub-steps: the force accumulator is empty, so the region forces
    are zero) against the reference function's arrays."""
    from icempm_2d_sp_b200 import capi
    capi.load()
    if capi.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    z, prms = _golden()
    n = int(z["n"])
    G = prms.GridXTotal * prms.GridYTotal
    with capi.Context(prms, z["status"], np.zeros(2 * G), capacity=n, options=Options.default()) as ctx:
        ctx.upload(z["soa"], n)
        ctx.clear_force_accumulator()
        got = ctx.prepare_frame(1, z["colors"])
    _compare(got, z, 1e-4, 2e-6, forces=False)
    assert np.abs(got["forces_per_region"]).max() == 0.0


def test_reference_restatement_single_point():
    """KAT of the restatement: one point at a cell centre spreads the B-spline
    weights 1/8, 3/4, 1/8 per axis: density 9/16 at the centre node."""
    sc = scenes.random_state(seed=1, gx=16, gy=16)
    soa = sc.soa[:, :1].copy()
    cell = (8 << 16) | 8
    soa[1, 0] = np.frombuffer(np.uint64(cell).tobytes(), np.float64)[0]
    soa[0, 0] = 0.0
    soa[2, 0] = 0.0
    soa[6, 0] = soa[7, 0] = 0.0
    soa[8, 0], soa[9, 0] = 2.0, -1.0
    status = np.full(256, 100, np.uint8)
    out = fr.prepare_frame(sc.prms, soa, 1, status, np.zeros(512), colors=np.array([0x102030], np.uint32))
    c = 8 * 16 + 8
    assert abs(out["density"][c] - 0.5625) < 1e-12
    assert abs(out["vx"][c] - 2.0) < 1e-12 and abs(out["vy"][c] + 1.0) < 1e-12
    assert out["count"][c] == 1 and out["mass_mask"][c] == 1
    # a side node holds 3/4 * 1/8 = 0.09375 < 0.1: masked and zeroed, colour blended with water
    assert out["mass_mask"][c + 1] == 0 and out["density"][c + 1] == 0.0
    a = 0.09375
    assert out["rgb"][3 * (c + 1)] == int(a * 0x10 + (1 - a) * 0x15)
    assert abs(out["r"][c] - 0x10) < 1e-9 and abs(out["b"][c] - 0x30) < 1e-9


@pytest.mark.gpu
def test_frame_arrays_match_restatement():
    from icempm_2d_sp_b200 import capi
    capi.load()
    if capi.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    sc = scenes.ridging(gx=256, gy=128, cells_x=120, cells_y=100, speed=2.0)
    rng = np.random.default_rng(5)
    soa = sc.soa.copy()
    util = H.get_u32(soa, IDX_UTILITY, sc.n).copy()
    util[rng.random(sc.n) < 0.05] |= STATUS_DISABLED            # some disabled points
    H.set_u32(soa, IDX_UTILITY, util, sc.n)
    colors = rng.integers(0, 1 << 24, sc.n).astype(np.uint32)
    steps = 30
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=Options.default()) as ctx:
        ctx.upload(soa, sc.n)
        ctx.step(steps, 0)
        got = ctx.prepare_frame(steps, colors)
        got2 = ctx.prepare_frame(steps, colors)                 # repeatable
        out, m = ctx.download(np.zeros_like(soa))
        forces = ctx.boundary_forces(steps)
    ref = fr.prepare_frame(sc.prms, out, m, sc.status, forces, colors)
    for k in capi.FRAME_CHANNELS:
        rk = "density" if k == "point_density" else k
        scale = max(np.abs(ref[rk]).max(), 1e-30)
        # Jpinv is sum(w Jp) / sum(w) - 1 with Jp ~ 1: FP32 sums leave ~1e-7 absolute
        tol = 2e-6 if k == "Jpinv" else 1e-4 * scale
        assert np.abs(got[k] - ref[rk]).max() <= tol, k
        assert np.abs(got2[k] - got[k]).max() <= tol, k
    border = np.abs(ref["density"] - 0.1) < 1e-5
    assert np.array_equal(got["mass_mask"][~border], ref["mass_mask"][~border])
    assert np.array_equal(got["count"], ref["count"])
    assert np.abs(got["rgb"].astype(int) - ref["rgb"].astype(int)).max() <= 1
    rf = ref["forces_per_region"]
    assert np.abs(got["forces_per_region"] - rf).max() <= 1e-4 * max(np.abs(rf).max(), 1e-30)
    assert np.abs(rf).max() > 0                                 # the wall took load
