"""Checkpoints and saved frames in the reference's data layout
(icempm_2d_sp_b200/snapshot.py, after SnapshotManager::SaveSnapshot /
ReadPointsFromSnapshot / SavePointColors / SaveFrame / SaveFrameCompressed,
simulation/data_manager/snapshotmanager.cpp:309-452, 769-830, 1067-1302).

CPU: the HSSOA round trip is bit-exact (uint32 rows and NaN payloads
included), the reader rejects what ReadPointsFromSnapshot rejects plus corrupt
or truncated payloads, quantisation matches the reference's float32 formula,
frame files hold [GridX, GridY] planes in node order x*GridY + y, the forces
file grows one frame slice at a time, and the writer thread follows
Model::SaveThread's snapshot period.
GPU: a run resumed from a snapshot in a fresh context is bit-identical to the
same run re-uploading its points in place, and within FP32-state tolerance of
the uninterrupted run; and
Model with SaveSnapshots writes the files, whose restored fields agree with the
frame arrays within half a quantisation step.
"""
import json
import os

import numpy as np
import pytest

from icempm_2d_sp_b200 import snapshot as S
from icempm_2d_sp_b200 import scenes, hssoa as H
from icempm_2d_sp_b200.params import SimParams, N_PTS_ARRAYS, IDX_POINT, IDX_UTILITY, Options


def _qtol(mn, mx):
    """Half a 12-bit quantisation step plus float32 rounding of the formula."""
    mn, mx = float(mn), float(mx)
    return 0.5 * (mx - mn) / 4095 + 4e-7 * max(abs(mn), abs(mx), mx - mn)


def _random_hssoa(n, cap, seed=3):
    rng = np.random.default_rng(seed)
    soa = np.zeros((N_PTS_ARRAYS, cap))
    soa[:, :n] = rng.normal(size=(N_PTS_ARRAYS, n))
    for row in (0, 1, 2):                                    # uint32 in the low bytes
        H.set_u32(soa, row, rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32), n)
    bits = soa.view(np.uint64)
    bits[5, 0] = 0x7ff8dead0000beef                          # a NaN with a payload
    bits[6, 1] = 0x8000000000000000                          # -0.0
    bits[7, 2] = 0x0000000000000001                          # a denormal
    return soa


def test_snapshot_round_trip_is_bit_exact(tmp_path):
    n, cap = 1037, 1200
    soa = _random_hssoa(n, cap)
    mgr = S.SnapshotManager("t", str(tmp_path))
    base = mgr.SaveSnapshot(soa, n, 2500, 0.123456789012345678, 100)
    assert base.endswith(os.path.join("output", "t", "snapshots", "s00025"))
    meta = json.load(open(base + ".json"))
    d = meta["datasets"]["pts_data"]
    assert d["shape"] == [19, n] and d["dtype"] == "<f8" and meta["source"] == "s00025.h5"
    assert d["attrs"] == {"SimulationStep": ["i4", 2500], "SimulationTime": ["f8", 0.123456789012345678],
                          "HSSOA_size": ["u4", n], "nPtsArrays": ["i4", 19]}
    assert os.path.getsize(base + ".bin") == 19 * n * 8
    for name in ("s00025", "s00025.h5", base, base + ".json"):
        got, m, step, t = mgr.ReadPointsFromSnapshot(name, capacity=cap + 5)
        assert (m, step, t) == (n, 2500, 0.123456789012345678)
        assert got.shape == (19, cap + 5)
        assert np.array_equal(got[:, :n].view(np.uint64), soa[:, :n].view(np.uint64))
        assert not got[:, n:].any()
    got, m, _, _ = mgr.ReadPointsFromSnapshot("s00025")
    assert got.shape == (19, n)
    with pytest.raises(ValueError):
        mgr.ReadPointsFromSnapshot("s00025", capacity=n - 1)


def test_empty_snapshot(tmp_path):
    mgr = S.SnapshotManager("t", str(tmp_path))
    mgr.SaveSnapshot(np.zeros((19, 4)), 0, 0, 0.0, 10)
    got, m, step, t = mgr.ReadPointsFromSnapshot("s00000")
    assert got.shape == (19, 0) and (m, step, t) == (0, 0, 0.0)


def _edit_meta(base, fn):
    meta = json.load(open(base + ".json"))
    fn(meta)
    json.dump(meta, open(base + ".json", "w"))


@pytest.mark.parametrize("damage", ["nPtsArrays", "HSSOA_size", "shape", "attr", "crc", "truncate", "format",
                                    "dataset", "json"])
def test_reader_rejects_bad_snapshots(tmp_path, damage):
    """ReadPointsFromSnapshot throws on dims[0] != 19, dims[1] != HSSOA_size or
    nPtsArrays != 19 (snapshotmanager.cpp:330-331); the raw form also checks
    the payload's extent and CRC-32."""
    n = 50
    mgr = S.SnapshotManager("t", str(tmp_path))
    base = mgr.SaveSnapshot(_random_hssoa(n, n), n, 10, 1.0, 10)
    pd = lambda m: m["datasets"]["pts_data"]
    if damage == "nPtsArrays":
        _edit_meta(base, lambda m: pd(m)["attrs"].update(nPtsArrays=["i4", 18]))
    elif damage == "HSSOA_size":
        _edit_meta(base, lambda m: pd(m)["attrs"].update(HSSOA_size=["u4", n + 1]))
    elif damage == "shape":
        _edit_meta(base, lambda m: pd(m).update(shape=[18, n], nbytes=18 * n * 8))
    elif damage == "attr":
        _edit_meta(base, lambda m: pd(m)["attrs"].pop("SimulationTime"))
    elif damage == "crc":
        with open(base + ".bin", "r+b") as f:
            f.seek(777)
            b = f.read(1)
            f.seek(777)
            f.write(bytes([b[0] ^ 0x10]))
    elif damage == "truncate":
        with open(base + ".bin", "r+b") as f:
            f.truncate(19 * n * 8 - 8)
    elif damage == "format":
        _edit_meta(base, lambda m: m.update(format="other"))
    elif damage == "dataset":
        _edit_meta(base, lambda m: m["datasets"].update(other=m["datasets"].pop("pts_data")))
    elif damage == "json":
        open(base + ".json", "w").write("{not json")
    with pytest.raises(S.SnapshotError):
        mgr.ReadPointsFromSnapshot("s00001")


def test_writer_rejects_bad_input(tmp_path):
    mgr = S.SnapshotManager("t", str(tmp_path))
    with pytest.raises(ValueError):
        mgr.SaveSnapshot(np.zeros((18, 4)), 4, 0, 0.0, 1)
    with pytest.raises(ValueError):
        mgr.SaveSnapshot(np.zeros((19, 4), np.float32), 4, 0, 0.0, 1)
    with pytest.raises(ValueError):
        mgr.SaveSnapshot(np.zeros((19, 4)), 5, 0, 0.0, 1)
    with pytest.raises(ValueError):
        mgr.SaveSnapshot(np.zeros((19, 4)), 4, 2**31, 0.0, 1)


def test_point_colors_round_trip(tmp_path):
    mgr = S.SnapshotManager("t", str(tmp_path))
    c = np.random.default_rng(1).integers(0, 1 << 24, 999).astype(np.uint32)
    mgr.SavePointColors(c)
    assert np.array_equal(mgr.ReadPointColors(), c)


def test_quantisation_matches_reference_formula():
    """u16 = std::round((x - min) / (max - min) * 4095) in float32
    (snapshotmanager.cpp:1067-1085); restore = min + u / 4095 * (max - min)
    (1516-1537)."""
    x = np.array([-2.0, -1.0, 0.0, 0.5, 3.0], np.float32)
    u, mn, mx = S.normalize_and_discretize(x)
    assert (mn, mx) == (-2.0, 3.0)
    assert u.tolist() == [0, 819, 1638, 2048, 4095]          # 819.0, 1638.0, 2047.5 -> 2048 (half away)
    r = S.restore_from_discretized(u, mn, mx)
    assert r.dtype == np.float32 and abs(r[0] + 2) < 1e-6 and abs(r[-1] - 3) < 1e-6
    rng = np.random.default_rng(2)
    y = rng.normal(size=100_000).astype(np.float32) * 7
    u, mn, mx = S.normalize_and_discretize(y)
    ref = np.array([np.round(np.float32((v - mn) / np.float32(mx - mn) * np.float32(4095))) for v in y[:2000]])
    assert np.array_equal(u[:2000].astype(np.float64), ref)   # numpy round is half-even: no exact halves here
    back = S.restore_from_discretized(u, mn, mx)
    assert np.abs(back - y).max() <= _qtol(mn, mx)
    u0, _, _ = S.normalize_and_discretize(np.full(10, 4.0, np.float32))
    assert not u0.any()
    assert np.all(S.restore_from_discretized(u0, 4.0, 4.0) == 4.0)


def _fake_frame(gx, gy, seed=0):
    rng = np.random.default_rng(seed)
    G = gx * gy
    f = {k: rng.normal(size=G).astype(np.float32) for k in ("point_density", "mass", "vx", "vy", "Jpinv", "P", "Q")}
    f["rgb"] = rng.integers(0, 256, 3 * G).astype(np.uint8)
    f["mass_mask"] = (rng.random(G) > 0.5).astype(np.uint8)
    f["count"] = rng.integers(0, 9, G).astype(np.uint8)
    f["forces_per_region"] = rng.normal(size=200).astype(np.float32)
    return f


def test_frame_files_layout(tmp_path):
    gx, gy = 12, 7
    f = _fake_frame(gx, gy)
    mgr = S.SnapshotManager("t", str(tmp_path))
    base = mgr.SaveFrame(f, gx, gy, 300, 3.5, 100)
    d = S.read_container(base)
    assert base.endswith("f00003")
    assert set(d) == {"vis_vx", "vis_vy", "vis_Jpinv", "vis_P", "vis_Q", "count", "rgb"}
    x, y = 5, 3
    assert d["vis_P"][0].shape == (gx, gy) and d["vis_P"][0][x, y] == f["P"][x * gy + y]
    assert d["rgb"][0].shape == (gx, gy, 3) and d["rgb"][0][x, y, 2] == f["rgb"][3 * (x * gy + y) + 2]
    assert d["count"][1] == {"SimulationStep": 300, "SimulationTime": 3.5}
    base = mgr.SaveFrameCompressed(f, gx, gy, 300, 3.5, 100, 2.0)
    out, step, t = mgr.LoadFrameCompressed(3)
    assert (step, t) == (300, 3.5)
    for k in ("Jpinv", "P", "Q", "vx", "vy"):
        ref = f[k].reshape(gx, gy)
        assert np.abs(out[k] - ref).max() <= _qtol(ref.min(), ref.max())
    at = S.read_container(base)["vis_P"][1]
    assert at["original_width"] == gx and at["original_height"] == gy and at["discretization_bits"] == 12
    assert np.array_equal(out["mass_mask"].reshape(-1), f["mass_mask"])
    assert np.array_equal(out["rgb"].reshape(-1), f["rgb"])


def test_forces_file_grows_per_frame(tmp_path):
    gx, gy = 6, 5
    mgr = S.SnapshotManager("t", str(tmp_path))
    f1, f4 = _fake_frame(gx, gy, 1), _fake_frame(gx, gy, 4)
    mgr.SaveFrameCompressed(f1, gx, gy, 10, 0.1, 10, 2.5)
    mgr.SaveFrameCompressed(f4, gx, gy, 40, 0.4, 10, 2.5)
    arr, cs = mgr.ReadForces()
    assert cs == 2.5 and arr.shape == (5, 100, 2) and arr.dtype == np.float32
    assert np.array_equal(arr[1].reshape(-1), f1["forces_per_region"])
    assert np.array_equal(arr[4].reshape(-1), f4["forces_per_region"])
    assert not arr[[0, 2, 3]].any()
    mgr.SaveFrameCompressed(f4, gx, gy, 10, 0.1, 10, 2.5)      # rewrites slice 1 only
    arr2, _ = mgr.ReadForces()
    assert arr2.shape == (5, 100, 2) and np.array_equal(arr2[1].reshape(-1), f4["forces_per_region"])


def test_frame_saver_period_and_errors(tmp_path):
    """Model::SaveThread (model.cpp:131-157): a snapshot when
    (step / UpdateEveryNthStep) % SnapshotPeriod == 0 or at the end time;
    the compressed frame always."""
    gx, gy = 8, 6
    p = SimParams.reset()
    p.GridXTotal, p.GridYTotal = gx, gy
    p.UpdateEveryNthStep, p.SnapshotPeriod = 10, 3
    p.SimulationEndTime = 1.0
    p.cellsize = 1.0
    mgr = S.SnapshotManager("t", str(tmp_path))
    sv = S.FrameSaver(mgr)
    soa = _random_hssoa(20, 20)
    for fr in range(1, 8):
        p.SimulationStep = 10 * fr
        p.SimulationTime = 0.1 * fr + (0.35 if fr == 7 else 0.0)
        sv.request(p, soa, 20, _fake_frame(gx, gy, fr))
    sv.close()
    snaps = sorted(os.listdir(os.path.join(tmp_path, "output", "t", "snapshots")))
    assert snaps == ["s00003.bin", "s00003.json", "s00006.bin", "s00006.json", "s00007.bin", "s00007.json"]
    frames = sorted(x for x in os.listdir(os.path.join(tmp_path, "output_compressed", "t", "frames"))
                    if x.endswith(".json"))
    assert frames == [f"f{k:05d}.json" for k in range(1, 8)] + ["forces.json"]
    sv = S.FrameSaver(mgr)
    p.SimulationStep = 30
    sv.request(p, soa, 20, _fake_frame(gx + 1, gy))           # wrong grid size: raised later
    with pytest.raises(ValueError):
        sv.close()


def test_attribute_types():
    assert S._attr("f4", 0.1) == ["f4", float(np.float32(0.1))]
    for t, v in (("u4", -1), ("u4", 2**32), ("i4", 2**31), ("x8", 0)):
        with pytest.raises(ValueError):
            S._attr(t, v)


# ----------------------------------------------------------------- GPU

def _by_pid(soa, n):
    order = np.argsort(H.get_u32(soa, IDX_POINT, n), kind="stable")
    return soa[:, :n][:, order].copy()


@pytest.mark.gpu
def test_resume_from_snapshot(tmp_path):
    """A run resumed from a snapshot in a fresh context is bit-identical to the
    same run re-uploading its own downloaded points at that step (both start
    the next sub-step with a P2G from the stored state; fixed-point grid sums
    make it independent of point order), and agrees with the uninterrupted run
    within FP32-state tolerance.  The uninterrupted run differs in the last
    bits because its fused kernel scatters from the stress it has in registers
    (the same FP32 value up to the rounding of its evaluation order)."""
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from parity_util import errors
    from icempm_2d_sp_b200 import capi
    capi.load()
    if capi.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    sc = scenes.ridging(gx=256, gy=128, cells_x=120, cells_y=100, speed=2.0)
    o = Options.default()
    mgr = S.SnapshotManager("resume", str(tmp_path))
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o) as ctx:
        ctx.upload(sc.soa, sc.n)
        ctx.step(20, 0)
        straight, ns = ctx.download(np.zeros_like(sc.soa))
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o) as ctx:
        ctx.upload(sc.soa, sc.n)
        ctx.step(10, 0)
        mid, nm = ctx.download(np.zeros_like(sc.soa))
        mgr.SaveSnapshot(mid, nm, 10, 10 * sc.prms.InitialTimeStep, 5)
        ctx.upload(mid, nm)
        ctx.step(10, 10)
        a, na = ctx.download(np.zeros_like(sc.soa))
        err_a = ctx.status()[0]
    soa, n, step, t = mgr.ReadPointsFromSnapshot("s00002", capacity=sc.n)
    assert (n, step) == (nm, 10) and np.array_equal(soa.view(np.uint64)[:, :n], mid.view(np.uint64)[:, :n])
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o) as ctx:
        ctx.upload(soa, n)
        ctx.step(10, step)
        b, nb = ctx.download(np.zeros_like(sc.soa))
        err_b = ctx.status()[0]
    assert na == nb == ns and err_a == err_b == 0
    A, B, R = _by_pid(a, na), _by_pid(b, nb), _by_pid(straight, ns)
    assert np.array_equal(A.view(np.uint64), B.view(np.uint64))
    assert (H.get_u32(A, IDX_UTILITY) & 0x10000).any()         # the return map was active
    e = errors(B, R, n, sc.prms.cellsize)
    assert e["pos_cells"] <= 1e-5 and e["vel_rel"] <= 1e-4 and e["fe_abs"] <= 1e-6, e
    assert e["flags_mismatch"] == 0 and e["cell_mismatch"] == 0, e


@pytest.mark.gpu
def test_model_saves_snapshots_and_frames(tmp_path):
    from icempm_2d_sp_b200 import capi
    from icempm_2d_sp_b200.model import Model
    capi.load()
    if capi.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    sc = scenes.ridging(gx=256, gy=128, cells_x=120, cells_y=100, speed=2.0)
    p = sc.prms.copy()
    p.AnimationFramePeriod = p.InitialTimeStep * 5.5
    p.compute_helper_variables()
    assert p.UpdateEveryNthStep == 5
    p.SaveSnapshots, p.SnapshotPeriod = True, 2
    colors = np.random.default_rng(0).integers(0, 1 << 24, sc.n).astype(np.uint32)
    m = Model(p, sc.status, sc.current, sc.soa.copy(), sc.n, capacity=sc.n, title="ridge",
              output_root=str(tmp_path), point_colors_rgb=colors)
    m.Prepare()
    frames = []
    try:
        for _ in range(4):
            assert m.Step()
            frames.append({k: v.copy() for k, v in m.frame.items()})
        last = m.hssoa[:, :m.size].copy()
        step, time = m.prms.SimulationStep, m.prms.SimulationTime
    finally:
        m.close()
    mgr = S.SnapshotManager("ridge", str(tmp_path))
    snap_dir = os.path.join(tmp_path, "output", "ridge", "snapshots")
    assert sorted(x for x in os.listdir(snap_dir) if x.endswith(".json")) == \
        ["point_colors.json", "s00002.json", "s00004.json"]
    soa, n, s_step, s_time = mgr.ReadPointsFromSnapshot("s00004.h5")
    assert (s_step, s_time) == (step, time) == (20, p.InitialTimeStep * 19)
    assert np.array_equal(soa.view(np.uint64), last.view(np.uint64))
    assert np.array_equal(mgr.ReadPointColors(), colors)
    gx, gy = p.GridXTotal, p.GridYTotal
    for fr in range(1, 5):
        out, st, _ = mgr.LoadFrameCompressed(fr)
        ref = frames[fr - 1]
        assert st == 5 * fr
        for k in ("Jpinv", "P", "Q", "vx", "vy"):
            r = ref[k].reshape(gx, gy)
            assert np.abs(out[k] - r).max() <= _qtol(r.min(), r.max()), (fr, k)
        assert np.array_equal(out["rgb"].reshape(-1), ref["rgb"])
    forces, cs = mgr.ReadForces()
    assert forces.shape == (5, 100, 2) and cs == p.cellsize
    assert np.array_equal(forces[4].reshape(-1), frames[3]["forces_per_region"])
    assert np.abs(forces[1:]).max() > 0                         # the wall took load
    # resume: Model.resume reads the snapshot and the point colours back
    r = Model.resume(p, sc.status, "s00004", sc.current, title="ridge", output_root=str(tmp_path))
    try:
        assert (r.prms.SimulationStep, r.size) == (20, n)
        assert np.array_equal(r.point_colors_rgb, colors)
        r.prms.SaveSnapshots = False
        r.Prepare()
        assert r.Step() and r.prms.SimulationStep == 25
    finally:
        r.close()
