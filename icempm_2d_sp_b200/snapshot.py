"""Checkpoints and saved frames in the reference's data layout.

The reference's SnapshotManager (simulation/data_manager/snapshotmanager.cpp)
writes HDF5 files:

  * snapshots  output/<title>/snapshots/sNNNNN.h5, dataset "pts_data", f64
    [19, size] (the HSSOA rows without the capacity padding), attributes
    SimulationStep (int), SimulationTime (double), HSSOA_size (uint),
    nPtsArrays (int) -- SaveSnapshot, snapshotmanager.cpp:358-408; read back by
    ReadPointsFromSnapshot (309-355), which rejects dims other than
    [19, HSSOA_size] or nPtsArrays != 19;
  * point colours  output/<title>/snapshots/point_colors.h5, dataset
    "pts_colors", uint32 [size] (SavePointColors / ReadPointColors, 411-452);
  * frames  output/<title>/frames/fNNNNN.h5: vis_vx, vis_vy, vis_Jpinv, vis_P,
    vis_Q f32 [GridX, GridY], count u8 [GridX, GridY], rgb u8 [GridX, GridY, 3];
    attributes SimulationStep, SimulationTime on "count" (SaveFrame, 769-830);
  * compressed frames  output_compressed/<title>/frames/fNNNNN.h5: vis_Jpinv,
    vis_P, vis_Q, vis_vx, vis_vy quantised to 12 bits over [min, max]
    (normalize_and_discretize, 1067-1085) and JPEG 2000 coded, attributes
    original_width, original_height, discretization_bits, min_value, max_value;
    rgb JPEG 2000 coded; mass_mask u8 [GridX, GridY]; SimulationStep and
    SimulationTime on vis_Jpinv; and forces.h5, dataset "ds_forces" f32
    [frames, 100, 2] grown one frame slice at a time, attribute cellsize
    (SaveFrameCompressed, 1187-1302).
  Frame number = SimulationStep / UpdateEveryNthStep; snapshots are written
  when (frame % SnapshotPeriod) == 0 or at the end time, compressed frames on
  every frame (Model::SaveThread, model.cpp:131-157).

libhdf5 and OpenJPEG are not available to this package, so each of those files
is written as a pair with the same base name:

  <base>.json   {"format": "icempm-raw/1", "source": "<reference file name>",
                 "datasets": {<name>: {"dtype": numpy dtype string (little
                 endian), "shape": [...], "offset": byte offset in <base>.bin,
                 "nbytes": n, "crc32": zlib CRC-32 of the payload,
                 "attrs": {<attr>: [type, value]}}}}
                attribute types "i4", "u4", "f4", "f8" (HDF5 NATIVE_INT,
                NATIVE_UINT, NATIVE_FLOAT, NATIVE_DOUBLE); f8 values are written
                with Python's shortest round-trip repr, so they read back bit
                for bit.
  <base>.bin    the datasets' payloads in C order, each at a 64-byte-aligned
                offset.

The dataset names, shapes, element types and attributes are the reference's;
the payload bytes equal what HDF5 would return from a read of the dataset.  The
JPEG 2000 stage of the compressed frame has no stand-in: its datasets hold the
12-bit quantised plane itself (u16 [GridX, GridY]) with the reference's
attributes, and rgb is stored uncoded (u8 [GridX, GridY, 3]).
"""
import json
import os
import queue
import threading
import zlib

import numpy as np

from .params import N_PTS_ARRAYS

FORMAT = "icempm-raw/1"
ALIGN = 64
MAX_REGIONS = 100
DEFAULT_DISCRETIZATION_BITS = 12
_ATTR_TYPES = {"i4": int, "u4": int, "f4": float, "f8": float}


class SnapshotError(RuntimeError):
    """A file that does not hold what the reader expects (the reference
    throws std::runtime_error in the same places)."""


# ---------------------------------------------------------------- container

def _attr(type_, value):
    if type_ not in _ATTR_TYPES:
        raise ValueError(f"attribute type {type_!r}")
    if type_ == "i4" and not -2**31 <= int(value) < 2**31:
        raise ValueError(f"attribute value {value} does not fit int32")
    if type_ == "u4" and not 0 <= int(value) < 2**32:
        raise ValueError(f"attribute value {value} does not fit uint32")
    v = _ATTR_TYPES[type_](value)
    if type_ == "f4":
        v = float(np.float32(v))
    return [type_, v]


def write_container(base, datasets, source):
    """Write `datasets` {name: (array, {attr: (type, value)})} as <base>.json +
    <base>.bin.  The payload is written first and the sidecar last, each
    through a temporary name, so a reader never sees a sidecar whose payload is
    incomplete."""
    meta = {"format": FORMAT, "source": source, "datasets": {}}
    os.makedirs(os.path.dirname(os.path.abspath(base)), exist_ok=True)
    tmp_bin, tmp_json = base + ".bin.tmp", base + ".json.tmp"
    off = 0
    with open(tmp_bin, "wb") as f:
        for name, (arr, attrs) in datasets.items():
            a = np.ascontiguousarray(arr)
            a = a.astype(a.dtype.newbyteorder("<"), copy=False)
            pad = (-off) % ALIGN
            f.write(b"\0" * pad)
            off += pad
            buf = memoryview(a.reshape(-1).view(np.uint8)) if a.size else b""
            f.write(buf)
            meta["datasets"][name] = {
                "dtype": a.dtype.str, "shape": list(a.shape), "offset": off, "nbytes": a.nbytes,
                "crc32": zlib.crc32(buf) & 0xffffffff,
                "attrs": {k: _attr(t, v) for k, (t, v) in (attrs or {}).items()}}
            off += a.nbytes
    with open(tmp_json, "w") as f:
        json.dump(meta, f, indent=1)
    os.replace(tmp_bin, base + ".bin")
    os.replace(tmp_json, base + ".json")


def read_container(base, names=None):
    """{name: (array, {attr: value})} from <base>.json + <base>.bin; checks the
    format tag, every payload's extent against the file and its CRC-32."""
    try:
        with open(base + ".json") as f:
            meta = json.load(f)
    except (OSError, ValueError) as e:
        raise SnapshotError(f"{base}.json: {e}") from e
    if meta.get("format") != FORMAT:
        raise SnapshotError(f"{base}.json: format {meta.get('format')!r}, expected {FORMAT!r}")
    ds = meta.get("datasets", {})
    want = list(ds) if names is None else list(names)
    out = {}
    with open(base + ".bin", "rb") as f:
        size = os.fstat(f.fileno()).st_size
        for name in want:
            if name not in ds:
                raise SnapshotError(f"{base}: no dataset {name!r}")
            d = ds[name]
            dt = np.dtype(d["dtype"])
            shape = tuple(int(s) for s in d["shape"])
            nbytes = int(np.prod(shape, dtype=np.int64)) * dt.itemsize
            if nbytes != d["nbytes"] or d["offset"] < 0 or d["offset"] + nbytes > size:
                raise SnapshotError(f"{base}: dataset {name!r} extent does not match the payload file")
            f.seek(d["offset"])
            raw = f.read(nbytes)
            if zlib.crc32(raw) & 0xffffffff != d["crc32"]:
                raise SnapshotError(f"{base}: dataset {name!r} fails its CRC-32")
            arr = np.frombuffer(raw, dt).reshape(shape).copy()
            attrs = {k: _ATTR_TYPES[t](v) for k, (t, v) in d.get("attrs", {}).items()}
            out[name] = (arr, attrs)
    return out


# ---------------------------------------------------------------- quantisation

def normalize_and_discretize(a, bits=DEFAULT_DISCRETIZATION_BITS):
    """SnapshotManager::normalize_and_discretize (snapshotmanager.cpp:1067-1085):
    u16 = round((x - min) / (max - min) * (2^bits - 1)), the arithmetic in
    float32 and round-half-away-from-zero as std::round.  A constant array
    (max == min) has no defined result in the reference (0/0); it gives 0 here."""
    x = np.ascontiguousarray(a, np.float32).reshape(-1)
    if x.size == 0:
        return np.zeros(0, np.uint16), np.float32(0), np.float32(0)
    mn, mx = x.min(), x.max()
    rng = np.float32(mx - mn)
    top = np.float32((1 << bits) - 1)
    if rng == 0:
        return np.zeros(x.size, np.uint16), mn, mx
    v = (x - mn) / rng * top                             # float32 throughout
    return np.floor(v.astype(np.float64) + 0.5).astype(np.uint16), mn, mx


def restore_from_discretized(u, mn, mx, bits=DEFAULT_DISCRETIZATION_BITS):
    """SnapshotManager::restore_from_discretized (snapshotmanager.cpp:1516-1537):
    min + u / (2^bits - 1) * (max - min) in float32; a range below 1e-9 gives min."""
    u = np.asarray(u, np.uint16)
    mn, mx = np.float32(mn), np.float32(mx)
    rng = np.float32(mx - mn)
    top = np.float32((1 << bits) - 1)
    if rng < np.float32(1e-9):
        return np.full(u.shape, mn, np.float32)
    return (mn + (u.astype(np.float32) / top) * rng).astype(np.float32)


# ---------------------------------------------------------------- manager

class SnapshotManager:
    """The reference's snapshot and frame files for one simulation title,
    under `root` (the reference writes relative to its working directory)."""

    def __init__(self, title="sim1", root="."):
        self.SimulationTitle = title
        self.root = root

    def _dir(self, top, sub):
        return os.path.join(self.root, top, self.SimulationTitle, sub)

    def snapshot_path(self, frame):
        return os.path.join(self._dir("output", "snapshots"), f"s{frame:05d}")

    def frame_path(self, frame):
        return os.path.join(self._dir("output", "frames"), f"f{frame:05d}")

    def compressed_frame_path(self, frame):
        return os.path.join(self._dir("output_compressed", "frames"), f"f{frame:05d}")

    # -- points
    def SaveSnapshot(self, hssoa, size, SimulationStep, SimulationTime, UpdateEveryNthStep):
        """SaveSnapshot (snapshotmanager.cpp:358-408): the first `size` columns
        of the [19, capacity] HSSOA; returns the base path written."""
        if hssoa.dtype != np.float64 or hssoa.ndim != 2 or hssoa.shape[0] != N_PTS_ARRAYS:
            raise ValueError(f"HSSOA must be float64 [{N_PTS_ARRAYS}, capacity]")
        if not 0 <= size <= hssoa.shape[1]:
            raise ValueError(f"size {size} outside capacity {hssoa.shape[1]}")
        frame = SimulationStep // UpdateEveryNthStep
        base = self.snapshot_path(frame)
        attrs = {"SimulationStep": ("i4", SimulationStep), "SimulationTime": ("f8", SimulationTime),
                 "HSSOA_size": ("u4", size), "nPtsArrays": ("i4", N_PTS_ARRAYS)}
        write_container(base, {"pts_data": (hssoa[:, :size], attrs)}, f"s{frame:05d}.h5")
        return base

    def ReadPointsFromSnapshot(self, path, capacity=None):
        """ReadPointsFromSnapshot (snapshotmanager.cpp:309-355) -> (hssoa
        [19, capacity], size, SimulationStep, SimulationTime).  A bare file
        name is looked up in this title's snapshot folder, as the CLI's resume
        path is (model.cpp:196-206); a ".h5" or ".json" suffix is accepted."""
        base = path
        for suf in (".h5", ".json", ".bin"):
            if base.endswith(suf):
                base = base[:-len(suf)]
        if not os.path.dirname(base):
            base = os.path.join(self._dir("output", "snapshots"), base)
        arr, at = read_container(base, ["pts_data"])["pts_data"]
        for k in ("SimulationStep", "SimulationTime", "HSSOA_size", "nPtsArrays"):
            if k not in at:
                raise SnapshotError(f"{base}: pts_data has no attribute {k}")
        size = int(at["HSSOA_size"])
        if arr.ndim != 2 or arr.shape[0] != N_PTS_ARRAYS or arr.shape[1] != size or at["nPtsArrays"] != N_PTS_ARRAYS:
            raise SnapshotError("ReadSnapshot array size mismatch")
        cap = size if capacity is None else int(capacity)
        if cap < size:
            raise ValueError(f"capacity {cap} below the snapshot's {size} points")
        soa = np.zeros((N_PTS_ARRAYS, cap), np.float64)
        soa[:, :size] = arr.view(np.float64)
        return soa, size, int(at["SimulationStep"]), float(at["SimulationTime"])

    def SavePointColors(self, colors):
        """SavePointColors (snapshotmanager.cpp:411-436): uint32 0xRRGGBB per point id."""
        base = os.path.join(self._dir("output", "snapshots"), "point_colors")
        write_container(base, {"pts_colors": (np.asarray(colors, np.uint32), {})}, "point_colors.h5")
        return base

    def ReadPointColors(self):
        """ReadPointColors (snapshotmanager.cpp:439-452)."""
        base = os.path.join(self._dir("output", "snapshots"), "point_colors")
        arr, _ = read_container(base, ["pts_colors"])["pts_colors"]
        if arr.dtype != np.uint32 or arr.ndim != 1:
            raise SnapshotError(f"{base}: pts_colors is not uint32 [n]")
        return arr

    # -- frames
    @staticmethod
    def _grid(frame, gx, gy, key):
        a = np.asarray(frame[key])
        if a.size != gx * gy:
            raise ValueError(f"frame channel {key} holds {a.size} values, grid has {gx * gy}")
        return a.reshape(gx, gy)

    def SaveFrame(self, frame_arrays, gx, gy, SimulationStep, SimulationTime, UpdateEveryNthStep):
        """SaveFrame (snapshotmanager.cpp:769-830) from the arrays of
        icempm_prepare_frame (node x*GridY + y, so [GridX, GridY] in C order)."""
        frame = SimulationStep // UpdateEveryNthStep
        g = lambda k: self._grid(frame_arrays, gx, gy, k)
        ds = {f"vis_{k}": (g(k).astype(np.float32), {}) for k in ("vx", "vy", "Jpinv", "P", "Q")}
        ds["count"] = (g("count").astype(np.uint8), {"SimulationStep": ("i4", SimulationStep),
                                                     "SimulationTime": ("f8", SimulationTime)})
        ds["rgb"] = (np.asarray(frame_arrays["rgb"], np.uint8).reshape(gx, gy, 3), {})
        base = self.frame_path(frame)
        write_container(base, ds, f"f{frame:05d}.h5")
        return base

    def SaveFrameCompressed(self, frame_arrays, gx, gy, SimulationStep, SimulationTime, UpdateEveryNthStep,
                            cellsize):
        """SaveFrameCompressed (snapshotmanager.cpp:1187-1302): the five fields
        quantised to 12 bits, rgb, mass_mask, and this frame's slice of the
        per-region forces in forces.{json,bin}."""
        frame = SimulationStep // UpdateEveryNthStep
        ds = {}
        for k in ("Jpinv", "P", "Q", "vx", "vy"):
            u, mn, mx = normalize_and_discretize(self._grid(frame_arrays, gx, gy, k))
            attrs = {"original_width": ("i4", gx), "original_height": ("i4", gy),
                     "discretization_bits": ("i4", DEFAULT_DISCRETIZATION_BITS),
                     "min_value": ("f4", float(mn)), "max_value": ("f4", float(mx))}
            if k == "Jpinv":
                attrs.update(SimulationStep=("i4", SimulationStep), SimulationTime=("f8", SimulationTime))
            ds[f"vis_{k}"] = (u.reshape(gx, gy), attrs)
        if "rgb" in frame_arrays and frame_arrays["rgb"] is not None:
            ds["rgb"] = (np.asarray(frame_arrays["rgb"], np.uint8).reshape(gx, gy, 3),
                         {"original_width": ("i4", gx), "original_height": ("i4", gy)})
        ds["mass_mask"] = (self._grid(frame_arrays, gx, gy, "mass_mask").astype(np.uint8), {})
        base = self.compressed_frame_path(frame)
        write_container(base, ds, f"f{frame:05d}.h5")
        self._save_forces(frame, np.asarray(frame_arrays["forces_per_region"], np.float32), cellsize)
        return base

    def _save_forces(self, frame, forces, cellsize):
        """ds_forces f32 [frames, MAX_REGIONS, 2]: the file grows to hold
        `frame` (unwritten slices stay zero, as HDF5's fill value) and the
        slice is replaced."""
        if forces.size != 2 * MAX_REGIONS:
            raise ValueError(f"forces_per_region holds {forces.size} values, expected {2 * MAX_REGIONS}")
        base = os.path.join(self._dir("output_compressed", "frames"), "forces")
        if os.path.exists(base + ".json"):
            arr, at = read_container(base, ["ds_forces"])["ds_forces"]
            cs = at.get("cellsize", cellsize)
        else:
            arr, cs = np.zeros((0, MAX_REGIONS, 2), np.float32), cellsize
        if arr.shape[0] <= frame:
            arr = np.concatenate([arr, np.zeros((frame + 1 - arr.shape[0], MAX_REGIONS, 2), np.float32)])
        arr[frame] = forces.reshape(MAX_REGIONS, 2)
        write_container(base, {"ds_forces": (arr, {"cellsize": ("f8", cs)})}, "forces.h5")

    def LoadFrameCompressed(self, frame):
        """The compressed frame's fields restored to float32 [GridX, GridY]
        (load_compressed_float_array_hdf5 + restore_from_discretized,
        snapshotmanager.cpp:1516-1590), with rgb, mass_mask, step and time."""
        d = read_container(self.compressed_frame_path(frame))
        out = {}
        for k in ("Jpinv", "P", "Q", "vx", "vy"):
            u, at = d[f"vis_{k}"]
            out[k] = restore_from_discretized(u, at["min_value"], at["max_value"], at["discretization_bits"])
        out["mass_mask"] = d["mass_mask"][0]
        if "rgb" in d:
            out["rgb"] = d["rgb"][0]
        at = d["vis_Jpinv"][1]
        return out, int(at["SimulationStep"]), float(at["SimulationTime"])

    def ReadForces(self):
        arr, at = read_container(os.path.join(self._dir("output_compressed", "frames"), "forces"))["ds_forces"]
        return arr, at["cellsize"]


class FrameSaver:
    """Model::SaveThread (model.cpp:131-157) on a Python thread: requests carry
    copies of the points and the frame arrays (the copy takes the place of the
    reference's accessing_point_data lock); at most one request waits, so a
    step that outruns the writer blocks in `request`, as the reference's Step
    blocks on that lock.  A write error is raised by the next `request` or by
    `close`."""

    def __init__(self, manager: SnapshotManager):
        self.mgr = manager
        self.q = queue.Queue(maxsize=1)
        self.error = None
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        while True:
            job = self.q.get()
            if job is None:
                return
            try:
                job()
            except Exception as e:       # reported to the caller's thread
                self.error = e

    def _raise(self):
        if self.error is not None:
            e, self.error = self.error, None
            raise e

    def request(self, prms, hssoa, size, frame_arrays):
        """SaveFrameRequest: a snapshot when (frame % SnapshotPeriod) == 0 or
        at the end time, and the compressed frame always."""
        self._raise()
        step, time = int(prms.SimulationStep), float(prms.SimulationTime)
        every, period = int(prms.UpdateEveryNthStep), int(prms.SnapshotPeriod)
        gx, gy, cs = int(prms.GridXTotal), int(prms.GridYTotal), float(prms.cellsize)
        save_pts = (step // every) % period == 0 or prms.SimulationTime >= prms.SimulationEndTime
        pts = hssoa[:, :size].copy() if save_pts else None
        fr = {k: np.array(v, copy=True) for k, v in frame_arrays.items()}

        def job():
            if pts is not None:
                self.mgr.SaveSnapshot(pts, size, step, time, every)
            self.mgr.SaveFrameCompressed(fr, gx, gy, step, time, every, cs)
        self.q.put(job)

    def close(self):
        self.q.put(None)
        self.t.join()
        self._raise()
