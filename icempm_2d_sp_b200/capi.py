"""ctypes binding of the C ABI (include/icempm.h) in libicempm_b200.so.

The library is built in-tree (icempm_2d_sp_b200/build.py).  Loading fails
loudly when it is missing: there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

from .params import SimParams, Options, N_PTS_ARRAYS

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("ICEMPM_LIBRARY", os.path.join(HERE, "libicempm_b200.so"))

EXPORTS = [
    "icempm_default_options", "icempm_create", "icempm_destroy", "icempm_upload_points",
    "icempm_update_constants", "icempm_set_current", "icempm_step", "icempm_download_points",
    "icempm_get_status", "icempm_clear_force_accumulator", "icempm_get_boundary_forces",
    "icempm_sort_compact", "icempm_timings", "icempm_phase_times", "icempm_fixed_point_scales",
    "icempm_host_register", "icempm_host_unregister", "icempm_device_count", "icempm_point_count",
    "icempm_get_stream", "icempm_launch_count", "icempm_last_error", "icempm_cell_order_noalloc",
    "icempm_batch_create", "icempm_batch_destroy", "icempm_batch_step", "icempm_batch_autotune",
    "icempm_batch_set_tuning", "icempm_batch_get_tuning", "icempm_batch_timings", "icempm_batch_launch_count",
    "icempm_mlp_param_count", "icempm_mlp_grad", "icempm_mlp_adam", "icempm_mlp_forward", "icempm_return_map_exact",
    "icempm_return_map_learned", "icempm_harvest_begin", "icempm_harvest_end", "icempm_prepare_frame",
    "icempm_set_flow_frames", "icempm_set_wind_frames", "icempm_set_forcing_time", "icempm_get_forcing",
    "icempm_download_points_async", "icempm_download_wait", "icempm_debug_barrier_timeout",
    "icempm_set_learned_map", "icempm_learned_map_counts", "icempm_tune_sort_cadence",
]

FRAME_CHANNELS = ("point_density", "mass", "vx", "vy", "Jpinv", "P", "Q", "r", "g", "b")


class FrameBuffers(C.Structure):
    """icempm_frame_t"""
    _fields_ = [(k, C.POINTER(C.c_float)) for k in FRAME_CHANNELS] + [
        ("rgb", C.POINTER(C.c_uint8)), ("mass_mask", C.POINTER(C.c_uint8)), ("count", C.POINTER(C.c_uint8)),
        ("forces_per_region", C.POINTER(C.c_float))]


class BatchTuning(C.Structure):
    """icempm_batch_tuning_t"""
    _fields_ = [("tile_nodes", C.c_int32), ("stages", C.c_int32), ("sort_every", C.c_int32),
                ("graph_steps", C.c_int32), ("ms_per_step", C.c_float), ("reserved", C.c_int32 * 3)]

    def as_dict(self):
        return {"tile_nodes": self.tile_nodes, "stages": self.stages, "sort_every": self.sort_every,
                "graph_steps": self.graph_steps, "ms_per_step": self.ms_per_step}


class IcempmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"icempm error {code}: {msg}")
        self.code = code


_lib = None


def load(path: str = LIB_PATH):
    """Load the CUDA library (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m icempm_2d_sp_b200.build`")
    L = C.CDLL(path)
    h = C.c_void_p
    sp, op = C.POINTER(SimParams), C.POINTER(Options)
    dp, u8p = C.POINTER(C.c_double), C.POINTER(C.c_uint8)
    sig = {
        "icempm_default_options": (None, [op]),
        "icempm_create": (C.c_int, [sp, u8p, dp, C.c_uint32, op, C.POINTER(h)]),
        "icempm_destroy": (C.c_int, [h]),
        "icempm_upload_points": (C.c_int, [h, dp, C.c_uint32, C.c_uint32, C.c_int32]),
        "icempm_update_constants": (C.c_int, [h, sp]),
        "icempm_set_current": (C.c_int, [h, dp]),
        "icempm_set_flow_frames": (C.c_int, [h, dp, dp]),
        "icempm_set_wind_frames": (C.c_int, [h, C.POINTER(C.c_float), C.c_int32, C.c_int32, C.c_double,
                                             C.c_double, C.c_double]),
        "icempm_set_forcing_time": (C.c_int, [h, C.c_double, C.c_double]),
        "icempm_get_forcing": (C.c_int, [h, dp, dp]),
        "icempm_step": (C.c_int, [h, C.c_int32, C.c_int32]),
        "icempm_download_points": (C.c_int, [h, dp, C.c_uint32, C.POINTER(C.c_uint32)]),
        "icempm_download_points_async": (C.c_int, [h, dp, C.c_uint32, C.POINTER(C.c_uint32)]),
        "icempm_download_wait": (C.c_int, [h]),
        "icempm_debug_barrier_timeout": (C.c_int, [h, C.c_uint32, C.c_uint32]),
        "icempm_set_learned_map": (C.c_int, [h, C.c_void_p, C.c_void_p, C.c_float]),
        "icempm_tune_sort_cadence": (C.c_int, [h, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
        "icempm_learned_map_counts": (C.c_int, [h, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "icempm_get_status": (C.c_int, [h, C.POINTER(C.c_uint32), C.POINTER(C.c_int32)]),
        "icempm_clear_force_accumulator": (C.c_int, [h]),
        "icempm_get_boundary_forces": (C.c_int, [h, dp, C.c_int32]),
        "icempm_sort_compact": (C.c_int, [h]),
        "icempm_timings": (C.c_int, [h, C.POINTER(C.c_float)]),
        "icempm_phase_times": (C.c_int, [h, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "icempm_fixed_point_scales": (C.c_int, [h, dp, dp]),
        "icempm_host_register": (C.c_int, [C.c_void_p, C.c_size_t]),
        "icempm_host_unregister": (C.c_int, [C.c_void_p]),
        "icempm_device_count": (C.c_int, [C.POINTER(C.c_int)]),
        "icempm_point_count": (C.c_int, [h, C.POINTER(C.c_uint32)]),
        "icempm_get_stream": (C.c_int, [h, C.POINTER(C.c_void_p)]),
        "icempm_launch_count": (C.c_int, [h, C.POINTER(C.c_uint64)]),
        "icempm_last_error": (C.c_char_p, []),
        "icempm_cell_order_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int32,
                                                C.c_void_p, C.c_void_p, C.c_void_p]),
        "icempm_batch_create": (C.c_int, [C.POINTER(h), C.c_int32, C.POINTER(h)]),
        "icempm_batch_destroy": (C.c_int, [h]),
        "icempm_batch_step": (C.c_int, [h, C.c_int32, C.c_int32]),
        "icempm_batch_autotune": (C.c_int, [h, C.c_int32, C.c_int32, C.POINTER(BatchTuning)]),
        "icempm_batch_set_tuning": (C.c_int, [h, C.POINTER(BatchTuning)]),
        "icempm_batch_get_tuning": (C.c_int, [h, C.POINTER(BatchTuning)]),
        "icempm_batch_timings": (C.c_int, [h, C.POINTER(C.c_float)]),
        "icempm_batch_launch_count": (C.c_int, [h, C.POINTER(C.c_uint64)]),
        "icempm_mlp_param_count": (C.c_int, []),
        "icempm_mlp_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                      C.c_void_p]),
        "icempm_mlp_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_float,
                                      C.c_void_p]),
        "icempm_mlp_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
        "icempm_return_map_exact": (C.c_int, [sp, C.c_void_p, C.c_uint32, C.c_void_p, C.c_int32, C.c_void_p]),
        "icempm_return_map_learned": (C.c_int, [sp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_float,
                                                C.c_void_p, C.c_void_p, C.c_void_p]),
        "icempm_harvest_begin": (C.c_int, [h, C.c_uint32, C.c_int32]),
        "icempm_harvest_end": (C.c_int, [h, C.POINTER(C.c_float), C.c_uint32, C.POINTER(C.c_uint32)]),
        "icempm_prepare_frame": (C.c_int, [h, C.POINTER(C.c_uint32), C.c_uint32, C.c_int32,
                                           C.POINTER(FrameBuffers)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc):
    if rc < 0:
        raise IcempmError(rc, _lib.icempm_last_error().decode())
    return rc


def _dp(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def device_count() -> int:
    L = load()
    n = C.c_int(0)
    L.icempm_device_count(C.byref(n))
    return n.value


def host_register(arr: np.ndarray) -> None:
    check(load().icempm_host_register(arr.ctypes.data, arr.nbytes))


def host_unregister(arr: np.ndarray) -> None:
    check(load().icempm_host_unregister(arr.ctypes.data))


class Context:
    """One scene on one GPU behind the C ABI (the role of GPU_Implementation5)."""

    def harvest_begin(self, capacity, stride=1):
        """Record return-map projections of the following steps (icempm_harvest_begin)."""
        check(self._L.icempm_harvest_begin(self.h, int(capacity), int(stride)))
        self._harvest_cap = int(capacity)

    def prepare_frame(self, elapsed_steps, colors=None):
        """Saved-frame grid arrays (icempm_prepare_frame) as numpy arrays."""
        out = {k: np.zeros(self.G, np.float32) for k in FRAME_CHANNELS}
        out["rgb"] = np.zeros(3 * self.G, np.uint8)
        out["mass_mask"] = np.zeros(self.G, np.uint8)
        out["count"] = np.zeros(self.G, np.uint8)
        out["forces_per_region"] = np.zeros(2 * 100, np.float32)
        fb = FrameBuffers()
        for k in FRAME_CHANNELS + ("forces_per_region",):
            setattr(fb, k, out[k].ctypes.data_as(C.POINTER(C.c_float)))
        for k in ("rgb", "mass_mask", "count"):
            setattr(fb, k, out[k].ctypes.data_as(C.POINTER(C.c_uint8)))
        cp, nc = None, 0
        if colors is not None:
            colors = np.ascontiguousarray(colors, np.uint32)
            cp, nc = colors.ctypes.data_as(C.POINTER(C.c_uint32)), len(colors)
        check(self._L.icempm_prepare_frame(self.h, cp, nc, int(elapsed_steps), C.byref(fb)))
        return out

    def harvest_end(self):
        """The recorded (trial, projected) pairs as float32 [count, 8], and how many were offered."""
        cap = self._harvest_cap
        rec = np.zeros((cap, 8), np.float32)
        cnt = C.c_uint32(0)
        check(self._L.icempm_harvest_end(self.h, rec.ctypes.data_as(C.POINTER(C.c_float)), cap, C.byref(cnt)))
        return rec[:min(cnt.value, cap)], cnt.value

    def __init__(self, prms: SimParams, grid_status: np.ndarray, current=None, capacity: int = 0,
                 options: Options = None):
        L = load()
        self._L = L
        self.prms = prms.copy()
        self.options = options if options is not None else Options.default()
        st = np.ascontiguousarray(grid_status, dtype=np.uint8)
        assert st.size == prms.GridXTotal * prms.GridYTotal
        cur = None if current is None else np.ascontiguousarray(current, dtype=np.float64)
        self.G = prms.GridXTotal * prms.GridYTotal
        h = C.c_void_p()
        check(L.icempm_create(C.byref(self.prms), st.ctypes.data_as(C.POINTER(C.c_uint8)), _dp(cur),
                              int(capacity), C.byref(self.options), C.byref(h)))
        self.h = h
        self.capacity = int(capacity)

    def close(self):
        if getattr(self, "h", None):
            self._L.icempm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, soa: np.ndarray, n: int, disabled: int = 0):
        assert soa.shape[0] == N_PTS_ARRAYS
        check(self._L.icempm_upload_points(self.h, _dp(soa), soa.shape[1], int(n), int(disabled)))

    def update_constants(self, prms: SimParams):
        self.prms = prms.copy()
        check(self._L.icempm_update_constants(self.h, C.byref(self.prms)))

    def set_current(self, current):
        cur = None if current is None else np.ascontiguousarray(current, dtype=np.float64)
        check(self._L.icempm_set_current(self.h, _dp(cur)))

    def set_flow_frames(self, current_a, current_b=None):
        """Current frames a, b ([2G] doubles each, vx block then vy block)."""
        a = None if current_a is None else np.ascontiguousarray(current_a, dtype=np.float64)
        b = None if current_b is None else np.ascontiguousarray(current_b, dtype=np.float64)
        for x in (a, b):
            if x is not None and x.size != 2 * self.G:
                raise ValueError(f"current frame holds {x.size} values, expected {2 * self.G}")
        check(self._L.icempm_set_flow_frames(self.h, _dp(a), _dp(b)))

    def set_wind_frames(self, wind, cell=1.0, x0=0.0, y0=0.0):
        """Wind frames float32 [rows, cols, 4] = {u_a, v_a, u_b, v_b}; None drops them."""
        if wind is None:
            check(self._L.icempm_set_wind_frames(self.h, None, 0, 0, 1.0, 0.0, 0.0))
            return
        w = np.ascontiguousarray(wind, dtype=np.float32)
        if w.ndim != 3 or w.shape[2] != 4:
            raise ValueError("wind frames must be [rows, cols, 4]")
        self._wind = w
        check(self._L.icempm_set_wind_frames(self.h, w.ctypes.data_as(C.POINTER(C.c_float)), w.shape[0],
                                             w.shape[1], float(cell), float(x0), float(y0)))

    def set_forcing_time(self, tc, tw=None):
        check(self._L.icempm_set_forcing_time(self.h, float(tc), float(tc if tw is None else tw)))

    def get_forcing(self):
        """(current [2G], wind stress [2G]) as the sub-steps read them."""
        cur, st = np.zeros(2 * self.G), np.zeros(2 * self.G)
        check(self._L.icempm_get_forcing(self.h, _dp(cur), _dp(st)))
        return cur, st

    def step(self, nsteps: int, first_step: int = 0):
        check(self._L.icempm_step(self.h, int(nsteps), int(first_step)))

    def download(self, soa: np.ndarray = None) -> tuple:
        if soa is None:
            soa = np.zeros((N_PTS_ARRAYS, max(self.count(), 1)), np.float64)
        n = C.c_uint32(0)
        check(self._L.icempm_download_points(self.h, _dp(soa), soa.shape[1], C.byref(n)))
        return soa, n.value

    def download_async(self, soa: np.ndarray) -> int:
        """Start the download into `soa` (keep it alive and unread until
        download_wait); returns the point count."""
        if soa.dtype != np.float64 or not soa.flags.c_contiguous or soa.ndim != 2 or soa.shape[0] != N_PTS_ARRAYS:
            raise ValueError("soa must be a C-contiguous float64 [19, capacity] array")
        n = C.c_uint32(0)
        check(self._L.icempm_download_points_async(self.h, _dp(soa), soa.shape[1], C.byref(n)))
        self._pending = soa
        return n.value

    def download_wait(self):
        check(self._L.icempm_download_wait(self.h))
        self._pending = None

    def tune_sort_cadence(self, trial_steps: int, first_step: int = 0) -> int:
        """Measure and set the locality re-sort cadence (advances the scene
        2 * trial_steps sub-steps); returns it (0: no periodic sort)."""
        k = C.c_int32(0)
        check(self._L.icempm_tune_sort_cadence(self.h, int(trial_steps), int(first_step), C.byref(k)))
        return k.value

    def set_learned_map(self, params_ptr, norm_ptr, tol: float):
        """Put the learned return map on the step path (device pointers to the
        FP32 parameters and the 14-float normalisation; params_ptr None: off)."""
        check(self._L.icempm_set_learned_map(self.h, params_ptr, norm_ptr, float(tol)))

    def learned_map_counts(self) -> tuple:
        """(answers kept, exact fallbacks) of the learned map since it was set."""
        a, b = C.c_uint64(0), C.c_uint64(0)
        check(self._L.icempm_learned_map_counts(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def debug_barrier_timeout(self, extra_bytes: int, wait_limit_us: int):
        """Test hook: make the fused kernel's chunk barriers expect extra_bytes
        more than their copies deliver, with a wait limit of wait_limit_us
        ((0, 0) restores the production setting)."""
        check(self._L.icempm_debug_barrier_timeout(self.h, int(extra_bytes), int(wait_limit_us)))

    def status(self) -> tuple:
        e, d = C.c_uint32(0), C.c_int32(0)
        check(self._L.icempm_get_status(self.h, C.byref(e), C.byref(d)))
        return e.value, d.value

    def clear_force_accumulator(self):
        check(self._L.icempm_clear_force_accumulator(self.h))

    def boundary_forces(self, elapsed_steps: int, out: np.ndarray = None) -> np.ndarray:
        """Boundary forces / (elapsed_steps * dt), fx block then fy block;
        `out` (2 G doubles, e.g. page-locked) is filled when given."""
        if out is None:
            out = np.empty(2 * self.G)
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size != 2 * self.G:
            raise ValueError(f"out must be a C-contiguous float64 array of {2 * self.G} values")
        check(self._L.icempm_get_boundary_forces(self.h, _dp(out), int(elapsed_steps)))
        return out

    def sort_compact(self):
        check(self._L.icempm_sort_compact(self.h))

    def timings(self):
        ms = (C.c_float * 4)()
        check(self._L.icempm_timings(self.h, ms))
        return list(ms)

    def phase_times(self, nsteps: int):
        u, f = C.c_float(0), C.c_float(0)
        check(self._L.icempm_phase_times(self.h, int(nsteps), C.byref(u), C.byref(f)))
        return u.value, f.value

    def fixed_point_scales(self):
        a, b = C.c_double(0), C.c_double(0)
        check(self._L.icempm_fixed_point_scales(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def count(self) -> int:
        n = C.c_uint32(0)
        check(self._L.icempm_point_count(self.h, C.byref(n)))
        return n.value

    def stream(self) -> int:
        s = C.c_void_p()
        check(self._L.icempm_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def launch_count(self) -> int:
        c = C.c_uint64(0)
        check(self._L.icempm_launch_count(self.h, C.byref(c)))
        return c.value


class Batch:
    """Ensemble of contexts (same variant, same device) advanced together:
    one launch of each kernel per sub-step for all scenes.  The contexts must
    outlive the batch."""

    def __init__(self, contexts):
        L = load()
        self._L = L
        self.contexts = list(contexts)
        arr = (C.c_void_p * max(1, len(self.contexts)))(*[c.h.value for c in self.contexts])
        h = C.c_void_p()
        check(L.icempm_batch_create(C.cast(arr, C.POINTER(C.c_void_p)), len(self.contexts), C.byref(h)))
        self.h = h

    def step(self, nsteps, first_step=0):
        check(self._L.icempm_batch_step(self.h, int(nsteps), int(first_step)))

    def autotune(self, trial_steps=100, first_step=0):
        t = BatchTuning()
        check(self._L.icempm_batch_autotune(self.h, int(trial_steps), int(first_step), C.byref(t)))
        return t

    def set_tuning(self, tuning):
        check(self._L.icempm_batch_set_tuning(self.h, C.byref(tuning)))

    def tuning(self):
        t = BatchTuning()
        check(self._L.icempm_batch_get_tuning(self.h, C.byref(t)))
        return t

    def timings(self):
        ms = (C.c_float * 4)()
        check(self._L.icempm_batch_timings(self.h, ms))
        return list(ms)

    def launch_count(self):
        v = C.c_uint64()
        check(self._L.icempm_batch_launch_count(self.h, C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "h", None):
            self._L.icempm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
