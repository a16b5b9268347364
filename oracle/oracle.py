"""ctypes front-end of the FP64 CPU oracle (oracle/icempm_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the
benchmark's CPU-baseline leg, as the checker.  It restates the reference step
(simulation/kernels.cuh, helper_math.cuh, givens.cuh; igorg520b/iceMPM_2d_sp);
each C function cites the reference lines it follows.

Arrays are numpy: the HSSOA is float64 [19, capacity] (row j of point i at
[j, i]); the grid is float64 [9, G] with node = y + x*GridY.
"""
import ctypes as C
import os

import numpy as np

from icempm_2d_sp_b200.params import SimParams, Options, N_PTS_ARRAYS, N_GRID_ARRAYS
from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        L = C.CDLL(path)
        dp, u8p = C.POINTER(C.c_double), C.POINTER(C.c_uint8)
        sp = C.POINTER(SimParams)
        L.orc_compute_helpers.argtypes = [sp]
        L.orc_reset_params.argtypes = [sp]
        L.orc_svd2x2.argtypes = [dp, dp, dp, dp]
        L.orc_compute_pq.argtypes = [sp, dp, dp, dp, dp]
        L.orc_kirchhoff.argtypes = [sp, dp, dp]
        L.orc_weights.argtypes = [dp, dp]
        L.orc_failure_check.argtypes = [sp, C.c_uint32, C.c_double, C.c_double]
        L.orc_failure_check.restype = C.c_uint32
        L.orc_wolper_dp.argtypes = [sp, C.c_double, C.c_double, C.c_double, C.c_double,
                                    dp, dp, dp, dp, dp, dp, C.POINTER(C.c_int)]
        L.orc_wolper_dp.restype = C.c_int
        L.orc_p2g.argtypes = [sp, dp, C.c_size_t, C.c_size_t, dp, C.c_size_t, C.POINTER(Options)]
        L.orc_p2g.restype = C.c_uint32
        L.orc_update_nodes.argtypes = [sp, dp, C.c_size_t, u8p, C.c_double]
        L.orc_update_nodes.restype = C.c_uint32
        L.orc_update_nodes_ext.argtypes = [sp, dp, C.c_size_t, u8p]
        L.orc_update_nodes_ext.restype = C.c_uint32
        L.orc_g2p.argtypes = [sp, dp, C.c_size_t, C.c_size_t, dp, C.c_size_t, C.c_int,
                              C.POINTER(C.c_int32)]
        L.orc_g2p.restype = C.c_uint32
        L.orc_run_steps.argtypes = [sp, C.POINTER(Options), dp, C.c_size_t, C.c_size_t, dp,
                                    C.c_size_t, u8p, C.c_int, C.c_int, C.POINTER(C.c_int32)]
        L.orc_run_steps.restype = C.c_uint32
        L.orc_remove_disabled_and_sort.argtypes = [dp, C.c_size_t, C.c_size_t, C.c_int]
        L.orc_remove_disabled_and_sort.restype = C.c_size_t
        L.orc_num_threads.restype = C.c_int
        L.orc_set_num_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _dp(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _u8p(a):
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def compute_helpers(p: SimParams) -> SimParams:
    lib().orc_compute_helpers(C.byref(p))
    return p


def svd2x2(F):
    """F row-major 2x2 -> (U, S, V) as the reference's svd2x2 returns them."""
    F = np.ascontiguousarray(np.asarray(F, dtype=np.float64).reshape(4))
    U, S, V = np.zeros(4), np.zeros(2), np.zeros(4)
    lib().orc_svd2x2(_dp(F), _dp(U), _dp(S), _dp(V))
    return U.reshape(2, 2), S, V.reshape(2, 2)


def compute_pq(p, F):
    F = np.ascontiguousarray(np.asarray(F, dtype=np.float64).reshape(4))
    Je, pp, qq = C.c_double(), C.c_double(), C.c_double()
    lib().orc_compute_pq(C.byref(p), _dp(F), C.byref(Je), C.byref(pp), C.byref(qq))
    return Je.value, pp.value, qq.value


def kirchhoff(p, F):
    F = np.ascontiguousarray(np.asarray(F, dtype=np.float64).reshape(4))
    out = np.zeros(4)
    lib().orc_kirchhoff(C.byref(p), _dp(F), _dp(out))
    return out.reshape(2, 2)


def weights(pos):
    pos = np.ascontiguousarray(np.asarray(pos, dtype=np.float64).reshape(2))
    ww = np.zeros(6)
    lib().orc_weights(_dp(pos), _dp(ww))
    return ww.reshape(3, 2)


def failure_check(p, utility, pp, q):
    return lib().orc_failure_check(C.byref(p), int(utility), float(pp), float(q))


def wolper_dp(p, thickness, p_tr, q_tr, Je_tr, U, V, sig2, shat, Fe, Jp_inv):
    """Returns (case, Fe_new (2x2), Jp_inv_new, nan_flag)."""
    U = np.ascontiguousarray(np.asarray(U, np.float64).reshape(4))
    V = np.ascontiguousarray(np.asarray(V, np.float64).reshape(4))
    sig2 = np.ascontiguousarray(np.asarray(sig2, np.float64).reshape(2))
    shat = np.ascontiguousarray(np.asarray(shat, np.float64).reshape(2))
    Fe = np.ascontiguousarray(np.array(Fe, np.float64).reshape(4))
    jp = C.c_double(Jp_inv)
    nanf = C.c_int(0)
    case = lib().orc_wolper_dp(C.byref(p), thickness, p_tr, q_tr, Je_tr, _dp(U), _dp(V),
                               _dp(sig2), _dp(shat), _dp(Fe), C.byref(jp), C.byref(nanf))
    return case, Fe.reshape(2, 2), jp.value, nanf.value


def new_grid(p: SimParams, status=None, current=None):
    G = p.GridXTotal * p.GridYTotal
    grid = np.zeros((N_GRID_ARRAYS, G), np.float64)
    if current is not None:
        grid[5] = current[:G]
        grid[6] = current[G:2 * G]
    return grid


def p2g(p, soa, n, grid, opts=None):
    """P2G into grid rows 0-2; opts with extended forcing adds the stress impulses."""
    ext = C.byref(opts) if (opts is not None and opts.forcing == 1) else None
    return lib().orc_p2g(C.byref(p), _dp(soa), soa.shape[1], n, _dp(grid), grid.shape[1], ext)


def update_nodes(p, grid, status, t):
    return lib().orc_update_nodes(C.byref(p), _dp(grid), grid.shape[1], _u8p(status), float(t))


def update_nodes_ext(p, grid, status):
    return lib().orc_update_nodes_ext(C.byref(p), _dp(grid), grid.shape[1], _u8p(status))


def g2p(p, soa, n, grid, recordPQ):
    dis = C.c_int32(0)
    err = lib().orc_g2p(C.byref(p), _dp(soa), soa.shape[1], n, _dp(grid), grid.shape[1],
                        int(bool(recordPQ)), C.byref(dis))
    return err, dis.value


def run_steps(p, soa, n, grid, status, nsteps, first_step=0, opts=None):
    """Runs the reference sub-step loop (model.cpp:18-39).  Mutates soa and grid.
    Returns (error_bits, newly_disabled_count)."""
    dis = C.c_int32(0)
    op = C.byref(opts) if opts is not None else None
    err = lib().orc_run_steps(C.byref(p), op, _dp(soa), soa.shape[1], n, _dp(grid),
                              grid.shape[1], _u8p(status), int(nsteps), int(first_step),
                              C.byref(dis))
    return err, dis.value


def remove_disabled_and_sort(soa, n, gridY):
    return lib().orc_remove_disabled_and_sort(_dp(soa), soa.shape[1], n, gridY)
