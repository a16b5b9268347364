"""CPU restatement of the time-varying forcing tables (test infrastructure:
the checker of k_blend_forcing, never on the product path).

The reference has no finished counterpart: SetTime is a stub
(simulation/data_manager/windandcurrentinterpolator.cpp:66-70) and the wind
interpolation is commented out (get_wind_vector, simulation/kernels.cuh:580-622).
This restatement follows that commented function -- bilinear weights
(1-u)(1-v), u(1-v), (1-u)v, uv of the position inside the wind cell over
samples wgrid[r][c], wgrid[r][c+1], wgrid[r+1][c], wgrid[r+1][c+1], then
(1-tb) W_a + tb W_b -- with positions clamped to the wind grid, and the
current blended as (1-tc) a + tc b.  Operations are evaluated in float64 in
the same order as the device kernel, so the tables agree bit for bit before
the final rounding to the engine's state type.  Parity unpinned (no
reference output exists for this path).
"""
import numpy as np


def blend_current(a, b, tc):
    """(1 - tc) a + tc b per entry (2 G doubles each)."""
    t1 = 1.0 - tc
    return t1 * np.asarray(a, np.float64) + tc * np.asarray(b, np.float64)


def wind_at(wind, cell, x0, y0, X, Y, tw):
    """Wind at world positions X, Y from frames wind[rows, cols, 4] = {u_a,
    v_a, u_b, v_b} (float32)."""
    rows, cols = wind.shape[:2]
    u = (np.asarray(X, np.float64) - x0) / cell
    v = (np.asarray(Y, np.float64) - y0) / cell
    u = np.minimum(np.maximum(u, 0.0), float(cols - 1))
    v = np.minimum(np.maximum(v, 0.0), float(rows - 1))
    c = np.minimum(u.astype(np.int64), max(cols - 2, 0))
    r = np.minimum(v.astype(np.int64), max(rows - 2, 0))
    c1 = np.minimum(c + 1, cols - 1)
    r1 = np.minimum(r + 1, rows - 1)
    ub, vb = u - c, v - r
    w00 = (1.0 - ub) * (1.0 - vb)
    w01 = ub * (1.0 - vb)
    w10 = (1.0 - ub) * vb
    w11 = ub * vb
    W = np.asarray(wind, np.float32).astype(np.float64)

    def bil(k):
        return ((w00 * W[r, c, k] + w01 * W[r, c1, k]) + w10 * W[r1, c, k]) + w11 * W[r1, c1, k]
    t1 = 1.0 - tw
    ux = t1 * bil(0) + tw * bil(2)
    uy = t1 * bil(1) + tw * bil(3)
    return ux, uy


def forcing_tables(gx, gy, h, air_ca, cur_a=None, cur_b=None, tc=0.0, wind=None, cell=1.0, x0=0.0, y0=0.0,
                   tw=0.0, real=np.float32):
    """(current [2G], wind stress [2G]) as the engine holds them (rounded to
    `real`, returned as float64); entries without frames are None."""
    G = gx * gy
    cur = st = None
    if cur_a is not None:
        cur = blend_current(cur_a, cur_a if cur_b is None else cur_b, tc).astype(real).astype(np.float64)
    if wind is not None:
        i = np.arange(G)
        X = (i // gy).astype(np.float64) * h
        Y = (i % gy).astype(np.float64) * h
        ux, uy = wind_at(wind, cell, x0, y0, X, Y, tw)
        um = np.sqrt(ux * ux + uy * uy)
        k = air_ca * um
        st = np.concatenate([(k * ux).astype(real), (k * uy).astype(real)]).astype(np.float64)
    return cur, st
