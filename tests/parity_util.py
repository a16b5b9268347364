"""Comparison metrics between two HSSOA states (reference layout, float64 [19, cap])."""
import numpy as np

from icempm_2d_sp_b200 import hssoa as H
from icempm_2d_sp_b200.params import IDX_UTILITY, IDX_CELL, IDX_POINT, STATUS_CRUSHED, STATUS_DISABLED


def world(soa, n, h):
    c = H.get_u32(soa, IDX_CELL, n).astype(np.int64)
    return ((soa[6, :n] + (c & 0xffff)) * h, (soa[7, :n] + (c >> 16)) * h)


def errors(got, ref, n, h):
    """Error measures used by the parity tests:
    pos_cells   max |x - x_ref| in cell units (world position / h)
    pos_rel     max |x - x_ref| / max |x_ref| over world positions
    vel_rel     max |v - v_ref| / max |v_ref|
    fe_abs      max |Fe - Fe_ref|
    bp_rel      max |Bp - Bp_ref| / max |Bp_ref|
    jp_rel      max |Jp - Jp_ref| / max |Jp_ref|
    pq_rel      max |P,Q - ref| / max |P,Q ref|
    flags_mismatch  points whose utility word differs
    cell_mismatch   points whose cell key differs
    """
    gx, gy = world(got, n, h)
    rx, ry = world(ref, n, h)
    dpos = np.hypot(gx - rx, gy - ry)
    rpos = np.hypot(rx, ry).max()
    dv = np.hypot(got[8, :n] - ref[8, :n], got[9, :n] - ref[9, :n])
    vref = max(np.hypot(ref[8, :n], ref[9, :n]).max(), 1e-30)
    bp = np.abs(got[14:18, :n] - ref[14:18, :n]).max()
    bpr = max(np.abs(ref[14:18, :n]).max(), 1e-30)
    pq = np.abs(got[3:5, :n] - ref[3:5, :n]).max()
    pqr = max(np.abs(ref[3:5, :n]).max(), 1e-30)
    return dict(
        pos_cells=float(dpos.max() / h),
        pos_rel=float(dpos.max() / max(rpos, 1e-30)),
        vel_rel=float(dv.max() / vref),
        fe_abs=float(np.abs(got[10:14, :n] - ref[10:14, :n]).max()),
        bp_rel=float(bp / bpr),
        jp_rel=float(np.abs(got[5, :n] - ref[5, :n]).max() / max(np.abs(ref[5, :n]).max(), 1e-30)),
        pq_rel=float(pq / pqr),
        flags_mismatch=int((H.get_u32(got, IDX_UTILITY, n) != H.get_u32(ref, IDX_UTILITY, n)).sum()),
        cell_mismatch=int((H.get_u32(got, IDX_CELL, n) != H.get_u32(ref, IDX_CELL, n)).sum()),
        pid_equal=bool(np.array_equal(H.get_u32(got, IDX_POINT, n), H.get_u32(ref, IDX_POINT, n))),
        thickness_equal=bool(np.array_equal(got[18, :n], ref[18, :n])),
    )


def aggregates(soa, n, prms):
    """Total mass, momentum and kinetic energy of the enabled points."""
    en = (H.get_u32(soa, IDX_UTILITY, n) & STATUS_DISABLED) == 0
    m = prms.ParticleMass * soa[18, :n][en]
    vx, vy = soa[8, :n][en], soa[9, :n][en]
    return dict(mass=float(m.sum()), px=float((m * vx).sum()), py=float((m * vy).sum()),
                ke=float(0.5 * (m * (vx * vx + vy * vy)).sum()))
