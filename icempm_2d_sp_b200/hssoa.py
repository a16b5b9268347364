"""Host-side SoA (HSSOA) helpers on numpy, in the reference layout.

The reference HostSideSOA (simulation/hssoa/host_side_soa.{h,cpp}) is one
buffer of 19 f64 rows with pitch = capacity; point i, row j is at
buf[i + capacity*j].  Rows 0-2 hold a uint32 in the low 4 bytes of the
double slot (ProxyPoint::getValueInt/setValueInt, proxypoint2d.cpp:115-129).
Here the buffer is a C-contiguous float64 numpy array of shape [19, capacity].
"""
import numpy as np

from .params import (N_PTS_ARRAYS, IDX_UTILITY, IDX_CELL, IDX_POINT, IDX_JP_INV, IDX_POSX,
                     IDX_FE00, IDX_THICKNESS, STATUS_DISABLED)


def allocate(capacity: int) -> np.ndarray:
    """HostSideSOA::Allocate (host_side_soa.cpp:50-75): zero-filled buffer."""
    return np.zeros((N_PTS_ARRAYS, int(capacity)), dtype=np.float64)


def u32_view(soa: np.ndarray, row: int) -> np.ndarray:
    """Writable uint32 view of the low 4 bytes of every slot of `row`."""
    assert soa.dtype == np.float64 and soa.flags.c_contiguous
    return soa.view(np.uint32).reshape(soa.shape[0], soa.shape[1], 2)[row, :, 0]


def get_u32(soa, row, n=None):
    v = u32_view(soa, row)
    return v if n is None else v[:n]


def set_u32(soa, row, values, n=None):
    v = u32_view(soa, row)
    if n is None:
        v[:] = values
    else:
        v[:n] = values


def cell_index(soa, n, grid_y):
    """ProxyPoint::getCellIndex (proxypoint2d.cpp:117-123): x*GridY + y."""
    c = get_u32(soa, IDX_CELL, n).astype(np.int64)
    return (c & 0xffff) * grid_y + (c >> 16)


def world_positions(soa, n, h):
    """ProxyPoint::getPos(cellsize) (proxypoint2d.cpp:141-148)."""
    c = get_u32(soa, IDX_CELL, n).astype(np.int64)
    x = (soa[IDX_POSX, :n] + (c & 0xffff)) * h
    y = (soa[IDX_POSX + 1, :n] + (c >> 16)) * h
    return x, y


def convert_to_integer_cell_format(soa, n, h):
    """ProxyPoint::ConvertToIntegerCellFormat (proxypoint2d.cpp:125-139):
    world positions in rows 6-7 become a cell key (y<<16 | x) and cell-local
    coordinates in [-0.5, 0.5]."""
    hinv = 1.0 / h
    x = soa[IDX_POSX, :n]
    y = soa[IDX_POSX + 1, :n]
    xi = (x * hinv + 0.5).astype(np.uint32)
    yi = (y * hinv + 0.5).astype(np.uint32)
    set_u32(soa, IDX_CELL, (yi << np.uint32(16)) | xi, n)
    soa[IDX_POSX, :n] = x * hinv - xi.astype(np.float64)
    soa[IDX_POSX + 1, :n] = y * hinv - yi.astype(np.float64)


def init_points(world_x, world_y, thickness, h, crushed=None, velocity=None, capacity=None):
    """Fill a new HSSOA the way SnapshotManager::PopulatePoints does
    (snapshotmanager.cpp:216-259): F = I, Jp_inv = 1, P = Q = 0, point id = k."""
    n = len(world_x)
    soa = allocate(capacity if capacity is not None else n)
    soa[IDX_POSX, :n] = world_x
    soa[IDX_POSX + 1, :n] = world_y
    set_u32(soa, IDX_POINT, np.arange(n, dtype=np.uint32), n)
    soa[IDX_THICKNESS, :n] = thickness
    util = np.zeros(n, np.uint32)
    if crushed is not None:
        util[np.asarray(crushed, bool)] |= np.uint32(0x10000)
    set_u32(soa, IDX_UTILITY, util, n)
    soa[IDX_JP_INV, :n] = 1.0
    soa[IDX_FE00, :n] = 1.0
    soa[IDX_FE00 + 3, :n] = 1.0
    if velocity is not None:
        soa[8, :n] = velocity[0]
        soa[9, :n] = velocity[1]
    convert_to_integer_cell_format(soa, n, h)
    return soa


def disabled_mask(soa, n):
    return (get_u32(soa, IDX_UTILITY, n) & STATUS_DISABLED) != 0
