"""icempm_cell_order_noalloc -- the entry point for callers that may not
allocate device memory -- against the existing compaction entry point.

This file sorts last on purpose (pytest collects files in name order), so a
run that stops at its first failure has run every other test before it.  The
test passes on its own in a fresh process (the first call does the per-device
set-up) and after the rest of the suite (the static scratch is reused).
"""
import ctypes as C
import os

import numpy as np
import pytest

from icempm_2d_sp_b200 import scenes, hssoa as H
from icempm_2d_sp_b200.params import SimParams, Options, IDX_UTILITY, IDX_CELL, STATUS_DISABLED

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def compact_with_context(capi, prms, status, current, soa, n):
    """The existing entry point: upload, icempm_sort_compact, download (FP64
    variant: bit-exact round trip)."""
    with capi.Context(prms, status, current, capacity=soa.shape[1],
                      options=Options.default(variant="fp64")) as ctx:
        ctx.upload(soa, n)
        ctx.sort_compact()
        out, m = ctx.download(np.zeros_like(soa))
    return out, m


def order_noalloc(capi, soa, n, grid_y):
    """Device inputs/outputs from torch; the entry point itself allocates nothing."""
    import torch
    L = capi.load()
    cell = torch.from_numpy(H.get_u32(soa, IDX_CELL, n).copy().view(np.int32)).cuda()
    util = torch.from_numpy(H.get_u32(soa, IDX_UTILITY, n).copy().view(np.int32)).cuda()
    order = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    count = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = L.icempm_cell_order_noalloc(cell.data_ptr(), util.data_ptr(), n, grid_y, order.data_ptr(),
                                     count.data_ptr(), None)
    assert rc == 0, L.icempm_last_error()
    torch.cuda.synchronize()
    return order.cpu().numpy().view(np.uint32)[:n], int(count.cpu().numpy().view(np.uint32)[0])


def test_noalloc_order_matches_sort_compact_twice():
    from icempm_2d_sp_b200 import capi
    capi.load()
    if capi.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    z = np.load(os.path.join(GOLDEN, "disable_then_sort.npz"))
    prms = SimParams.from_buffer_copy(z["prms"].tobytes())
    first = (prms, z["status"], z["current"], np.ascontiguousarray(z["soa_out"]), int(z["n"]))
    sc = scenes.random_state(seed=41, gx=48, gy=40)
    soa2 = sc.soa.copy()
    rng = np.random.default_rng(0)
    util = H.get_u32(soa2, IDX_UTILITY, sc.n).copy()
    util[rng.random(sc.n) < 0.2] |= STATUS_DISABLED
    H.set_u32(soa2, IDX_UTILITY, util, sc.n)
    second = (sc.prms, sc.status, sc.current, soa2, sc.n)
    assert int((H.get_u32(first[3], IDX_UTILITY, first[4]) & STATUS_DISABLED != 0).sum()) > 0
    for prms_i, status, current, soa, n in (first, second):       # two calls in a row
        ref, m = compact_with_context(capi, prms_i, status, current, soa, n)
        order, count = order_noalloc(capi, soa, n, prms_i.GridYTotal)
        assert count == m
        got = soa[:, order[:count]]
        # integer work: the reordered points are identical bit for bit
        assert np.array_equal(got.view(np.uint64), ref[:, :m].view(np.uint64))


def _pts(seed, n, disabled_frac, gx=48, gy=40):
    """n points on random cells of a gx x gy grid (several per cell), a
    fraction of them disabled; only the cell and utility rows matter here."""
    rng = np.random.default_rng(seed)
    soa = np.zeros((19, max(n, 1)))
    cx = rng.integers(2, gx - 2, n).astype(np.uint32)
    cy = rng.integers(2, gy - 2, n).astype(np.uint32)
    H.set_u32(soa, IDX_CELL, (cy << 16) | cx, n)
    util = np.where(rng.random(n) < disabled_frac, STATUS_DISABLED, 0).astype(np.uint32)
    H.set_u32(soa, IDX_UTILITY, util, n)
    return soa


def expected_order(soa, n, grid_y):
    """The compaction order by definition: enabled points, stable by cell index x*grid_y + y."""
    cell = H.get_u32(soa, IDX_CELL, n).astype(np.int64)
    util = H.get_u32(soa, IDX_UTILITY, n)
    idx = np.nonzero((util & STATUS_DISABLED) == 0)[0]
    key = (cell[idx] & 0xffff) * grid_y + (cell[idx] >> 16)
    return idx[np.argsort(key, kind="stable")].astype(np.uint32)


@pytest.mark.parametrize("n,disabled_frac", [(0, 0.0), (100, 0.3), (257, 1.0), (5000, 0.1)])
def test_noalloc_edge_sizes_twice(n, disabled_frac):
    """No points, a small set (the sort's single-tile path), every point
    disabled, and a few thousand points: the count and the order, bit for bit,
    on two calls in a row."""
    from icempm_2d_sp_b200 import capi
    capi.load()
    if capi.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    soa = _pts(7 + n, n, disabled_frac)
    want = expected_order(soa, n, 40)
    for _ in range(2):
        order, count = order_noalloc(capi, soa, n, 40)
        assert count == len(want)
        assert np.array_equal(order[:count], want)
