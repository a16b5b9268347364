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


def test_noalloc_rejects_oversize_without_touching_memory():
    from icempm_2d_sp_b200 import capi
    L = capi.load()
    rc = L.icempm_cell_order_noalloc(None, None, (1 << 20) + 1, 8, None, None, None)
    assert rc == -5 and b"ICEMPM_NOALLOC_MAX_POINTS" in L.icempm_last_error()
