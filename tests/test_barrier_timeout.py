"""The bounded barrier wait of the fused kernel runs out and reports, without
a fault: through the C ABI the test makes every chunk barrier expect 16 bytes
more than its bulk copies deliver (icempm_debug_barrier_timeout), so the wait
gives up after its 2 ms limit although every copy has landed.  The step must
return with ICEMPM_ERR_BARRIER_TIMEOUT in the status word within a bounded
time, and the context must step normally again once the hook is off and the
error word is cleared."""
import time

import numpy as np
import pytest

from icempm_2d_sp_b200 import scenes
from icempm_2d_sp_b200.params import Options

ERR_BARRIER_TIMEOUT = 0x2000


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["fixed", "fp32"])
def test_barrier_wait_runs_out_and_reports(variant):
    from icempm_2d_sp_b200 import capi
    capi.load()
    if capi.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    sc = scenes.random_state(seed=5, gx=64, gy=48)
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n,
                      options=Options.default(variant=variant, use_graphs=0)) as ctx:
        ctx.upload(sc.soa, sc.n)
        ctx.step(2, 0)
        assert ctx.status()[0] == 0
        before, _ = ctx.download(np.zeros_like(sc.soa))
        ctx.debug_barrier_timeout(16, 2000)
        t0 = time.perf_counter()
        ctx.step(1, 2)
        err, _ = ctx.status()
        dt = time.perf_counter() - t0
        assert err & ERR_BARRIER_TIMEOUT
        assert dt < 5.0
        # every CTA left at its first chunk: no point was advanced
        after, _ = ctx.download(np.zeros_like(sc.soa))
        assert np.array_equal(after[6:10, :sc.n], before[6:10, :sc.n])
        ctx.debug_barrier_timeout(0, 0)
        ctx.update_constants(sc.prms)          # clears the error word, re-primes the scatter
        ctx.step(3, 3)
        err, _ = ctx.status()
        assert err == 0
        moved, _ = ctx.download(np.zeros_like(sc.soa))
        assert not np.array_equal(moved[6:10, :sc.n], before[6:10, :sc.n])


def test_hook_rejects_unaligned_byte_count():
    """Byte counts that are not whole 16-byte units are refused on the host."""
    from icempm_2d_sp_b200 import capi
    L = capi.load()
    rc = L.icempm_debug_barrier_timeout(None, 8, 1000)
    assert rc < 0 and b"multiple of 16" in L.icempm_last_error()
