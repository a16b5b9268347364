"""Ensembles (icempm_batch_*): many scenes advanced by one launch of each kernel
per sub-step.  A batch must leave every scene exactly where stepping it alone
leaves it -- bit for bit in the fixed-point form, whose sums do not depend on
the order of the atomics -- with each scene's own error word and disabled count.
"""
import numpy as np
import pytest

from icempm_2d_sp_b200 import scenes
from icempm_2d_sp_b200.params import Options, IDX_VELX

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    from icempm_2d_sp_b200 import capi as C
    C.load()
    if C.device_count() < 1:
        pytest.fail("no CUDA device visible to the library")
    return C


@pytest.fixture(scope="module")
def small_ensemble():
    return scenes.ensemble(n_scenes=5, seed=11, n_min=10_000, n_max=120_000)


def options_of(sc, variant="fixed"):
    o = Options.default(variant=variant, forcing=sc.options.forcing)
    for f in ("wind_kind", "wind_u", "wind_v", "wind_cx", "wind_cy", "wind_vmax", "wind_radius"):
        setattr(o, f, getattr(sc.options, f))
    return o


def open_contexts(capi, scs, variant="fixed", soas=None):
    ctxs = []
    for k, sc in enumerate(scs):
        c = capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=options_of(sc, variant))
        c.upload(sc.soa if soas is None else soas[k], sc.n)
        ctxs.append(c)
    return ctxs


def state(ctx, sc):
    out, m = ctx.download(np.zeros_like(sc.soa))
    err, dis = ctx.status()
    return out[:, :m], err, dis


def test_batch_matches_contexts_stepped_alone(capi, small_ensemble):
    scs = small_ensemble
    alone = []
    for c, sc in zip(open_contexts(capi, scs), scs):
        c.step(37, 0)
        alone.append(state(c, sc))
        c.close()
    ctxs = open_contexts(capi, scs)
    with capi.Batch(ctxs) as b:
        b.step(37, 0)
        assert b.timings()[0] > 0 and b.launch_count() > 0
    for c, sc, (ref, rerr, rdis) in zip(ctxs, scs, alone):
        got, err, dis = state(c, sc)
        assert err == rerr and dis == rdis
        assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
        c.close()


def test_graphs_and_direct_launches_agree(capi, small_ensemble):
    scs = small_ensemble[:3]
    results = []
    for graph_steps in (0, 50):
        ctxs = open_contexts(capi, scs)
        with capi.Batch(ctxs) as b:
            t = b.tuning()
            t.graph_steps = graph_steps
            b.set_tuning(t)
            b.step(120, 5)
            b.step(30, 125)      # a second call continues the sub-step indices
        results.append([state(c, sc) for c, sc in zip(ctxs, scs)])
        for c in ctxs:
            c.close()
    for (a, ea, da), (g, eg, dg) in zip(*results):
        assert ea == eg and da == dg and np.array_equal(a.view(np.uint64), g.view(np.uint64))


def test_autotune_picks_a_supported_form_and_stepping_goes_on(capi, small_ensemble):
    scs = small_ensemble
    ctxs = open_contexts(capi, scs)
    with capi.Batch(ctxs) as b:
        t = b.autotune(trial_steps=50, first_step=0)
        assert (t.tile_nodes, t.stages) in [(0, 2), (0, 1), (512, 1), (1024, 1)]
        assert t.sort_every in (0, 100, 400) and t.graph_steps == 50 and t.ms_per_step > 0
        b.step(60, 200)
    for c, sc in zip(ctxs, scs):
        _, err, _ = state(c, sc)
        assert err == 0
        c.close()


def test_errors_stay_with_their_scene(capi, small_ensemble):
    scs = small_ensemble[:3]
    soas = [sc.soa.copy() for sc in scs]
    soas[1][IDX_VELX, 0] = np.nan          # one NaN velocity in scene 1 only
    ctxs = open_contexts(capi, scs, soas=soas)
    with capi.Batch(ctxs) as b:
        b.step(3, 0)
    errs = [state(c, sc)[1] for c, sc in zip(ctxs, scs)]
    assert errs[0] == 0 and errs[2] == 0 and errs[1] != 0
    for c in ctxs:
        c.close()


def test_batch_rejects_mixed_variants_and_empty(capi, small_ensemble):
    scs = small_ensemble[:2]
    a = open_contexts(capi, scs[:1], "fixed")[0]
    b = open_contexts(capi, scs[1:], "fp32")[0]
    with pytest.raises(capi.IcempmError):
        capi.Batch([a, b])
    with pytest.raises(capi.IcempmError):
        capi.Batch([])
    a.close()
    b.close()
