"""Small drivers that run one family of kernels on a fixed workload, for
profiling with ncu (they print one line and check nothing beyond the device
error bits).

    python tests/kernel_drivers.py ensemble [n_scenes]   # k_g2p_p2g_batch, k_grid_update_batch
    python tests/kernel_drivers.py frame [small]         # k_frame_scatter, k_frame_finish, k_blend_forcing
    python tests/kernel_drivers.py learned               # k_return_map_learned, k_return_map_exact

ensemble: the first n_scenes (default 24) scenes of the ensemble generator in
one batch, the default kernel shape (no shared tile, two stages), direct
launches, 5 + 3 sub-steps.
frame: the floe-field scene (4096x2048, 23.0M points; `small`: the same rules
on 2048x1024), 2 sub-steps, two current frames and a 64x128 wind grid, then
three rounds of prepare_frame, set_forcing_time and get_forcing.
learned: projections harvested from 40 sub-steps of a 256x128 ridging scene,
a network trained on them for 4 epochs, then the batch maps on 10M trial
states (the harvested ones repeated; every row a projection): the exact map
and the learned map at tolerance 1e-2, three calls each.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from icempm_2d_sp_b200 import capi, scenes  # noqa: E402
from icempm_2d_sp_b200.params import Options  # noqa: E402


def ensemble(n_scenes):
    specs = scenes.ensemble_specs(n_scenes)
    scs = [scenes.ensemble_scene(**s) for s in specs]
    ctxs = []
    for sc in scs:
        o = Options.default(variant="fixed", forcing=sc.options.forcing, use_graphs=0)
        for f in ("wind_kind", "wind_u", "wind_v"):
            setattr(o, f, getattr(sc.options, f))
        c = capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o)
        c.upload(sc.soa, sc.n)
        ctxs.append(c)
    try:
        with capi.Batch(ctxs) as b:
            t = capi.BatchTuning()
            t.tile_nodes, t.stages, t.sort_every, t.graph_steps = 0, 2, 0, 0
            b.set_tuning(t)
            b.step(5, 0)
            b.step(3, 5)
            ms = b.timings()[0] / 3
        errs = [c.status()[0] for c in ctxs]
    finally:
        for c in ctxs:
            c.close()
    print(f"scenes {n_scenes} points {sum(s.n for s in scs)} nodes {sum(s.grid_nodes for s in scs)} "
          f"ms per step {ms:.4f} errors {max(errs):#x}")
    return 1 if any(errs) else 0


def frame(small):
    sc = scenes.floe_field(gx=2048, gy=1024, n_seeds=500) if small else scenes.floe_field()
    o = Options.default()
    for f, _ in Options._fields_:
        setattr(o, f, getattr(sc.options, f))
    G = sc.grid_nodes
    rng = np.random.default_rng(0)
    colors = rng.integers(0, 1 << 24, sc.n).astype(np.uint32)
    a, b = rng.normal(0, 0.1, 2 * G), rng.normal(0, 0.1, 2 * G)
    w = rng.normal(0, 10, (64, 128, 4)).astype(np.float32)
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o) as ctx:
        ctx.upload(sc.soa, sc.n)
        ctx.step(2, 0)
        ctx.set_flow_frames(a, b)
        ctx.set_wind_frames(w, cell=64.0)
        for k in range(3):
            ctx.prepare_frame(2, colors)
            ctx.set_forcing_time(0.3 + 0.1 * k, 0.6)
            ctx.get_forcing()
        err = ctx.status()[0]
    print(f"points {sc.n} nodes {G} errors {err:#x}")
    return 1 if err else 0


def learned():
    from icempm_2d_sp_b200 import surrogate
    sc = scenes.ridging(gx=256, gy=128, cells_x=120, cells_y=100, speed=2.0)
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=Options.default()) as ctx:
        ctx.upload(sc.soa, sc.n)
        ctx.harvest_begin(400_000, stride=1)
        ctx.step(40, 0)
        rec, _ = ctx.harvest_end()
    params, norm, _ = surrogate.train(rec, epochs=4)
    trial = np.tile(rec[:, :4], (10_000_000 // len(rec) + 1, 1))[:10_000_000]
    for _ in range(3):
        surrogate.exact_map(sc.prms, trial, fp64=False)
        _, nfb, ms = surrogate.learned_map(sc.prms, params, norm, trial, tol=1e-2)
    print(f"records {len(rec)} rows {len(trial)} learned ms {ms:.3f} fallbacks {nfb}")
    return 0


def main(argv):
    capi.load()
    if len(argv) < 2 or argv[1] not in ("ensemble", "frame", "learned"):
        print(__doc__)
        return 2
    if argv[1] == "ensemble":
        return ensemble(int(argv[2]) if len(argv) > 2 else 24)
    if argv[1] == "learned":
        return learned()
    return frame(len(argv) > 2 and argv[2] == "small")


if __name__ == "__main__":
    sys.exit(main(sys.argv))
