"""Learned return map study (16M-point ridging scene, 8192x2048 grid).

1. Training pairs: projections recorded by the fused kernel from plain-method
   runs -- the floe-field scene (config-1 rules on a 2048x1024 grid, 200
   sub-steps) and 1M-point ridging scenes (1024x512 grid, against the wall at
   1-4 m/s, 1000 sub-steps each) -- up to --pairs records.
2. Training: the library's GPU kernels (icempm_mlp_grad + icempm_mlp_adam),
   minibatch Adam on standardised features.
3. Evaluation: trial states recorded from a 16M-point compressive ridging
   scene (8192x2048 grid, h = 1 m, 2 m/s against the wall, --eval-steps
   sub-steps), mapped by the learned map (BF16 tensor cores, exact fallback
   above the yield residual) and by the exact map (FP32 and FP64): fallback
   rate, error of the answers against FP64, device time per trial state.
4. The learned map fused into the step (icempm_set_learned_map) on the same
   scene and sub-steps against the exact step: device time per sub-step,
   answers kept and fallbacks, state deviation from the FP64 variant.

    python tests/learned_map_study.py [--pairs 20000000] [--eval-steps 500] [--json out.json]

A checker and measurement script (it is not on the product path).
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from icempm_2d_sp_b200 import capi, scenes, surrogate  # noqa: E402
from icempm_2d_sp_b200.params import Options  # noqa: E402


def harvest(sc, steps, capacity, stride, forcing_opts=True):
    o = Options.default(forcing=sc.options.forcing)
    if forcing_opts:
        for f in ("wind_kind", "wind_u", "wind_v", "wind_cx", "wind_cy", "wind_vmax", "wind_radius"):
            setattr(o, f, getattr(sc.options, f))
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o) as ctx:
        ctx.upload(sc.soa, sc.n)
        ctx.harvest_begin(capacity, stride)
        ctx.step(steps, 0)
        rec, offered = ctx.harvest_end()
    return rec, offered


def run_scene(sc, steps, variant="fixed", net=None, tol=None):
    """The scene advanced `steps` sub-steps (CUDA graphs); returns (state,
    error bits, device ms per sub-step, (kept, fallbacks))."""
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n,
                      options=Options.default(variant=variant, forcing=sc.options.forcing)) as ctx:
        ctx.upload(sc.soa, sc.n)
        if net is not None:
            net.attach(ctx, tol)
        ctx.step(steps, 0)
        ms = ctx.timings()[0] / steps
        out, _ = ctx.download(np.zeros_like(sc.soa))
        err, _ = ctx.status()
        counts = ctx.learned_map_counts() if net is not None else (0, 0)
    return out, err, ms, counts


def fused_runs(sc, params, norm, steps):
    n = sc.n
    ref64, e64, ms64, _ = run_scene(sc, steps, "fp64")
    vref = np.abs(ref64[8:10, :n]).max()

    def dev(st):
        return {"pos_max_cells": float(np.abs(st[6:8, :n] - ref64[6:8, :n]).max()),
                "vel_max_rel": float(np.abs(st[8:10, :n] - ref64[8:10, :n]).max() / vref),
                "vel_rms_rel": float(np.sqrt(((st[8:10, :n] - ref64[8:10, :n]) ** 2).mean()) / vref),
                "fe_max": float(np.abs(st[10:14, :n] - ref64[10:14, :n]).max()),
                "jp_max_rel": float(np.abs(st[5, :n] / ref64[5, :n] - 1.0).max())}
    exact, e0, ms0, _ = run_scene(sc, steps)
    res = {"points": int(n), "steps": steps, "fp64_ms_per_step": ms64,
           "exact": {"ms_per_step": ms0, "err_bits": int(e0), **dev(exact)}}
    net = surrogate.StepNetwork(params, norm)
    for tol in (1e-4, 1e-3, 1e-2):
        st, e1, ms1, (kept, fb) = run_scene(sc, steps, net=net, tol=tol)
        res["learned_tol_%g" % tol] = {"ms_per_step": ms1, "err_bits": int(e1), "kept": int(kept),
                                       "fallback": int(fb), "fallback_rate": fb / max(1, kept + fb), **dev(st)}
        print(f"# fused learned map tol {tol}: {ms1:.4f} ms/step (exact {ms0:.4f}), kept {kept}, fallback {fb}",
              file=sys.stderr)
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=20_000_000)
    ap.add_argument("--eval-steps", type=int, default=500)
    ap.add_argument("--eval-states", type=int, default=16_000_000)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    out = {}
    t0 = time.time()
    # 1. training pairs: the floe-field scene (config-1 rules on a 2048x1024
    # grid, 200 sub-steps), then ridging runs at several speeds until --pairs
    sc1 = scenes.floe_field(gx=2048, gy=1024, n_seeds=500)
    r0, _ = harvest(sc1, 200, a.pairs, 1)
    out["pairs_floe_field"] = int(len(r0))
    parts = [r0]
    have = len(r0)
    out["pairs_ridging"] = []
    # four ridging runs share the pairs; every 4th point-step is offered, so a
    # run's records spread over its 1000 sub-steps instead of its first ones
    runs = ((1236, 2.0), (1237, 1.0), (1238, 4.0), (1239, 3.0))
    for k, (seed, speed) in enumerate(runs):
        if have >= a.pairs:
            break
        cap = -(-(a.pairs - have) // (len(runs) - k))
        r1, offered = harvest(scenes.ridging(seed=seed, speed=speed), 1000, cap, 4)
        parts.append(r1)
        have += len(r1)
        out["pairs_ridging"].append({"seed": seed, "speed": speed, "pairs": int(len(r1)), "offered": int(offered)})
    rec = np.concatenate(parts)
    out["pairs"] = int(len(rec))
    print(f"# {len(rec)} pairs ({time.time() - t0:.1f} s)", file=sys.stderr)
    # 2. training
    x = surrogate.feats(rec[:, :4])
    y = surrogate.targets(rec[:, :4], rec[:, 4:7])
    norm = surrogate.Norm.fit(x, y)
    xs = ((x - norm.x_mean) / norm.x_std).astype(np.float32)
    ys = ((y - norm.y_mean) / norm.y_std).astype(np.float32)
    tr = surrogate.Trainer(lr=2e-3)
    t1 = time.time()
    hist = tr.fit(xs, ys, epochs=a.epochs, batch=8192)
    out["train_seconds"] = time.time() - t1
    out["loss_per_epoch"] = hist
    params = tr.params()
    print(f"# trained: loss {hist} ({out['train_seconds']:.1f} s)", file=sys.stderr)
    # 3. evaluation on the 16M-point ridging scene
    ev = scenes.ridging(gx=8192, gy=2048, cells_x=4000, cells_y=1000, h=1.0, dt=1e-4, speed=2.0,
                        steps=a.eval_steps)
    stride = 1
    trial, offered = harvest(ev, a.eval_steps, a.eval_states, stride)
    out["eval_points"] = int(ev.n)
    out["eval_states"] = int(len(trial))
    exact64, _ = surrogate.exact_map(ev.prms, trial[:, :4], fp64=True)
    exact32, ms_exact = surrogate.exact_map(ev.prms, trial[:, :4], fp64=False, repeat=5)
    out["exact_fp32_ms"] = ms_exact
    rel = lambda a_, b_: np.abs(a_[:, :3] - b_[:, :3]) / np.abs(b_[:, :3])
    out["exact_fp32_err_max"] = float(rel(exact32, exact64).max())
    rows = []
    for tol in (1e-4, 1e-3, 1e-2):
        got, nfb, ms = surrogate.learned_map(ev.prms, params, norm, trial[:, :4], tol=tol, repeat=5)
        how = got[:, 3]
        net = how == 1.0
        e = rel(got, exact64)
        rows.append({"tol": tol, "fallback_rate": float((how == 2.0).mean()), "exact_form_rate": float((how == 0).mean()),
                     "network_rate": float(net.mean()), "ms": ms,
                     "err_max_all": float(e.max()), "err_rms_all": float(np.sqrt((e ** 2).mean())),
                     "err_max_network": float(e[net].max()) if net.any() else 0.0,
                     "err_rms_network": float(np.sqrt((e[net] ** 2).mean())) if net.any() else 0.0})
    out["learned"] = rows
    raw, _, ms_raw = surrogate.learned_map(ev.prms, params, norm, trial[:, :4], tol=1e30, repeat=5)
    er = rel(raw, exact64)
    out["network_only"] = {"ms": ms_raw, "err_max": float(er.max()), "err_rms": float(np.sqrt((er ** 2).mean()))}
    # 4. the learned map fused into the step (icempm_set_learned_map) against
    # the exact step on the same scene and sub-steps; error against the FP64
    # variant's state
    out["fused"] = fused_runs(ev, params, norm, a.eval_steps)
    print(json.dumps(out, indent=1))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
