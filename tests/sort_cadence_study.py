"""Locality decay of the cell-sorted point order, and the re-sort cadence it
calls for (a measurement script, not a test; one B200).

The fused kernel reads each thread's points as one cell's run (the order the
locality sort leaves), so its speed depends on how far the points have
drifted from that order.  For each scene this script advances the points from
a fresh sort in windows of sub-steps (CUDA graphs) and records the device
time per sub-step of each window against the sub-steps since the sort, then
times one locality sort, and runs the library's cadence tuner
(icempm_tune_sort_cadence) on the drifted state.

    python tests/sort_cadence_study.py [--json out.json]

Scenes: the floe field (4096x2048, 23.0M points, 200
sub-steps) and the 1M-point ridging scene (1024x512, 2 m/s against the wall,
1000 sub-steps).
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from icempm_2d_sp_b200 import capi, scenes  # noqa: E402
from icempm_2d_sp_b200.params import Options  # noqa: E402


def decay(sc, steps, window):
    o = Options.default(forcing=sc.options.forcing)
    for f, _ in Options._fields_:
        setattr(o, f, getattr(sc.options, f))
    o.sort_every = 0
    rows = []
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o) as ctx:
        ctx.upload(sc.soa, sc.n)            # the upload sorts
        ctx.step(3, 0)
        done = 3
        while done < steps:
            k = min(window, steps - done)
            ctx.step(k, done)
            rows.append({"since_sort": done + k // 2, "ms_per_step": ctx.timings()[0] / k})
            done += k
        # the drifted state: downloaded (re-sorted by a fresh upload below),
        # and the cadence tuner run on it
        out, n = ctx.download(np.zeros_like(sc.soa))
        err, _ = ctx.status()
        k = ctx.tune_sort_cadence(window, done)
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o) as c2:
        c2.upload(out, n)
        c2.step(3, done)
        c2.step(window, done + 3)
        fresh = c2.timings()[0] / window
    return {"points": int(sc.n), "window": window, "decay": rows, "err": int(err),
            "fresh_sort_ms_per_step": fresh, "tuned_sort_every": k,
            "first_window_ms": rows[0]["ms_per_step"], "last_window_ms": rows[-1]["ms_per_step"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    capi.load()
    out = {"floe_field": decay(scenes.floe_field(), 200, 20),
           "ridging": decay(scenes.ridging(), 1000, 50)}
    for name, r in out.items():
        print(f"# {name}: {r['points']} points, ms/step first window {r['first_window_ms']:.4f}, "
              f"last {r['last_window_ms']:.4f}, after a fresh sort {r['fresh_sort_ms_per_step']:.4f}, "
              f"tuned sort_every {r['tuned_sort_every']}", file=sys.stderr)
    print(json.dumps(out, indent=1))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
