"""Precision study: the GPU step's variants against the
FP64 CPU oracle.

Scenes: the ice block (64,000 points, 10 m/s wind, current 0.1 m/s) and the
ridging scene (1024x512 grid, 1M points driven at 2 m/s against the x=0 wall,
all points crushed, so the Drucker-Prager return map acts on every point).
Each runs 1, 100 and 1000 sub-steps from its initial state in three
variants -- FP32 atomics, int64 fixed-point P2G (FP64 only in near-degenerate
SVD and the Jp update), full FP64 on the GPU -- and is compared with the
oracle at the same step:

  pos_max / pos_rms   position error in cells (max / root mean square)
  vel_max / vel_rms   velocity error relative to the oracle's largest speed
  mom                 |P - P_ref| / |P_ref| of the total momentum of enabled points
  ke                  |KE - KE_ref| / KE_ref
  mass                relative difference of the total mass of enabled points
  flags               points whose utility word (crushed / disabled) differs

    python tests/precision_study.py [--scenes ice_block,ridging] [--steps 1,100,1000] [--json out.json]

The oracle is test infrastructure; this script is a checker, never on the
product path.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from icempm_2d_sp_b200 import scenes, hssoa as H  # noqa: E402
from icempm_2d_sp_b200.params import Options, IDX_UTILITY, STATUS_DISABLED, FORCING_EXTENDED  # noqa: E402

VARIANTS = ["fp32", "fixed", "fp64"]


def make(name):
    if name == "ice_block":
        return scenes.ice_block(forcing=FORCING_EXTENDED)
    if name == "ridging":
        return scenes.ridging()
    raise ValueError(name)


def metrics(got, ref, n, prms):
    h = prms.cellsize
    en_r = (H.get_u32(ref, IDX_UTILITY, n) & STATUS_DISABLED) == 0
    en_g = (H.get_u32(got, IDX_UTILITY, n) & STATUS_DISABLED) == 0
    from parity_util import world
    gx, gy = world(got, n, h)
    rx, ry = world(ref, n, h)
    both = en_r & en_g
    dp = np.hypot(gx - rx, gy - ry)[both] / h
    vmax = max(np.hypot(ref[8, :n], ref[9, :n])[en_r].max(), 1e-30)
    dv = np.hypot(got[8, :n] - ref[8, :n], got[9, :n] - ref[9, :n])[both] / vmax

    def agg(soa, en):
        m = prms.ParticleMass * soa[18, :n][en]
        vx, vy = soa[8, :n][en], soa[9, :n][en]
        return m.sum(), np.array([(m * vx).sum(), (m * vy).sum()]), 0.5 * (m * (vx * vx + vy * vy)).sum()

    mg, pg, kg = agg(got, en_g)
    mr, pr, kr = agg(ref, en_r)
    return {
        "pos_max": float(dp.max()) if dp.size else 0.0,
        "pos_rms": float(np.sqrt((dp ** 2).mean())) if dp.size else 0.0,
        "vel_max": float(dv.max()) if dv.size else 0.0,
        "vel_rms": float(np.sqrt((dv ** 2).mean())) if dv.size else 0.0,
        "mom": float(np.linalg.norm(pg - pr) / max(np.linalg.norm(pr), 1e-300)),
        "ke": float(abs(kg - kr) / max(kr, 1e-300)),
        "mass": float(abs(mg - mr) / max(mr, 1e-300)),
        "flags": int((H.get_u32(got, IDX_UTILITY, n) != H.get_u32(ref, IDX_UTILITY, n)).sum()),
    }


def oracle_snapshots(sc, steps):
    """FP64 oracle from the initial state; a copy of the points at each step count."""
    import oracle
    soa = sc.soa.copy()
    grid = oracle.new_grid(sc.prms, current=sc.current)
    out, done, t0 = {}, 0, time.time()
    opts = sc.options if sc.options.forcing == FORCING_EXTENDED else None
    for k in sorted(steps):
        oracle.run_steps(sc.prms, soa, sc.n, grid, sc.status, k - done, done, opts=opts)
        done = k
        out[k] = soa.copy()
    return out, time.time() - t0


def gpu_snapshots(sc, steps, variant):
    from icempm_2d_sp_b200 import capi
    o = Options.default(variant=variant, forcing=sc.options.forcing)
    for f in ("wind_kind", "wind_u", "wind_v", "wind_cx", "wind_cy", "wind_vmax", "wind_radius"):
        setattr(o, f, getattr(sc.options, f))
    out, done = {}, 0
    with capi.Context(sc.prms, sc.status, sc.current, capacity=sc.n, options=o) as ctx:
        ctx.upload(sc.soa, sc.n)
        for k in sorted(steps):
            ctx.step(k - done, done)
            done = k
            s, m = ctx.download(np.zeros_like(sc.soa))
            assert m == sc.n
            out[k] = s
        err, _ = ctx.status()
    return out, err


def run(scene_names, steps, variants=VARIANTS):
    rows = []
    for name in scene_names:
        sc = make(name)
        ref, t_oracle = oracle_snapshots(sc, steps)
        for v in variants:
            got, err = gpu_snapshots(sc, steps, v)
            for k in sorted(steps):
                r = {"scene": name, "points": int(sc.n), "variant": v, "steps": k, "device_errors": int(err)}
                r.update(metrics(got[k], ref[k], sc.n, sc.prms))
                rows.append(r)
        print(f"# {name}: {sc.n} points, oracle {t_oracle:.1f} s", file=sys.stderr)
    return rows


def table(rows):
    out = ["| scene | variant | steps | pos max (cells) | pos rms | vel max (rel) | vel rms | momentum | KE | mass | flags |",
           "|---|---|---|---|---|---|---|---|---|---|---|"]
    for r in rows:
        out.append(f"| {r['scene']} | {r['variant']} | {r['steps']} | {r['pos_max']:.2e} | {r['pos_rms']:.2e} | "
                   f"{r['vel_max']:.2e} | {r['vel_rms']:.2e} | {r['mom']:.2e} | {r['ke']:.2e} | {r['mass']:.1e} | "
                   f"{r['flags']} |")
    return "\n".join(out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", default="ice_block,ridging")
    ap.add_argument("--steps", default="1,100,1000")
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    rows = run(a.scenes.split(","), [int(s) for s in a.steps.split(",")])
    print(table(rows))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(rows, f, indent=1)


if __name__ == "__main__":
    main()
