"""Generate the golden fixtures in tests/golden/ from the reference's own code.

    python tests/golden/make_golden.py

Each fixture is a seeded synthetic scene (icempm_2d_sp_b200.scenes) advanced
by the reference sources themselves -- simulation/kernels.cuh, helper_math.cuh,
givens.cuh, parameters_sim.cpp and hssoa/host_side_soa.cpp compiled on the host
by oracle/refbuild/build_ref.py -- so the expected outputs are the reference's,
not the oracle's.  Needs the reference checkout (only where fixtures are made);
the committed .npz files are what the tests read.

Stored per fixture: the SimParams bytes, grid status, current field, the input
HSSOA, the number of steps and first step index, the output HSSOA, the output
grid (mass/velocity rows after the last step), error bits and disabled count.
frame_ridging holds the reference's PrepareFrameArrays output instead (see
frame_fixture).
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from icempm_2d_sp_b200 import scenes, hssoa as H  # noqa: E402
from icempm_2d_sp_b200.params import SimParams, IDX_VELX, IDX_UTILITY, STATUS_DISABLED  # noqa: E402
from oracle.refbuild import build_ref  # noqa: E402


def _grid(sc):
    G = sc.grid_nodes
    g = np.zeros((9, G))
    g[5], g[6] = sc.current[:G], sc.current[G:]
    return g


def save(name, sc, nsteps, first_step=0, extra=None):
    soa_in = sc.soa.copy()
    soa = sc.soa.copy()
    grid = _grid(sc)
    err, dis = build_ref.run_steps(sc.prms, soa, sc.n, grid, sc.status, nsteps, first_step)
    d = dict(prms=np.frombuffer(bytes(sc.prms), np.uint8), status=sc.status, current=sc.current,
             soa_in=soa_in, n=np.int64(sc.n), nsteps=np.int64(nsteps), first_step=np.int64(first_step),
             soa_out=soa, grid_out=grid[:3], err=np.uint32(err), disabled=np.int64(dis))
    if extra:
        d.update(extra)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
    print(f"{name}: n={sc.n} steps={nsteps} err={err:#x} disabled={dis}")


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    prms = SimParams.from_buffer_copy(z["prms"].tobytes())
    return z, prms


def main():
    build_ref.build()
    sc = scenes.random_state(seed=11, gx=24, gy=20, fill=0.7, crushed_frac=0.6, strain=4e-3)
    save("random_1step", sc, 1, 0)
    sc = scenes.random_state(seed=11, gx=24, gy=20, fill=0.7, crushed_frac=0.6, strain=4e-3)
    save("random_10step", sc, 10, 5)
    sc = scenes.random_state(seed=12, gx=32, gy=24, fill=0.8, crushed_frac=1.0, strain=2e-2,
                             low_jp_frac=0.3)
    save("random_plastic_20step", sc, 20, 0)
    sc = scenes.ridging(seed=13, gx=48, gy=24, cells_x=30, cells_y=16, steps=60)
    save("ridging_60step", sc, 60, 0)
    # points pushed out of the domain get disabled; then RemoveDisabledAndSort
    sc = scenes.random_state(seed=14, gx=20, gy=16, fill=0.9, crushed_frac=0.0, strain=1e-4, vel=0.0,
                             dt=2e-3, h=1.0)
    n = sc.n
    x, y = H.world_positions(sc.soa, n, sc.prms.cellsize)
    sc.soa[IDX_VELX, :n] = np.where(x < 10, -30.0, 30.0)
    sc.soa[IDX_VELX + 1, :n] = 0.0
    sc.soa[14:18, :n] = 0.0
    soa = sc.soa.copy()
    grid = _grid(sc)
    nsteps = 40
    err, dis = build_ref.run_steps(sc.prms, soa, n, grid, sc.status, nsteps, 0)
    sorted_soa = soa.copy()
    m = build_ref.load().ref_remove_disabled_and_sort(sorted_soa.ctypes.data_as(C.POINTER(C.c_double)),
                                                      soa.shape[1], n, sc.prms.GridYTotal)
    save("disable_then_sort", sc, nsteps, 0,
         extra=dict(sorted_soa=sorted_soa, sorted_n=np.int64(m)))
    z, _ = load("disable_then_sort")
    assert int(z["disabled"]) > 0 and int(z["sorted_n"]) == n - int(z["disabled"]), (int(z["disabled"]), int(z["sorted_n"]))
    frame_fixture()


def frame_fixture():
    """frame_ridging: the saved-frame arrays of the reference's own
    SnapshotManager::PrepareFrameArrays (snapshotmanager.cpp:623-765, compiled
    by oracle/refbuild/build_ref.py build_frame) for a ridging scene advanced
    20 steps by the reference kernels, with 5% of the points disabled, random
    point colours, the reference's grid status and seeded boundary forces."""
    sc = scenes.ridging(seed=15, gx=96, gy=64, cells_x=40, cells_y=30, speed=2.0)
    rng = np.random.default_rng(15)
    soa = sc.soa.copy()
    n, G = sc.n, sc.grid_nodes
    util = H.get_u32(soa, IDX_UTILITY, n).copy()
    util[rng.random(n) < 0.05] |= STATUS_DISABLED
    H.set_u32(soa, IDX_UTILITY, util, n)
    grid = _grid(sc)
    err, dis = build_ref.run_steps(sc.prms, soa, n, grid, sc.status, 20, 0)
    colors = rng.integers(0, 1 << 24, n).astype(np.uint32)
    forces = rng.normal(0.0, 50.0, 2 * G)
    out = build_ref.prepare_frame(sc.prms, soa, n, sc.status, forces, colors)
    d = dict(prms=np.frombuffer(bytes(sc.prms), np.uint8), status=sc.status, soa=soa, n=np.int64(n),
             colors=colors, forces=forces, err=np.uint32(err))
    d.update({"out_" + k: v for k, v in out.items()})
    np.savez_compressed(os.path.join(HERE, "frame_ridging.npz"), **d)
    print(f"frame_ridging: n={n} nodes={G} masked={int(out['mass_mask'].sum())} err={err:#x}")

if __name__ == "__main__":
    if sys.argv[1:] == ["frame"]:
        frame_fixture()
    else:
        main()
