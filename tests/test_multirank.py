"""The N>1 path of bench.py on CPU: two gloo ranks.

bench.py under torchrun runs one independent scene per rank (weak scaling, no
collective inside the step) and reports the slowest rank's time and the points
of all ranks.  These tests run that combination and the reference arm's
rank-0-only rule with the gloo backend, world size 2, on 127.0.0.1.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _combine_worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.init_ranks(world, rank)
    assert dist.get_backend() == "gloo"
    t_ms, n = [(3.0, 10), (5.0, 32)][rank]
    res = bench.combine_ranks(dist, t_ms, n)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)
    dist.barrier()
    dist.destroy_process_group()


def test_combine_ranks_takes_slowest_time_and_all_points(tmp_path):
    import torch.multiprocessing as mp
    port = free_port()
    mp.start_processes(_combine_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        with open(tmp_path / f"rank{r}.json") as f:
            t_ms, n = json.load(f)
        assert t_ms == 5.0 and n == 42


def test_combine_ranks_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.combine_ranks(None, 2.5, 7) == (2.5, 7)


def test_reference_arm_under_torchrun_prints_once(tmp_path):
    """--impl reference with two ranks: rank 0 alone runs the reference on the
    host cores and prints one JSON line; rank 1 exits 0 without work."""
    from oracle.refbuild import build_ref
    if not (build_ref.available() or os.path.exists(build_ref.LIB)):
        pytest.skip("reference host build not available")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="4")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--grid", "512", "256"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("reference", "port")


def test_ensemble_scenes_split_by_size_over_ranks():
    """bench.py --workload ensemble under torchrun: each rank generates and
    steps its share of the scenes; every scene goes to exactly one rank and
    the ranks' point totals stay within a few percent of each other."""
    from icempm_2d_sp_b200 import scenes
    sizes = [s["target_points"] for s in scenes.ensemble_specs(96)]
    for world in (1, 2, 4, 8):
        parts = scenes.split_by_size(sizes, world)
        assert sorted(i for p in parts for i in p) == list(range(96))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) <= 1.05 * min(loads)
