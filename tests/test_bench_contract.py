"""bench.py's reported DRAM traffic stays tied to the committed ncu summary it
cites: the per-point constant is the capture's dram bytes over its points,
and the summary file carries the same byte count."""
import importlib.util
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_traffic_constant_matches_its_capture():
    b = _bench()
    cap = b.TRAFFIC_CAPTURE
    assert abs(cap["dram_bytes"] / cap["points"] - b.TRAFFIC_B_PER_POINT) < 0.01
    path = os.path.join(ROOT, cap["capture"])
    assert os.path.exists(path), path
    text = open(path).read()
    # the summary's dram row: "<read> MB + <write> MB = <total> MB (<per point> B/point"
    m = re.search(r"dram__bytes_read\.sum \+ dram__bytes_write\.sum \| ([\d.]+) MB \+ ([\d.]+) MB = ([\d.]+) MB "
                  r"\(([\d.]+) B/point", text)
    assert m, "dram row not found in " + cap["capture"]
    total_mb, per_point = float(m.group(3)), float(m.group(4))
    assert abs(total_mb * 1e6 - cap["dram_bytes"]) < 0.1e6
    assert abs(per_point - b.TRAFFIC_B_PER_POINT) < 0.01
    assert f"{cap['points']:,}" in text


def test_default_run_fits_the_contract():
    """No flags: one GPU, at least 3 warm-up steps."""
    b = _bench()
    import sys
    argv = sys.argv
    try:
        sys.argv = ["bench.py"]
        a = b.parse()
    finally:
        sys.argv = argv
    assert a.gpus == 1 and a.warmup >= 3 and a.steps >= 1 and a.impl == "ours"
