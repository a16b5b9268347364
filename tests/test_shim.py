"""The C++ GPU_Implementation5 shim (include/icempm_gpu_implementation5.hpp)
driving the reference's frame loop (model.cpp:7-78) gives the same points as
the Python Model mirror over the same C ABI."""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "cpp"))

from icempm_2d_sp_b200 import scenes  # noqa: E402


def test_shim_driver_compiles():
    import build_driver
    from icempm_2d_sp_b200 import build
    build.build()
    assert os.path.exists(build_driver.build())


def write_scene(path, sc):
    with open(path, "wb") as f:
        f.write(bytes(sc.prms))
        f.write(np.array([sc.n, sc.soa.shape[1]], np.uint32).tobytes())
        f.write(np.ascontiguousarray(sc.status, np.uint8).tobytes())
        f.write(np.ascontiguousarray(sc.current, np.float64).tobytes())
        f.write(np.ascontiguousarray(sc.soa, np.float64).tobytes())


@pytest.mark.gpu
def test_shim_frames_match_python_model(tmp_path):
    import build_driver
    from icempm_2d_sp_b200.model import Model
    exe = build_driver.build()
    sc = scenes.random_state(seed=31, gx=40, gy=32, crushed_frac=0.5, strain=3e-3)
    frames = 3
    scene = tmp_path / "scene.bin"
    out = tmp_path / "out.bin"
    write_scene(scene, sc)
    subprocess.check_call([exe, str(scene), str(out), str(frames)])
    raw = np.fromfile(out, dtype=np.uint8)
    cap = sc.soa.shape[1]
    soa_shim = raw[:19 * cap * 8].view(np.float64).reshape(19, cap)
    size, err = raw[19 * cap * 8:19 * cap * 8 + 8].view(np.uint32)
    dis = raw[19 * cap * 8 + 8:].view(np.int32)[0]

    m = Model(sc.prms, sc.status, sc.current, soa=sc.soa.copy(), n=sc.n, capacity=cap)
    m.Prepare()
    for _ in range(frames):
        assert m.Step()
    assert size == m.size == sc.n
    assert err == m.error_code == 0 and dis == m.disabled_points_count
    assert m.prms.SimulationStep == frames * sc.prms.UpdateEveryNthStep
    # the fixed-point form is deterministic: one-sub-step calls and graph-batched
    # frames give identical bits
    assert np.array_equal(soa_shim[:, :size].view(np.uint64), m.hssoa[:, :size].view(np.uint64))
    m.close()
