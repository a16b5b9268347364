"""Recipe: compile the reference's own CUDA step for sm_100a.

    python -m oracle.refbuild.build_ref_gpu     # -> oracle/_ref/libicempm_ref_gpu.so

nvcc compiles ref_gpu_harness.cu, which #includes the reference's
simulation/kernels.cuh, helper_math.cuh, givens.cuh and parameters_sim.h
where they lie in the reference checkout, with the stand-in headers in
oracle/refbuild/stubs (a host+device 2x2 subset of the Eigen API, spdlog and
HDF5 no-ops) and the real CUDA runtime.  The reference builds these kernels
with nvcc's default floating-point flags (its CMakeLists.txt leaves
CMAKE_CUDA_FLAGS at the default); so does this recipe, for sm_100a instead of
its "80;89".  Needs the reference checkout, so it runs only where the checkout
exists; the built library travels with the repository snapshot.  TEST AND
MEASUREMENT INFRASTRUCTURE ONLY.
"""
import ctypes as C
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT_DIR = os.path.join(ORACLE, "_ref")
LIB = os.path.join(OUT_DIR, "libicempm_ref_gpu.so")
# the reference checkout: ICEMPM_REFERENCE_DIR, else the one build_ref.py uses
from oracle.refbuild.build_ref import REF  # noqa: E402
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def available() -> bool:
    return os.path.isdir(os.path.join(REF, "simulation"))


def build(force: bool = False) -> str:
    if not available():
        if os.path.exists(LIB):
            return LIB
        raise FileNotFoundError("reference checkout not found and no prebuilt " + LIB)
    sim = os.path.join(REF, "simulation")
    src = os.path.join(HERE, "ref_gpu_harness.cu")
    deps = [src, os.path.join(HERE, "stubs", "Eigen", "Core"), os.path.join(sim, "kernels.cuh"),
            os.path.join(sim, "helper_math.cuh"), os.path.join(sim, "parameters_sim.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [NVCC, "-std=c++20", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
           "--expt-relaxed-constexpr", "-w", "-shared", "-Xcompiler", "-fPIC", "-cudart", "static",
           "-I", os.path.join(HERE, "stubs"),
           "-I", sim, "-I", os.path.join(sim, "hssoa"),
           "-I", os.path.join(REF, "External"),
           "-o", LIB, src]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))


_lib = None


def load():
    """ctypes handle on the built library (builds it when the reference
    checkout is present)."""
    global _lib
    if _lib is None:
        from icempm_2d_sp_b200.params import SimParams
        path = build() if available() else LIB
        if not os.path.exists(path):
            raise FileNotFoundError("reference GPU library not built: " + LIB)
        L = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        L.ref_gpu_last_error.restype = C.c_char_p
        L.ref_gpu_device_count.restype = C.c_int
        L.ref_gpu_create.argtypes = [C.POINTER(SimParams), C.POINTER(C.c_uint8), dp, C.c_size_t, C.c_size_t]
        L.ref_gpu_upload.argtypes = [dp, C.c_size_t, C.c_size_t]
        L.ref_gpu_run.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_float)]
        L.ref_gpu_download.argtypes = [dp, C.c_size_t, dp, C.c_size_t, C.POINTER(C.c_uint32), C.POINTER(C.c_int)]
        for f in ("ref_gpu_create", "ref_gpu_upload", "ref_gpu_run", "ref_gpu_download"):
            getattr(L, f).restype = C.c_int
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError("reference GPU step: " + load().ref_gpu_last_error().decode())


class RefGpuScene:
    """One scene on the reference's own CUDA step (the library keeps a single
    scene: its state lives in the kernels' __constant__ symbols)."""

    def __init__(self, prms, status, grid, capacity):
        import numpy as np
        self.L = load()
        self.prms = prms
        dp = C.POINTER(C.c_double)
        g = np.ascontiguousarray(grid, dtype=np.float64)
        st = np.ascontiguousarray(status, dtype=np.uint8)
        _check(self.L.ref_gpu_create(C.byref(prms), st.ctypes.data_as(C.POINTER(C.c_uint8)),
                                     g.ctypes.data_as(dp), g.shape[1], capacity))
        self.n = 0

    def upload(self, soa, n):
        import numpy as np
        s = np.ascontiguousarray(soa, dtype=np.float64)
        _check(self.L.ref_gpu_upload(s.ctypes.data_as(C.POINTER(C.c_double)), s.shape[1], n))
        self.n = n

    def run(self, nsteps, first_step=0):
        ms = C.c_float(0.0)
        _check(self.L.ref_gpu_run(nsteps, first_step, C.byref(ms)))
        return ms.value

    def download(self, soa, grid=None):
        dp = C.POINTER(C.c_double)
        err = C.c_uint32(0)
        dis = C.c_int(0)
        gp = grid.ctypes.data_as(dp) if grid is not None else None
        _check(self.L.ref_gpu_download(soa.ctypes.data_as(dp), soa.shape[1], gp,
                                       grid.shape[1] if grid is not None else 0, C.byref(err), C.byref(dis)))
        return err.value, dis.value

    def close(self):
        self.L.ref_gpu_destroy()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
