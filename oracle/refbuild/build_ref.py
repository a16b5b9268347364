"""Recipe: compile the reference's own sources on the host for the oracle pin.

    python -m oracle.refbuild.build_ref     # -> oracle/_ref/libicempm_ref.so

Compiles ref_harness.cpp (which #includes simulation/kernels.cuh,
helper_math.cuh, givens.cuh and parameters_sim.h where they lie) together
with simulation/parameters_sim.cpp, hssoa/host_side_soa.cpp and
hssoa/proxypoint2d.cpp, all read in place from the reference checkout, with
g++ and the stand-in headers in oracle/refbuild/stubs_host (CUDA qualifiers and
atomics for a host build) and oracle/refbuild/stubs (spdlog/fmt/HDF5
no-ops, a 2x2 subset of the Eigen API).  Needs the
reference checkout, so it runs only where the checkout exists; the built
library travels with the repository snapshot.  TEST INFRASTRUCTURE ONLY.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT_DIR = os.path.join(ORACLE, "_ref")
LIB = os.path.join(OUT_DIR, "libicempm_ref.so")
REF = os.environ.get("ICEMPM_REFERENCE_DIR", "/root/reference")


def available() -> bool:
    return os.path.isdir(os.path.join(REF, "simulation"))


def build(force: bool = False) -> str:
    if not available():
        if os.path.exists(LIB):
            return LIB
        raise FileNotFoundError("reference checkout not found and no prebuilt " + LIB)
    sim = os.path.join(REF, "simulation")
    srcs = [os.path.join(HERE, "ref_harness.cpp"),
            os.path.join(sim, "parameters_sim.cpp"),
            os.path.join(sim, "hssoa", "host_side_soa.cpp"),
            os.path.join(sim, "hssoa", "proxypoint2d.cpp")]
    deps = srcs + [os.path.join(HERE, "stubs", "Eigen", "Core"), os.path.join(HERE, "stubs_host", "cuda_runtime.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["g++", "-std=c++20", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-w",
           "-I", os.path.join(HERE, "stubs_host"), "-I", os.path.join(HERE, "stubs"),
           "-I", sim, "-I", os.path.join(sim, "hssoa"),
           "-I", os.path.join(REF, "External"),
           "-o", LIB] + srcs
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))


_lib = None


def load():
    """ctypes handle on the built reference library (builds it when the
    reference checkout is present)."""
    global _lib
    if _lib is None:
        import ctypes as C
        from icempm_2d_sp_b200.params import SimParams
        path = build() if available() else LIB
        if not os.path.exists(path):
            raise FileNotFoundError("reference library not built: " + LIB)
        L = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        sp = C.POINTER(SimParams)
        L.ref_params_reset.argtypes = [sp]
        L.ref_compute_helpers.argtypes = [sp]
        L.ref_simparams_layout.argtypes = [C.POINTER(C.c_longlong), C.c_int]
        L.ref_simparams_layout.restype = C.c_int
        L.ref_svd2x2.argtypes = [dp, dp, dp, dp]
        L.ref_run_steps.argtypes = [sp, dp, C.c_size_t, C.c_size_t, dp, C.c_size_t,
                                    C.POINTER(C.c_uint8), C.c_int, C.c_int, C.POINTER(C.c_int)]
        L.ref_run_steps.restype = C.c_uint32
        L.ref_remove_disabled_and_sort.argtypes = [dp, C.c_uint, C.c_uint, C.c_int]
        L.ref_remove_disabled_and_sort.restype = C.c_uint
        L.ref_num_threads.restype = C.c_int
        _lib = L
    return _lib


def run_steps(prms, soa, n, grid, status, nsteps, first_step=0):
    """Reference sub-step loop on numpy arrays (mutates soa, grid)."""
    import ctypes as C
    L = load()
    dp = C.POINTER(C.c_double)
    dis = C.c_int(0)
    st = status.copy()
    err = L.ref_run_steps(C.byref(prms), soa.ctypes.data_as(dp), soa.shape[1], n,
                          grid.ctypes.data_as(dp), grid.shape[1],
                          st.ctypes.data_as(C.POINTER(C.c_uint8)), nsteps, first_step, C.byref(dis))
    return err, dis.value
