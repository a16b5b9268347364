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
# the reference checkout: ICEMPM_REFERENCE_DIR, else a sibling of the repository
REF = os.environ.get("ICEMPM_REFERENCE_DIR", os.path.join(os.path.dirname(os.path.dirname(ORACLE)), "reference"))
FRAME_LIB = os.path.join(OUT_DIR, "libicempm_ref_frame.so")
# the two member functions of simulation/data_manager/snapshotmanager.cpp the
# frame harness compiles (CalculateWeightCoeffs, PrepareFrameArrays)
FRAME_FUNCS = ("void icy::SnapshotManager::CalculateWeightCoeffs(", "void icy::SnapshotManager::PrepareFrameArrays()")


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


def _extract_function(text, signature):
    """The definition that starts with `signature`, through its closing brace
    (braces inside string and character literals and comments are skipped),
    preceded by a #line directive that points at the reference file."""
    start = text.index(signature)
    i = text.index("{", start)
    depth, n = 0, len(text)
    while i < n:
        c = text[i]
        if c in "\"'":
            j = i + 1
            while text[j] != c:
                j += 2 if text[j] == "\\" else 1
            i = j + 1
            continue
        if text.startswith("//", i):
            i = text.index("\n", i)
            continue
        if text.startswith("/*", i):
            i = text.index("*/", i) + 2
            continue
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                line = text.count("\n", 0, start) + 1
                return '#line %d "%s"\n%s\n' % (line, "simulation/data_manager/snapshotmanager.cpp", text[start:i + 1])
        i += 1
    raise ValueError("unterminated definition: " + signature)


def build_frame(force: bool = False) -> str:
    """oracle/_ref/libicempm_ref_frame.so: oracle/refbuild/frame_harness.cpp with
    the reference's PrepareFrameArrays and CalculateWeightCoeffs, read from
    the checkout at build time into oracle/_ref/frame_extract.inc, plus
    hssoa/host_side_soa.cpp and hssoa/proxypoint2d.cpp."""
    if not available():
        if os.path.exists(FRAME_LIB):
            return FRAME_LIB
        raise FileNotFoundError("reference checkout not found and no prebuilt " + FRAME_LIB)
    sim = os.path.join(REF, "simulation")
    smc = os.path.join(sim, "data_manager", "snapshotmanager.cpp")
    harness = os.path.join(HERE, "frame_harness.cpp")
    srcs = [harness, os.path.join(sim, "hssoa", "host_side_soa.cpp"), os.path.join(sim, "hssoa", "proxypoint2d.cpp")]
    deps = srcs + [smc, os.path.join(HERE, "stubs", "Eigen", "Core"), os.path.join(HERE, "stubs", "Eigen", "Dense"),
                   os.path.join(HERE, "stubs", "openjpeg.h"), os.path.join(HERE, "stubs", "H5Cpp.h")]
    if not force and os.path.exists(FRAME_LIB) and all(os.path.getmtime(FRAME_LIB) >= os.path.getmtime(d) for d in deps):
        return FRAME_LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    with open(smc) as f:
        text = f.read()
    with open(os.path.join(OUT_DIR, "frame_extract.inc"), "w") as f:
        f.write("\n".join(_extract_function(text, sig) for sig in FRAME_FUNCS))
    cmd = ["g++", "-std=c++20", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-w",
           "-I", os.path.join(HERE, "stubs_host"), "-I", os.path.join(HERE, "stubs"),
           "-I", sim, "-I", os.path.join(sim, "hssoa"), "-I", os.path.join(sim, "data_manager"),
           "-I", os.path.join(REF, "External"), "-I", REF, "-I", OUT_DIR, "-o", FRAME_LIB] + srcs
    subprocess.check_call(cmd)
    return FRAME_LIB


_frame_lib = None


def load_frame():
    """ctypes handle on the reference frame library (builds it when the
    reference checkout is present)."""
    global _frame_lib
    if _frame_lib is None:
        import ctypes as C
        from icempm_2d_sp_b200.params import SimParams
        path = build_frame() if available() else FRAME_LIB
        if not os.path.exists(path):
            raise FileNotFoundError("reference frame library not built: " + FRAME_LIB)
        L = C.CDLL(path)
        fp, u8 = C.POINTER(C.c_float), C.POINTER(C.c_uint8)
        L.ref_prepare_frame.argtypes = ([C.POINTER(SimParams), C.POINTER(C.c_double), C.c_uint, C.c_uint,
                                         C.POINTER(C.c_uint32), C.c_uint, u8, C.POINTER(C.c_double)]
                                        + [fp] * 10 + [u8, u8, u8, fp])
        L.ref_prepare_frame.restype = C.c_int
        _frame_lib = L
    return _frame_lib


FRAME_KEYS = ("density", "mass", "vx", "vy", "Jpinv", "P", "Q", "r", "g", "b")


def prepare_frame(prms, soa, n, status, forces_fxfy, colors):
    """The reference's PrepareFrameArrays on numpy arrays: returns a dict with
    the ten float channels, rgb, mass_mask, count and forces_per_region."""
    import ctypes as C
    import numpy as np
    L = load_frame()
    G = prms.GridXTotal * prms.GridYTotal
    soa = np.ascontiguousarray(soa, np.float64)
    colors = np.ascontiguousarray(colors, np.uint32)
    status = np.ascontiguousarray(status, np.uint8)
    forces = np.ascontiguousarray(forces_fxfy, np.float64)
    assert status.size == G and forces.size == 2 * G
    out = {k: np.zeros(G, np.float32) for k in FRAME_KEYS}
    out["rgb"] = np.zeros(3 * G, np.uint8)
    out["mass_mask"] = np.zeros(G, np.uint8)
    out["count"] = np.zeros(G, np.uint8)
    out["forces_per_region"] = np.zeros((100, 2), np.float32)
    fp, u8 = C.POINTER(C.c_float), C.POINTER(C.c_uint8)
    L.ref_prepare_frame(C.byref(prms), soa.ctypes.data_as(C.POINTER(C.c_double)), soa.shape[1], n,
                        colors.ctypes.data_as(C.POINTER(C.c_uint32)), colors.size, status.ctypes.data_as(u8),
                        forces.ctypes.data_as(C.POINTER(C.c_double)),
                        *[out[k].ctypes.data_as(fp) for k in FRAME_KEYS],
                        out["rgb"].ctypes.data_as(u8), out["mass_mask"].ctypes.data_as(u8),
                        out["count"].ctypes.data_as(u8), out["forces_per_region"].ctypes.data_as(fp))
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
    print(build_frame(force="--force" in sys.argv))


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
        L.ref_run_steps_parallel.argtypes = L.ref_run_steps.argtypes
        L.ref_run_steps_parallel.restype = C.c_uint32
        L.ref_remove_disabled_and_sort.argtypes = [dp, C.c_uint, C.c_uint, C.c_int]
        L.ref_remove_disabled_and_sort.restype = C.c_uint
        L.ref_num_threads.restype = C.c_int
        _lib = L
    return _lib


def run_steps(prms, soa, n, grid, status, nsteps, first_step=0, parallel_p2g=False):
    """Reference sub-step loop on numpy arrays (mutates soa, grid).
    parallel_p2g: P2G's blocks run over all host threads with atomic adds (as
    on the GPU; the sums' order then varies); otherwise serially in point
    order (deterministic, the golden fixtures)."""
    import ctypes as C
    L = load()
    dp = C.POINTER(C.c_double)
    dis = C.c_int(0)
    st = status.copy()
    fn = L.ref_run_steps_parallel if parallel_p2g else L.ref_run_steps
    err = fn(C.byref(prms), soa.ctypes.data_as(dp), soa.shape[1], n,
                          grid.ctypes.data_as(dp), grid.shape[1],
                          st.ctypes.data_as(C.POINTER(C.c_uint8)), nsteps, first_step, C.byref(dis))
    return err, dis.value
