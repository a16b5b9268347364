"""Build the CUDA library in-tree for sm_100a.

    python -m icempm_2d_sp_b200.build        # -> icempm_2d_sp_b200/libicempm_b200.so

nvcc compiles each translation unit of csrc/ (in parallel) with
-gencode arch=compute_100a,code=sm_100a and links one shared library whose
exported symbols are the extern "C" functions of include/icempm.h.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.environ.get("ICEMPM_BUILD_DIR", os.path.join(HERE, "_build"))
LIB = os.environ.get("ICEMPM_LIB_OUT", os.path.join(HERE, "libicempm_b200.so"))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]
# developer knob for tuning builds, e.g. ICEMPM_EXTRA_FLAGS="-maxrregcount=96"
FLAGS += os.environ.get("ICEMPM_EXTRA_FLAGS", "").split()
SOURCES = ["capi.cu", "engine_fixed.cu", "engine_fp32.cu", "engine_fp64.cu", "noalloc.cu", "surrogate.cu"]
# The FP32-state engines use approximate single-precision division and square
# root (a few ulp, far inside the parity tolerances); the FP64 engine is exact.
PER_SOURCE = {"engine_fixed.cu": ["-use_fast_math"], "engine_fp32.cu": ["-use_fast_math"]}


def _deps():
    out = [os.path.join(ROOT, "include", "icempm.h")]
    for f in os.listdir(CSRC):
        out.append(os.path.join(CSRC, f))
    return out


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    cmd = [NVCC] + ARCH + FLAGS + PER_SOURCE.get(src, []) + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    deps = _deps()
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
