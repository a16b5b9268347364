"""Build recipe for the oracle shared library (test infrastructure only).

    python -m oracle.build          # -> oracle/_build/libicempm_oracle.so
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libicempm_oracle.so")
SRC = os.path.join(HERE, "icempm_oracle.c")


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    deps = [SRC, os.path.join(HERE, "..", "include", "icempm.h")]
    if not force and os.path.exists(LIB) and all(
            os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    cmd = ["gcc", "-O2", "-std=c11", "-fopenmp", "-ffp-contract=off", "-fPIC",
           "-shared", "-Wall", "-Wno-unused-function", "-o", LIB, SRC, "-lm"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
