"""Compile tests/cpp/shim_driver.cpp against include/ and the in-tree library."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build", "shim_driver")


def build() -> str:
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    lib_dir = os.path.join(ROOT, "icempm_2d_sp_b200")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"),
                           os.path.join(HERE, "shim_driver.cpp"), "-o", OUT,
                           "-L", lib_dir, "-l:libicempm_b200.so", "-Wl,-rpath," + lib_dir])
    return OUT
