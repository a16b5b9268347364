"""The C-ABI library on a machine without a GPU: it loads, exports every entry
point include/icempm.h declares, its struct layouts match the ctypes mirrors,
and argument errors come back as negative codes without touching a device."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from icempm_2d_sp_b200 import capi
from icempm_2d_sp_b200.params import SimParams, Options

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "icempm.h")


@pytest.fixture(scope="module")
def lib():
    from icempm_2d_sp_b200 import build
    build.build()
    return capi.load()


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"ICEMPM_API\s+[\w\s\*]+?\b(icempm_\w+)\s*\(", txt)))


def test_header_declares_the_binding_exports():
    assert declared_functions() == sorted(capi.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (icempm_\w+)", out))
    missing = set(declared_functions()) - exported
    assert not missing, missing
    for name in declared_functions():
        assert getattr(lib, name) is not None


def _c_offsets(struct_name, fields, tmp_path):
    src = tmp_path / "layout.c"
    body = "\n".join(f'printf("%zu\\n", offsetof({struct_name}, {f}));' for f in fields)
    src.write_text(f'#include <stdio.h>\n#include <stddef.h>\n#include "icempm.h"\n'
                   f'int main(void) {{ printf("%zu\\n", sizeof({struct_name}));\n{body}\nreturn 0; }}\n')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    vals = [int(v) for v in subprocess.check_output([str(exe)]).split()]
    return vals[0], vals[1:]


def test_simparams_header_layout_matches_ctypes(tmp_path):
    fields = [f if f != "lambda_" else "lambda" for f, _ in SimParams._fields_]
    size, offs = _c_offsets("icempm_simparams_t", fields, tmp_path)
    assert size == C.sizeof(SimParams) == 328
    assert offs == [getattr(SimParams, f).offset for f, _ in SimParams._fields_]


def test_options_header_layout_matches_ctypes(tmp_path):
    fields = [f for f, _ in Options._fields_]
    size, offs = _c_offsets("icempm_options_t", fields, tmp_path)
    assert size == C.sizeof(Options)
    assert offs == [getattr(Options, f).offset for f, _ in Options._fields_]


def test_default_options(lib):
    o = Options()
    lib.icempm_default_options(C.byref(o))
    d = Options.default()
    for f, _ in Options._fields_:
        if f != "block_threads":
            assert getattr(o, f) == getattr(d, f), f


def test_argument_errors_without_a_device(lib):
    h = C.c_void_p()
    assert lib.icempm_create(None, None, None, 0, None, C.byref(h)) == -1
    assert b"required" in lib.icempm_last_error()
    assert lib.icempm_create(None, None, None, 0, None, None) == -1
    assert lib.icempm_step(None, 1, 0) == -1
    assert lib.icempm_download_points(None, None, 0, None) == -1
    assert lib.icempm_get_status(None, None, None) == -1
    assert lib.icempm_destroy(None) == 0
    p = SimParams.reset()
    st = np.zeros(16, np.uint8)
    o = Options.default()
    o.variant = 7
    assert lib.icempm_create(C.byref(p), st.ctypes.data_as(C.POINTER(C.c_uint8)), None, 0,
                             C.byref(o), C.byref(h)) == -1
    assert b"variant" in lib.icempm_last_error()


def test_device_count_is_safe_without_gpu(lib):
    n = C.c_int(-5)
    lib.icempm_device_count(C.byref(n))
    assert n.value >= 0


def test_noalloc_rejects_oversize_before_any_device_work(lib):
    """icempm_cell_order_noalloc refuses n above ICEMPM_NOALLOC_MAX_POINTS with
    ICEMPM_E_CAPACITY and a message, before it touches a device (no GPU here)."""
    rc = lib.icempm_cell_order_noalloc(None, None, (1 << 20) + 1, 8, None, None, None)
    assert rc == -5 and b"ICEMPM_NOALLOC_MAX_POINTS" in lib.icempm_last_error()
