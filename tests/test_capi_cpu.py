"""CPU-side checks of the C ABI: the library loads, exports every entry point that
include/regb200.h declares, and its host-only transform algebra matches the
reference's (golden fixtures) bit for bit.  No device is touched."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from tipl_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "regb200.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(regb_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def L():
    from tipl_b200 import build

    build.build()
    return _lib.lib()


def test_header_symbols_exported(L):
    names = declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), f"{n} declared in regb200.h but not exported"
    # and the Python binding covers them all
    assert set(names) <= set(_lib.declared_symbols()) | {"regb_status"}


def bits(a):
    return np.asarray(a).view(np.uint32)


def test_transforms_match_reference(L, golden):
    import tipl_b200 as tb

    g = golden("transforms")
    for p, s, T, Ti in zip(g["params"], g["shapes"], g["T"], g["Tinv"]):
        fs = (s[0], s[1], s[2])  # numpy (z, y, x)
        ts = (s[3], s[4], s[5])
        got = tb.affine_to_matrix(p[:12], fs, p[12:15], ts, p[15:18])
        assert np.array_equal(bits(got), bits(T))
        assert np.array_equal(bits(tb.matrix_inverse(T)), bits(Ti))


def test_f64_composition_close(L, golden):
    import tipl_b200 as tb

    g = golden("transforms")
    for p, s, T in zip(g["params"], g["shapes"], g["T"]):
        fs = (s[0], s[1], s[2])
        ts = (s[3], s[4], s[5])
        T64 = tb.affine_to_matrix_f64(p[:12].astype(np.float64), fs, p[12:15], ts, p[15:18])
        assert np.allclose(T64, T, rtol=1e-5, atol=1e-3)


def test_bad_arguments_are_status_codes(L):
    v = _lib.Volume(None, (C.c_int * 3)(4, 4, 4), _lib.U8, _lib.HOST)
    st = L.regb_resample(C.byref(v), C.byref(v), None, 0, None)
    assert st == _lib.REGB_ERR_ARG
    assert b"null" in L.regb_last_error()
    assert L.regb_matrix_inverse(None) == _lib.REGB_ERR_ARG
    sing = np.zeros(12, np.float32)
    assert L.regb_matrix_inverse(sing.ctypes.data_as(C.c_void_p)) == _lib.REGB_FALSE


def test_param_defaults(L):
    p = _lib.LinearParam()
    L.regb_linear_param_default(C.byref(p))
    assert (p.reg_type, p.cost_type, p.search_count, p.absolute_bound) == (15, 1, 16, 1)
    q = _lib.CdmParam()
    L.regb_cdm_param_default(C.byref(q))
    assert (q.resolution, q.min_dimension, chr(q.gradient_type)) == (2.0, 16, "r")
    assert abs(q.speed - 0.3) < 1e-7 and abs(q.smoothing - 0.05) < 1e-7


def test_engine_config_defaults_match_python(L):
    """regb_engine_config_default (host only) and the Python Engine's keyword defaults agree:
    slots, gather window, affine workers and CDM iterations per round."""
    import inspect

    import tipl_b200 as tb

    c = _lib.EngineConfig()
    L.regb_engine_config_default(C.byref(c))
    assert (c.hbm_budget_bytes, c.max_active, c.gather_us, c.cdm_iters_per_round, c.affine_workers) == \
        (0, 64, 10, 4, 3)
    sig = inspect.signature(tb.Engine.__init__).parameters
    assert (sig["max_active"].default, sig["gather_us"].default, sig["cdm_iters_per_round"].default,
            sig["affine_workers"].default) == (c.max_active, c.gather_us, c.cdm_iters_per_round, c.affine_workers)


def test_runner_state_from_param(L):
    """The runner state of tipl::reg::linear for an affine MI registration: the four DOF
    stages, bounds around the identity from reg_bound (reg/linear.hpp:258-263, 370-420)."""
    p = _lib.LinearParam()
    L.regb_linear_param_default(C.byref(p))
    s = _lib.RunnerState()
    fd = np.array([182, 218, 182], np.int32)
    vs = np.array([1, 1, 1], np.float32)
    arg = np.array([0, 0, 0, 0, 0, 0, 1, 1, 1, 0, 0, 0], np.float32)
    st = L.regb_runner_state_from_param(fd.ctypes.data_as(C.c_void_p), vs.ctypes.data_as(C.c_void_p),
                                        fd.ctypes.data_as(C.c_void_p), vs.ctypes.data_as(C.c_void_p),
                                        arg.ctypes.data_as(C.c_void_p), C.byref(p), C.byref(s))
    assert st == 0
    assert list(s.reg_list[: s.n_reg]) == [1, 5, 7, 15]
    assert s.search_count == 16 and s.multi_resolution == 1 and s.max_iterations == 128
    up = np.array(s.arg_upper[:], np.float32)
    lo = np.array(s.arg_lower[:], np.float32)
    assert up[0] == np.float32(np.float32(182 * 0.5) * np.float32(0.75))   # half extent * 0.75
    assert up[1] == np.float32(np.float32(218 * 0.5) * np.float32(0.75))
    assert up[3] == np.float32(0.0) + np.float32(1.57079632679) * np.float32(0.4)
    assert up[6] == np.float32(1.5) and lo[6] == np.float32(0.7)
    assert up[9] == np.float32(0.1) and lo[9] == np.float32(-0.1)
    p.bound = 1  # narrow: around arg, no search, no pyramid
    L.regb_runner_state_from_param(fd.ctypes.data_as(C.c_void_p), vs.ctypes.data_as(C.c_void_p),
                                   fd.ctypes.data_as(C.c_void_p), vs.ctypes.data_as(C.c_void_p),
                                   arg.ctypes.data_as(C.c_void_p), C.byref(p), C.byref(s))
    assert s.search_count == 0 and s.multi_resolution == 0


def test_mi_rejects_rows_wider_than_16_bit_counters(L):
    """The 256-bin MI counts in 16-bit per-block counters and a block holds at least one
    row of the fixed grid, so a fixed width above 65535 is an argument error (checked
    before anything reaches the device), for regb_mi_cost and regb_mi_cost_noalloc."""
    buf = np.zeros(70000, np.uint8)
    wide = _lib.Volume(buf.ctypes.data_as(C.c_void_p), (C.c_int * 3)(70000, 1, 1), _lib.U8, _lib.HOST)
    small = _lib.Volume(buf.ctypes.data_as(C.c_void_p), (C.c_int * 3)(8, 8, 8), _lib.U8, _lib.HOST)
    T = np.zeros(12, np.float32)
    cost = np.zeros(1, np.float64)
    st = L.regb_mi_cost(C.byref(wide), C.byref(small), T.ctypes.data_as(C.c_void_p), 1,
                        cost.ctypes.data_as(C.c_void_p), None, None)
    assert st == _lib.REGB_ERR_ARG and b"65535" in L.regb_last_error()
    fd = np.array([70000, 1, 1], np.int32)
    md = np.array([8, 8, 8], np.int32)
    st = L.regb_mi_cost_noalloc(buf.ctypes.data_as(C.c_void_p), fd.ctypes.data_as(C.c_void_p),
                                buf.ctypes.data_as(C.c_void_p), md.ctypes.data_as(C.c_void_p),
                                T.ctypes.data_as(C.c_void_p), 1, cost.ctypes.data_as(C.c_void_p), None)
    assert st == _lib.REGB_ERR_ARG and b"65535" in L.regb_last_error()


# The ctypes mirrors of the header's structs: every field at the header's offset and
# every struct of the header's size, so a field added on one side only cannot go unnoticed.
MIRRORED = {"Volume": "regb_volume", "Field": "regb_field", "LinearParam": "regb_linear_param",
            "CdmParam": "regb_cdm_param", "Stats": "regb_stats", "RunnerState": "regb_runner_state",
            "EngineConfig": "regb_engine_config", "NiftiInfo": "regb_nifti_info", "Job": "regb_job",
            "Result": "regb_result", "EngineStats": "regb_engine_stats"}


def test_ctypes_structs_match_header(tmp_path):
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "regb200.h"', "int main(void) {"]
    expect = []
    for py, c in MIRRORED.items():
        cls = getattr(_lib, py)
        lines.append(f'printf("%zu\\n", sizeof({c}));')
        expect.append(C.sizeof(cls))
        for name, _ in cls._fields_:
            lines.append(f'printf("%zu\\n", offsetof({c}, {name}));')
            expect.append(getattr(cls, name).offset)
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = [int(v) for v in subprocess.check_output([str(exe)]).split()]
    assert got == expect
