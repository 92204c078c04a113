"""The C ABI library builds, loads and exports every entry point declared in
include/smaug_b200.h (no device work: these run without a GPU)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from smaug_b200 import LIB_PATH, load_library

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "smaug_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(smaug_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["smaug_create", "smaug_destroy", "smaug_set_metric", "smaug_set_state", "smaug_get_state",
                 "smaug_step", "smaug_sync", "smaug_get_scalars", "smaug_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    assert LIB_PATH.exists(), "libsmaug_b200.so not built"
    lib = ctypes.CDLL(str(LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_pure_host_entry_points():
    lib = load_library()
    assert lib.smaug_nvar(2) == 10 and lib.smaug_nvar(3) == 13
    lib.smaug_last_error.restype = ctypes.c_char_p
    assert lib.smaug_last_error(None) == b"null context"
    assert lib.smaug_destroy(None) == 0


def test_create_rejects_bad_arguments():
    from smaug_b200 import Params
    lib = load_library()
    p = Params()
    p.ndim = 4
    h = ctypes.c_void_p()
    rc = lib.smaug_create(ctypes.byref(p), 0, ctypes.byref(h))
    assert rc == -1
    assert b"ndim" in lib.smaug_last_error(h)
    lib.smaug_destroy(h)
    p.ndim = 2
    p.n[0], p.n[1] = 8, 40
    h = ctypes.c_void_p()
    assert lib.smaug_create(ctypes.byref(p), 0, ctypes.byref(h)) == -1
    lib.smaug_destroy(h)


def test_create_rejects_bad_precision():
    """Parameter checks run before any CUDA call, so they need no GPU."""
    from smaug_b200 import PREC_MIXED, Params
    lib = load_library()
    lib.smaug_last_error.restype = ctypes.c_char_p
    p = Params()
    p.ndim = 2
    p.n[0], p.n[1], p.n[2] = 20, 20, 1
    p.rk4 = 1
    p.precision = 7
    h = ctypes.c_void_p()
    assert lib.smaug_create(ctypes.byref(p), 0, ctypes.byref(h)) == -1
    assert b"precision" in lib.smaug_last_error(h)
    lib.smaug_destroy(h)
    for rk4, exact in [(0, 0), (1, 1)]:
        p.precision, p.rk4, p.exact = PREC_MIXED, rk4, exact
        h = ctypes.c_void_p()
        assert lib.smaug_create(ctypes.byref(p), 0, ctypes.byref(h)) == -1
        assert b"mixed" in lib.smaug_last_error(h)
        lib.smaug_destroy(h)


def test_batch_footprint_and_argument_checks():
    """Batch footprints and parameter checks are host-only."""
    from smaug_b200 import PREC_FP64, PREC_MIXED, footprint, problems
    p = problems.orszag_tang(30)
    N, NW, NB = p.ncells, 6, 4
    a = lambda x: (x + 255) // 256 * 256  # noqa: E731  (arena blocks are 256-byte aligned)
    nl = p.n[0] + p.n[1] + 1
    base = a(16 * nl) + a(8 * nl) + a(8 * N) + a(8 * NB * N) + a(8 * NW * N)  # metric lines + reciprocals, driver
    fp64 = footprint(p, PREC_FP64)
    mixed = footprint(p, PREC_MIXED)
    # scalars block + metric and driver lines + dxlast + backgrounds + W0, then 3 FP64 or 5 FP32 buffers
    assert fp64 - mixed == 3 * a(8 * NW * N) - 5 * a(4 * NW * N)
    assert fp64 > base + 3 * a(8 * NW * N) and fp64 - (base + 3 * a(8 * NW * N)) <= 1024
    lib = load_library()
    h = ctypes.c_void_p()
    assert lib.smaug_batch_create(4, 0, 0, 1 << 20, 4, ctypes.byref(h)) == -1
    assert b"ndim" in lib.smaug_batch_last_error(h)
    lib.smaug_batch_destroy(h)
    h = ctypes.c_void_p()
    assert lib.smaug_batch_create(2, 5, 0, 1 << 20, 4, ctypes.byref(h)) == -1
    lib.smaug_batch_destroy(h)


def test_params_struct_layout_matches_header(tmp_path):
    """The ctypes mirror of smaug_params has the C struct's size and offsets."""
    import subprocess

    from smaug_b200 import Params
    names = [f[0] for f in Params._fields_]
    src = tmp_path / "lay.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "smaug_b200.h"\nint main(void){\n'
                   '  printf("%zu\\n", sizeof(smaug_params));\n'
                   + "".join(f'  printf("%zu\\n", offsetof(smaug_params, {n}));\n' for n in names)
                   + "  return 0;\n}\n")
    exe = tmp_path / "lay"
    subprocess.run(["gcc", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(Params)
    assert vals[1:] == [getattr(Params, n).offset for n in names]


def test_initgrid_bits_equal_reference_metric():
    """smaug_initgrid (C++, the reference's initgrid from positions) gives the
    bits of problems.metric, the restatement the oracle and the fixtures use,
    on 2-D and 3-D grids with positions as init_parallel sets them."""
    from smaug_b200 import initgrid, problems
    for prob in (problems.orszag_tang(20, ny=12), problems.blast_wave(7, seed=2), problems.atmosphere(24, 10)):
        D = prob.ndim
        shape = prob.w.shape[1:]
        pos = []
        for d in range(D):
            x = prob.xmin[d] + np.arange(prob.n[d]) * prob.dx[d]
            view = [1] * D
            view[D - 1 - d] = prob.n[d]
            pos.append(np.broadcast_to(x.reshape(view), shape))
        got = initgrid(prob.n, pos, prob.dx)
        want = prob.delx()
        for d in range(D):
            assert np.array_equal(got[d], want[d]), (prob.name, d)


def test_host_driver_is_built_and_links():
    """The C host driver links against the library and runs without a GPU
    as far as its usage text."""
    import subprocess

    from smaug_b200.build import HOST_EXE
    assert HOST_EXE.exists(), "smaug_run not built"
    r = subprocess.run([str(HOST_EXE), "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "usage: smaug_run" in r.stderr
    r = subprocess.run([str(HOST_EXE)], capture_output=True, text=True)
    assert r.returncode == 2
