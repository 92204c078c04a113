"""smaug_step_noalloc: the step for callers that cannot allocate device memory.

Some hosts cannot call cudaMalloc -- a framework whose caching allocator owns
the GPU's memory, or a serving loop that must not allocate after start-up --
so the library offers one entry point whose scratch (the Runge-Kutta stage
buffers and the device-side scalars) sits in a fixed device array inside the
library.  These tests call it through the C ABI with device buffers the test
owns and compare its output with the regular context API (smaug_create /
smaug_step) on the same inputs, within the tolerance of the other GPU tests,
on two calls in a row: the second call must not see anything the first left
in the shared scratch.

The file is collected last (tests/test_zz_*) so a run that stops at the first
failure has already run every other test.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from smaug_b200 import Engine, Params, load_library, problems

pytestmark = pytest.mark.gpu

RTOL = 1e-6  # the production-build tolerance of tests/test_gpu_parity.py


def _params(prob, rk4=True, exact=False):
    p = Params()
    p.ndim = prob.ndim
    for d in range(3):
        p.n[d] = prob.n[d] if d < prob.ndim else 1
        p.btype[d] = prob.btype[d] if d < prob.ndim else 0
        p.g[d] = 0.0
    p.gamma = prob.gamma
    p.courant = prob.courant
    for f in range(len(prob.chyp)):
        p.chyp[f] = float(prob.chyp[f])
    p.hyperdif = int(prob.hyperdif)
    p.rk4 = int(rk4)
    p.dt_mode = 1
    p.dt0 = 0.0
    p.exact = int(exact)
    return p


def _noalloc(lib, prob, w_in, nsteps, rk4=True, exact=False):
    import torch
    p = _params(prob, rk4, exact)
    delx = torch.from_numpy(np.concatenate([a.ravel() for a in prob.delx()])).cuda()
    win = torch.from_numpy(np.ascontiguousarray(w_in)).cuda()
    wout = torch.empty_like(win)
    sc = (ctypes.c_double * 8)()
    err = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.smaug_step_noalloc(ctypes.byref(p), ctypes.c_void_p(delx.data_ptr()), ctypes.c_void_p(win.data_ptr()),
                                ctypes.c_void_p(wout.data_ptr()), nsteps, ctypes.c_void_p(stream), sc, err, 256)
    assert rc == 0, err.value
    return wout.cpu().numpy(), list(sc)


def _regular(prob, w_in, nsteps, rk4=True, exact=False):
    eng = Engine(prob, rk4=rk4, exact=exact)
    eng.set_state(w_in)
    eng.step(nsteps)
    eng.sync()
    out = eng.state()
    s = eng.scalars()
    eng.close()
    return out, s


def _lib():
    lib = load_library()
    lib.smaug_step_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                       ctypes.c_char_p, ctypes.c_size_t]
    return lib


def _rel(a, b):
    return max(np.linalg.norm(a[f] - b[f]) / max(np.linalg.norm(b[f]), 1e-300) for f in range(a.shape[0]))


def test_noalloc_matches_regular_api_two_calls(need_gpu):
    lib = _lib()
    # call 1: 2-D Orszag-Tang, RK4
    p1 = problems.orszag_tang(48)
    a1, s1 = _noalloc(lib, p1, p1.w, 6)
    b1, t1 = _regular(p1, p1.w, 6)
    assert _rel(a1, b1) <= RTOL
    assert s1[0] == pytest.approx(t1["dt"], rel=RTOL)
    # call 2 right after, different problem and shape: the scratch holds call 1's data
    p2 = problems.blast_wave(14, seed=5)
    a2, s2 = _noalloc(lib, p2, p2.w, 3)
    b2, t2 = _regular(p2, p2.w, 3)
    assert _rel(a2, b2) <= RTOL
    assert s2[0] == pytest.approx(t2["dt"], rel=RTOL)
    # call 3: continue call 1's output in single-step mode (odd step count)
    a3, _ = _noalloc(lib, p1, a1, 3, rk4=False)
    b3, _ = _regular(p1, a1, 3, rk4=False)
    assert _rel(a3, b3) <= RTOL


def test_noalloc_rejects_oversized_grid(need_gpu):
    import torch
    lib = _lib()
    prob = problems.orszag_tang(16)
    p = _params(prob)
    p.n[0] = p.n[1] = 2048  # needs ~600 MB of scratch
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    err = ctypes.create_string_buffer(256)
    rc = lib.smaug_step_noalloc(ctypes.byref(p), ctypes.c_void_p(dummy.data_ptr()), ctypes.c_void_p(dummy.data_ptr()),
                                ctypes.c_void_p(dummy.data_ptr()), 1, None, None, err, 256)
    assert rc == -1
    assert b"maximum" in err.value


def test_noalloc_in_place_matches_regular_api(need_gpu):
    import torch
    lib = _lib()
    prob = problems.orszag_tang(40)
    p = _params(prob)
    delx = torch.from_numpy(np.concatenate([a.ravel() for a in prob.delx()])).cuda()
    w = torch.from_numpy(np.ascontiguousarray(prob.w)).cuda()
    err = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    # w_out == w_in: the header allows it; the result replaces the input
    rc = lib.smaug_step_noalloc(ctypes.byref(p), ctypes.c_void_p(delx.data_ptr()), ctypes.c_void_p(w.data_ptr()),
                                ctypes.c_void_p(w.data_ptr()), 4, ctypes.c_void_p(stream), None, err, 256)
    assert rc == 0, err.value
    b, _ = _regular(prob, prob.w, 4)
    assert _rel(w.cpu().numpy(), b) <= RTOL


def test_noalloc_bad_metric_leaves_input_untouched(need_gpu):
    import torch
    lib = _lib()
    prob = problems.orszag_tang(24)
    p = _params(prob)
    m = np.concatenate([a.ravel() for a in prob.delx()])
    m[len(m) // 3] = 0.0  # a zero cell width
    delx = torch.from_numpy(m).cuda()
    w0 = np.ascontiguousarray(prob.w).copy()
    w = torch.from_numpy(w0.copy()).cuda()
    err = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.smaug_step_noalloc(ctypes.byref(p), ctypes.c_void_p(delx.data_ptr()), ctypes.c_void_p(w.data_ptr()),
                                ctypes.c_void_p(w.data_ptr()), 3, ctypes.c_void_p(stream), None, err, 256)
    assert rc == -1
    assert b"metric" in err.value
    # in place: the caller's state is exactly as it was (no ghost fill, no step)
    assert np.array_equal(w.cpu().numpy(), w0)
