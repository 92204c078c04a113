"""Python binding of the B200 ideal-MHD step (libsmaug_b200.so, C ABI in
include/smaug_b200.h).

The library is the product; this module only marshals arguments.  It refuses
to run without the compiled CUDA library -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import problems  # noqa: F401

PKG = Path(__file__).resolve().parents[2]
LIB_PATH = PKG / "lib" / "libsmaug_b200.so"

_D = ctypes.c_double
_I = ctypes.c_int
_PD = ctypes.POINTER(_D)
_SZ = ctypes.c_size_t

SMAUG_OK = 0


class Params(ctypes.Structure):
    _fields_ = [("ndim", _I), ("n", _I * 3), ("gamma", _D), ("courant", _D), ("chyp", _D * 13),
                ("btype", _I * 3), ("g", _D * 3), ("hyperdif", _I), ("rk4", _I), ("dt_mode", _I),
                ("dt0", _D), ("exact", _I), ("precision", _I),
                ("drv_on", _I), ("drv_dir", _I), ("drv_amp", _D), ("drv_period", _D),
                ("drv_center", _D * 3), ("drv_width", _D * 3), ("xmin", _D * 3), ("dx", _D * 3),
                ("bmask", _I * 3), ("divb", _I)]


PREC_FP64 = 0   # SMAUG_PREC_FP64
PREC_MIXED = 1  # SMAUG_PREC_MIXED: FP32 stage states and stencils, FP64 where accuracy needs it


class SmaugError(RuntimeError):
    pass


_lib = None


def load_library(path: Path | None = None):
    """Load libsmaug_b200.so (raises if it is missing: no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise SmaugError(f"{p} not built: run `python -c 'import __graft_entry__ as g; g.build()'`")
    L = ctypes.CDLL(str(p))
    L.smaug_create.argtypes = [ctypes.POINTER(Params), _I, ctypes.POINTER(ctypes.c_void_p)]
    L.smaug_destroy.argtypes = [ctypes.c_void_p]
    L.smaug_set_metric.argtypes = [ctypes.c_void_p, _PD, _SZ]
    L.smaug_set_state.argtypes = [ctypes.c_void_p, _PD, _SZ]
    L.smaug_get_state.argtypes = [ctypes.c_void_p, _PD, _SZ]
    L.smaug_set_state_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _SZ]
    L.smaug_get_state_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _SZ]
    L.smaug_step.argtypes = [ctypes.c_void_p, _I]
    L.smaug_step_on.argtypes = [ctypes.c_void_p, _I, ctypes.c_void_p]
    L.smaug_stage.argtypes = [ctypes.c_void_p, _I, ctypes.c_void_p]
    L.smaug_initgrid.argtypes = [_I, ctypes.POINTER(_I), _PD, _PD, _PD]
    L.smaug_vac_last_error.restype = ctypes.c_char_p
    L.smaug_sync.argtypes = [ctypes.c_void_p]
    L.smaug_get_scalars.argtypes = [ctypes.c_void_p, _PD]
    L.smaug_stream.argtypes = [ctypes.c_void_p]
    L.smaug_stream.restype = ctypes.c_void_p
    L.smaug_launch_count.argtypes = [ctypes.c_void_p]
    L.smaug_launch_count.restype = ctypes.c_longlong
    L.smaug_last_error.argtypes = [ctypes.c_void_p]
    L.smaug_last_error.restype = ctypes.c_char_p
    L.smaug_nvar.argtypes = [_I]
    L.smaug_profile_stages.argtypes = [ctypes.c_void_p, _I]
    L.smaug_stage_times.argtypes = [ctypes.c_void_p, _PD, ctypes.POINTER(ctypes.c_longlong)]
    _LL = ctypes.c_longlong
    _VP = ctypes.c_void_p
    L.smaug_batch_footprint.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(_SZ)]
    L.smaug_batch_create.argtypes = [_I, _I, _I, _SZ, _I, ctypes.POINTER(_VP)]
    L.smaug_batch_destroy.argtypes = [_VP]
    L.smaug_batch_add.argtypes = [_VP, ctypes.POINTER(Params), _PD, _PD, _LL, ctypes.POINTER(_I)]
    L.smaug_batch_remove.argtypes = [_VP, _I]
    L.smaug_batch_step.argtypes = [_VP, _I]
    L.smaug_batch_poll.argtypes = [_VP, ctypes.POINTER(_LL), _I]
    L.smaug_batch_sync.argtypes = [_VP, ctypes.POINTER(_I)]
    L.smaug_batch_poll_begin.argtypes = [_VP, ctypes.POINTER(_LL)]
    L.smaug_batch_poll_end.argtypes = [_VP, _LL, ctypes.POINTER(_LL), _I]
    L.smaug_batch_get_state_async.argtypes = [_VP, _I, _PD, _SZ]
    L.smaug_batch_io_wait.argtypes = [_VP]
    L.smaug_batch_get_state.argtypes = [_VP, _I, _PD, _SZ]
    L.smaug_batch_get_scalars.argtypes = [_VP, _I, _PD]
    L.smaug_batch_tune.argtypes = [_VP, _I, ctypes.POINTER(_I), _PD, _I]
    L.smaug_batch_set_variant.argtypes = [_VP, _I]
    L.smaug_batch_info.argtypes = [_VP, ctypes.POINTER(_SZ), ctypes.POINTER(_SZ), ctypes.POINTER(_I)]
    L.smaug_batch_profile_stages.argtypes = [_VP, _I]
    L.smaug_batch_stage_times.argtypes = [_VP, _PD, ctypes.POINTER(_LL)]
    L.smaug_batch_stream.argtypes = [_VP]
    L.smaug_batch_stream.restype = _VP
    L.smaug_batch_launch_count.argtypes = [_VP]
    L.smaug_batch_launch_count.restype = _LL
    L.smaug_batch_last_error.argtypes = [_VP]
    L.smaug_batch_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def initgrid(n, pos, dx) -> list:
    """The metric from cell positions (smaug_initgrid, the reference's
    initgrid): pos is ndim grid-shaped arrays (storage order [k,] j, i) of the
    position components of every cell; returns ndim grid-shaped arrays."""
    lib = load_library()
    D = len(n)
    pos = _f64(np.stack([np.asarray(p) for p in pos]))
    out = np.empty_like(pos)
    nn = (_I * 3)(*(list(n) + [1] * (3 - D)))
    d = (_D * 3)(*(list(dx) + [0.0] * (3 - D)))
    rc = lib.smaug_initgrid(D, nn, pos.ctypes.data_as(_PD), d, out.ctypes.data_as(_PD))
    if rc != SMAUG_OK:
        raise SmaugError(f"smaug_initgrid failed ({rc}): {lib.smaug_vac_last_error().decode()}")
    return [out[k] for k in range(D)]


def make_params(prob, rk4: bool = True, dt_mode: int = 1, exact: bool = False, dt0: float = 0.0,
                precision: int = PREC_FP64) -> Params:
    """smaug_params for a problem (problems.Problem)."""
    p = Params()
    p.ndim = prob.ndim
    for d in range(3):
        p.n[d] = prob.n[d] if d < prob.ndim else 1
        p.btype[d] = prob.btype[d] if d < prob.ndim else 0
        p.g[d] = prob.g[d] if d < len(prob.g) else 0.0
    bm = tuple(getattr(prob, "bmask", (0, 0, 0))) + (0, 0, 0)
    for d in range(3):
        p.bmask[d] = int(bm[d]) if d < prob.ndim else 0
    p.gamma = prob.gamma
    p.divb = int(getattr(prob, "divb", 0))
    p.courant = prob.courant
    for f in range(len(prob.chyp)):
        p.chyp[f] = float(prob.chyp[f])
    p.hyperdif = int(prob.hyperdif)
    p.rk4 = int(rk4)
    p.dt_mode = int(dt_mode)
    p.dt0 = float(dt0)
    p.exact = int(exact)
    p.precision = int(precision)
    for d in range(prob.ndim):
        p.xmin[d] = float(prob.xmin[d])
        p.dx[d] = float(prob.dx[d])
    drv = getattr(prob, "driver", None)
    if drv:
        p.drv_on = 1
        p.drv_dir = int(drv.get("dir", 0))
        p.drv_amp = float(drv["amp"])
        p.drv_period = float(drv.get("period", 0.0))
        for d in range(prob.ndim):
            p.drv_center[d] = float(drv["center"][d])
            p.drv_width[d] = float(drv["width"][d])
    return p


class Engine:
    """One simulation resident on one GPU."""

    def __init__(self, prob, rk4: bool = True, dt_mode: int = 1, exact: bool = False, device: int = 0,
                 dt0: float = 0.0, precision: int = PREC_FP64):
        self.lib = load_library()
        self.prob = prob
        p = make_params(prob, rk4=rk4, dt_mode=dt_mode, exact=exact, dt0=dt0, precision=precision)
        self.params = p
        h = ctypes.c_void_p()
        rc = self.lib.smaug_create(ctypes.byref(p), device, ctypes.byref(h))
        self.h = h
        self._check(rc, "smaug_create")
        delx = _f64(np.concatenate([a.ravel() for a in prob.delx()]))
        self._check(self.lib.smaug_set_metric(self.h, delx.ctypes.data_as(_PD), delx.size), "smaug_set_metric")
        self.set_state(prob.w)

    def _check(self, rc, what):
        if rc != SMAUG_OK:
            msg = self.lib.smaug_last_error(self.h).decode() if self.h else ""
            raise SmaugError(f"{what} failed ({rc}): {msg}")

    def set_state(self, w):
        w = _f64(w)
        self._check(self.lib.smaug_set_state(self.h, w.ctypes.data_as(_PD), w.size), "smaug_set_state")

    def state(self) -> np.ndarray:
        out = np.empty(self.prob.w.shape, dtype=np.float64)
        self._check(self.lib.smaug_get_state(self.h, out.ctypes.data_as(_PD), out.size), "smaug_get_state")
        return out

    def set_state_device(self, ptr: int, count: int):
        self._check(self.lib.smaug_set_state_device(self.h, ctypes.c_void_p(ptr), count), "smaug_set_state_device")

    def get_state_device(self, ptr: int, count: int):
        self._check(self.lib.smaug_get_state_device(self.h, ctypes.c_void_p(ptr), count), "smaug_get_state_device")

    def step(self, n: int = 1):
        self._check(self.lib.smaug_step(self.h, n), "smaug_step")

    def step_on(self, n: int, stream: int):
        """n steps on the caller's CUDA stream (a cudaStream_t handle)."""
        self._check(self.lib.smaug_step_on(self.h, n, ctypes.c_void_p(stream)), "smaug_step_on")

    def stage(self, k: int, stream: int = 0):
        """RK stage k (1..4; 1 in single-step mode) of the current step."""
        self._check(self.lib.smaug_stage(self.h, k, ctypes.c_void_p(stream)), "smaug_stage")

    def sync(self):
        self._check(self.lib.smaug_sync(self.h), "smaug_sync")

    def scalars(self) -> dict:
        out = (_D * 8)()
        self._check(self.lib.smaug_get_scalars(self.h, out), "smaug_get_scalars")
        return {"dt": out[0], "maxcourant": out[1], "maxviscoef": out[2], "dtdiffvisc": out[3],
                "cmax": list(out[4:4 + self.prob.ndim]), "steps": int(out[7])}

    def profile_stages(self, enable: bool = True):
        self._check(self.lib.smaug_profile_stages(self.h, int(enable)), "smaug_profile_stages")

    def stage_times(self):
        """(total ms, launches) of the stage kernels timed since the last call."""
        ms = _D()
        n = ctypes.c_longlong()
        self._check(self.lib.smaug_stage_times(self.h, ctypes.byref(ms), ctypes.byref(n)), "smaug_stage_times")
        return ms.value, n.value

    @property
    def stream(self) -> int:
        return self.lib.smaug_stream(self.h) or 0

    @property
    def launches(self) -> int:
        return int(self.lib.smaug_launch_count(self.h))

    def close(self):
        if self.h:
            self.lib.smaug_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


from .batch import Batch, footprint  # noqa: E402,F401
