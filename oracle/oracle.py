"""ctypes bindings for the oracle -- TEST INFRASTRUCTURE ONLY.

* ``Oracle``     -- our C restatement (oracle/smaug_oracle.c), built into
                    ``oracle/libsmaug_oracle.so``.
* ``Reference``  -- the SMAUG reference's own sources built for the host by
                    ``oracle/ref_shim/build_ref.py`` into ``oracle/_ref/``.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  Both classes work on problems from smaug_b200.problems.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libsmaug_oracle.so"
REF_DIR = HERE / "_ref"

_D = ctypes.c_double
_I = ctypes.c_int
_PD = ctypes.POINTER(_D)
_PI = ctypes.POINTER(_I)


def build_oracle(force: bool = False) -> Path:
    src = HERE / "smaug_oracle.c"
    if force or not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-o", str(LIB),
                        str(src), "-lm"], check=True)
    return LIB


class _Driver(ctypes.Structure):
    _fields_ = [("on", _I), ("dir", _I), ("amp", _D), ("period", _D), ("center", _D * 3),
                ("width", _D * 3), ("xmin", _D * 3), ("dx", _D * 3)]


class _Grid(ctypes.Structure):
    _fields_ = [("ndim", _I), ("n", _I * 3), ("gamma", _D), ("chyp", _D * 13),
                ("btype", _I * 3), ("g", _D * 3), ("courant", _D), ("hyperdif", _I),
                ("delx", _PD * 3), ("drv", ctypes.POINTER(_Driver)), ("bmask", _I * 3), ("fixed", _PD),
                ("divb", _I), ("dxs", _D * 3)]


class _State(ctypes.Structure):
    _fields_ = [("dt", _D), ("dtdiffvisc", _D), ("maxviscoef", _D), ("maxcourant", _D),
                ("cmax", _D * 3), ("t", _D)]


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_PD)


class Oracle:
    """FP64 CPU oracle for one problem (single step or RK4)."""

    def __init__(self, prob, dt_fixed: float = 0.0):
        self.lib = ctypes.CDLL(str(build_oracle()))
        L = self.lib
        L.sm_oracle_step.argtypes = [ctypes.POINTER(_Grid), _PD, _I, _I, _I, ctypes.POINTER(_State), _PD]
        L.sm_oracle_stage.argtypes = [ctypes.POINTER(_Grid), _PD, _PD, _PD, _D, _PD]
        L.sm_oracle_stage.restype = _D
        L.sm_oracle_select_dt.argtypes = [ctypes.POINTER(_Grid), _PD, _I, ctypes.POINTER(_State)]
        L.sm_oracle_select_dt.restype = _D
        L.sm_oracle_cmax.argtypes = [ctypes.POINTER(_Grid), _PD, _PD]
        L.sm_oracle_cfast.argtypes = [ctypes.POINTER(_Grid), _PD, _I, _PD]
        L.sm_oracle_boundary.argtypes = [ctypes.POINTER(_Grid), _PD]
        self.prob = prob
        self.delx = [np.ascontiguousarray(a, dtype=np.float64) for a in prob.delx()]  # per cell
        g = _Grid()
        g.ndim = prob.ndim
        for d in range(3):
            g.n[d] = prob.n[d] if d < prob.ndim else 1
            g.btype[d] = prob.btype[d] if d < prob.ndim else 0
            g.g[d] = prob.g[d] if d < len(prob.g) else 0.0
            g.delx[d] = _ptr(self.delx[d]) if d < prob.ndim else _PD()
        g.gamma = prob.gamma
        for f in range(len(prob.chyp)):
            g.chyp[f] = prob.chyp[f]
        g.courant = prob.courant
        g.hyperdif = prob.hyperdif
        drv = getattr(prob, "driver", None)
        self.drv = _Driver()
        if drv:
            self.drv.on = 1
            self.drv.dir = int(drv.get("dir", 0))
            self.drv.amp = float(drv["amp"])
            self.drv.period = float(drv.get("period", 0.0))
            for d in range(prob.ndim):
                self.drv.center[d] = float(drv["center"][d])
                self.drv.width[d] = float(drv["width"][d])
                self.drv.xmin[d] = float(prob.xmin[d])
                self.drv.dx[d] = float(prob.dx[d])
            g.drv = ctypes.pointer(self.drv)
        bm = tuple(getattr(prob, "bmask", (0, 0, 0))) + (0, 0, 0)
        for d in range(3):
            g.bmask[d] = int(bm[d]) if d < prob.ndim else 0
        # fixed boundaries keep the values of the state as loaded (captured
        # before the initial ghost fill, as iosmaug.cpp:645-654 does at it=-1)
        self.fixed = np.ascontiguousarray(prob.w, dtype=np.float64).copy()
        g.fixed = _ptr(self.fixed)
        g.divb = int(getattr(prob, "divb", 0))
        for d in range(prob.ndim):
            g.dxs[d] = float(prob.dx[d])
        self.g = g
        self.s = _State()
        self.s.dt = 1.0e-8 if dt_fixed == 0.0 else dt_fixed
        # initial ghost fill of the evolved fields, as iosmaug.cpp:786-794
        self.w = self.boundary(np.ascontiguousarray(prob.w, dtype=np.float64))
        self.work = np.zeros((4,) + self.w.shape)
        self.nstep = 0

    def step(self, nsteps: int = 1, rk4: bool = True, dt_mode: int = 1):
        for _ in range(nsteps):
            self.nstep += 1
            self.lib.sm_oracle_step(ctypes.byref(self.g), _ptr(self.w), self.nstep, int(rk4), dt_mode,
                                    ctypes.byref(self.s), _ptr(self.work))
        return self.w

    def stage(self, win, wbase, h, cmax):
        out = np.empty_like(win)
        cm = np.ascontiguousarray(cmax, dtype=np.float64)
        nu = self.lib.sm_oracle_stage(ctypes.byref(self.g), _ptr(win), _ptr(wbase), _ptr(out), h, _ptr(cm))
        return out, nu

    def cmax(self, w):
        out = np.zeros(3)
        self.lib.sm_oracle_cmax(ctypes.byref(self.g), _ptr(np.ascontiguousarray(w)), _ptr(out))
        return out[: self.prob.ndim]

    def cfast(self, w, dim):
        out = np.zeros(w.shape[1:])
        self.lib.sm_oracle_cfast(ctypes.byref(self.g), _ptr(np.ascontiguousarray(w)), dim, _ptr(out))
        return out

    def boundary(self, w):
        w = np.ascontiguousarray(w.copy())
        self.lib.sm_oracle_boundary(ctypes.byref(self.g), _ptr(w))
        return w

    @property
    def dt(self):
        return self.s.dt

    @property
    def t(self):
        return self.s.t


class Reference:
    """The reference's own step, built for the host (oracle/_ref).

    The reference library holds one global simulation; create one instance per
    process (tests run it in a subprocess when they need more)."""

    _loaded: dict = {}

    def __init__(self, prob, variant: str = ""):
        """variant "drv": the 2-D build with the spicule model's driver."""
        path = REF_DIR / f"libsmaug_ref{prob.ndim}d{'_' + variant if variant else ''}.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run oracle/ref_shim/build_ref.py")
        L = ctypes.CDLL(str(path))
        L.ref_init.argtypes = [_PI, _PD, _PD, _D, _PD, _PI, _D, _I, _I, _D, _PD]
        L.ref_set_state.argtypes = [_PD]
        L.ref_get_state.argtypes = [_PD, _I]
        L.ref_get_wd.argtypes = [_PD]
        L.ref_get_dt.restype = _D
        L.ref_get_scalar.restype = _D
        L.ref_set_dt.argtypes = [_D]
        L.ref_set_maxviscoef.argtypes = [_D]
        self.lib = L
        self.prob = prob
        D = prob.ndim
        n = (_I * D)(*prob.n)
        xmin = (_D * D)(*prob.xmin)
        dx = (_D * D)(*prob.dx)
        chyp = (_D * len(prob.chyp))(*prob.chyp)
        bt = (_I * D)(*prob.btype)
        g = (_D * 3)(*(list(prob.g) + [0.0] * 3)[:3])
        L.ref_init(n, xmin, dx, prob.gamma, chyp, bt, prob.courant, 1, prob.hyperdif, 0.0, g)
        # fields that take asymm on symm dims (the reference keeps a type per field)
        bm = tuple(getattr(prob, "bmask", (0, 0, 0))) + (0, 0, 0)
        nw = 2 + 2 * D
        for d in range(D):
            if prob.btype[d] == 6:
                for f in range(nw):
                    if (bm[d] >> f) & 1:
                        L.ref_set_btype(f, d, 7)
        if getattr(prob, "divb", 0):
            L.ref_set_divb(1)
        w = np.ascontiguousarray(prob.w)
        L.ref_set_state(_ptr(w))
        self.nstep = 0

    def step(self, nsteps: int = 1):
        for _ in range(nsteps):
            self.nstep += 1
            self.lib.ref_step(self.nstep)
        return self.state()

    def state(self, slot: int = 1):
        out = np.zeros(self.prob.w.shape)
        self.lib.ref_get_state(_ptr(out), slot)
        return out

    def derived(self):
        nderv = self.lib.ref_nderv()
        out = np.zeros((nderv,) + self.prob.w.shape[1:])
        self.lib.ref_get_wd(_ptr(out))
        return out

    @property
    def dt(self):
        return self.lib.ref_get_dt()

    def scalar(self, which: int) -> float:
        return self.lib.ref_get_scalar(which)
