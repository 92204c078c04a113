"""VAC configuration files (the reference's ascii .ini and binary .out
formats) through the C ABI (smaug_vac_* in include/smaug_b200.h).

Arrays follow the reference's layout: positions (ndim, [n2,] n1, n0) and
states (nw, [n2,] n1, n0), x fastest.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import SMAUG_OK, SmaugError, load_library
from .problems import NG, Problem, _chyp, nvar


class VacHeader(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 80), ("it", ctypes.c_int), ("t", ctypes.c_double),
                ("ndim", ctypes.c_int), ("neqpar", ctypes.c_int), ("nw", ctypes.c_int), ("n", ctypes.c_int * 3),
                ("eqpar", ctypes.c_double * 16), ("names", ctypes.c_char * 80)]


_PD = ctypes.POINTER(ctypes.c_double)


def _lib():
    L = load_library()
    if not getattr(L, "_vac_ready", False):
        for fn in (L.smaug_vac_read_ascii, L.smaug_vac_read_binary):
            fn.argtypes = [ctypes.c_char_p, ctypes.POINTER(VacHeader), _PD, ctypes.c_size_t, _PD, ctypes.c_size_t]
        for fn in (L.smaug_vac_write_ascii, L.smaug_vac_write_binary):
            fn.argtypes = [ctypes.c_char_p, ctypes.POINTER(VacHeader), _PD, _PD]
        L.smaug_vac_last_error.restype = ctypes.c_char_p
        L._vac_ready = True
    return L


def _check(rc, what):
    if rc != SMAUG_OK:
        raise SmaugError(f"{what}: {_lib().smaug_vac_last_error().decode()}")


def _header_dict(h: VacHeader) -> dict:
    return {"name": h.name.decode(errors="replace"), "it": h.it, "t": h.t, "ndim": h.ndim, "neqpar": h.neqpar,
            "nw": h.nw, "n": tuple(h.n[: h.ndim]), "eqpar": list(h.eqpar[: h.neqpar]),
            "names": h.names.decode(errors="replace")}


def _read(fn, path, what):
    L = _lib()
    h = VacHeader()
    _check(fn(str(path).encode(), ctypes.byref(h), None, 0, None, 0), what)
    shape = tuple(reversed(h.n[: h.ndim]))
    pos = np.empty((h.ndim,) + shape)
    w = np.empty((h.nw,) + shape)
    _check(fn(str(path).encode(), ctypes.byref(h), pos.ctypes.data_as(_PD), pos.size, w.ctypes.data_as(_PD), w.size),
           what)
    del L
    return _header_dict(h), pos, w


def read_ascii(path):
    """(header dict, positions, state) of a VAC ascii file."""
    return _read(_lib().smaug_vac_read_ascii, path, f"read {path}")


def read_binary(path):
    """(header dict, positions, state) of a VAC binary file."""
    return _read(_lib().smaug_vac_read_binary, path, f"read {path}")


def _write(fn, path, header: dict, pos, w, what):
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    h = VacHeader()
    h.name = header.get("name", "smaug_b200").encode()[:79]
    h.it = int(header.get("it", 0))
    h.t = float(header.get("t", 0.0))
    h.ndim = pos.shape[0]
    h.nw = w.shape[0]
    n = list(reversed(w.shape[1:]))
    for d in range(3):
        h.n[d] = n[d] if d < len(n) else 1
    eq = list(header.get("eqpar", []))
    h.neqpar = len(eq)
    for k, v in enumerate(eq):
        h.eqpar[k] = float(v)
    h.names = header.get("names", "").encode()[:79]
    if pos.shape[1:] != w.shape[1:]:
        raise SmaugError("positions and state must cover the same grid")
    _check(fn(str(path).encode(), ctypes.byref(h), pos.ctypes.data_as(_PD), w.ctypes.data_as(_PD)), what)


def write_ascii(path, header: dict, pos, w):
    _write(_lib().smaug_vac_write_ascii, path, header, pos, w, f"write {path}")


def write_binary(path, header: dict, pos, w):
    _write(_lib().smaug_vac_write_binary, path, header, pos, w, f"write {path}")


def positions(prob: Problem) -> np.ndarray:
    """Cell positions xmin + i dx of a problem, (ndim, [n2,] n1, n0)."""
    D = prob.ndim
    shape = tuple(reversed(prob.n))
    out = np.empty((D,) + shape)
    for d in range(D):
        x = prob.xmin[d] + np.arange(prob.n[d]) * prob.dx[d]
        out[d] = np.broadcast_to(x.reshape((-1,) + (1,) * d), shape)
    return out


def header_for(prob: Problem, it: int = 0, t: float = 0.0, name: str = "smaug_b200") -> dict:
    """A VAC header for a problem's state: eqpar = gamma, eta (0), g_1..g_ndim."""
    D = prob.ndim
    names = {2: "x y h m1 m2 e b1 b2 eb rhob bg1 bg2   gamma eta   grav1 grav2",
             3: "x y z h m1 m2 m3 e b1 b2 b3 eb rhob bg1 bg2 bg3   gamma eta   grav1 grav2 grav3"}[D]
    return {"name": name, "it": it, "t": t, "eqpar": [prob.gamma, 0.0] + list(prob.g[:D]), "names": names}


def problem_from_vac(path, binary: bool = False, ghosts: str = "file", btype=None, courant: float = 0.3) -> Problem:
    """A problem from a VAC file whose state holds the reference's NVAR
    fields.  ghosts="file": the file's grid includes the 2 ghost layers per
    side; "pad": the file holds inner cells only, ghosts are added by a
    periodic fill.  gamma and gravity come from eqpar (gamma, eta, g...)."""
    hdr, pos, w = (read_binary if binary else read_ascii)(path)
    D = hdr["ndim"]
    if hdr["nw"] != nvar(D):
        raise SmaugError(f"{path}: {hdr['nw']} variables, the step needs {nvar(D)}")
    n = list(hdr["n"])
    dx = []
    for d in range(D):
        line = np.moveaxis(pos[d], D - 1 - d, -1).reshape(-1, n[d])[0]
        dx.append(float(line[1] - line[0]) if n[d] > 1 else 1.0)
    xmin = [float(pos[d].reshape(-1)[0]) for d in range(D)]
    if ghosts == "pad":
        from .problems import _periodic_fill
        w = np.stack([_periodic_fill(np.pad(f, NG)) for f in w])
        n = [m + 2 * NG for m in n]
        xmin = [xmin[d] - NG * dx[d] for d in range(D)]
    eq = hdr["eqpar"]
    g = tuple(eq[2:2 + D]) + (0.0,) * (3 - D) if len(eq) >= 2 + D else (0.0, 0.0, 0.0)
    return Problem(Path(str(path)).stem, D, tuple(n), tuple(dx), tuple(xmin), float(eq[0]), _chyp(D),
                   tuple(btype or (0,) * D), courant, np.ascontiguousarray(w), g=g,
                   meta={"vac": hdr, "ghosts": ghosts})
