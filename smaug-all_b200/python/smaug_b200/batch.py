"""Python binding of the batch C ABI (smaug_batch_* in include/smaug_b200.h).

A batch advances many independent simulations of one ndim and one precision
(any sizes, each with its own parameters and dt) together: one launch per RK
stage for all of them, replayed from CUDA graphs.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import PREC_FP64, SMAUG_OK, SmaugError, _f64, _PD, load_library, make_params

SMAUG_ERR_FULL = -5


def footprint(prob, precision: int = PREC_FP64, dt_mode: int = 1, dt0: float = 0.0) -> int:
    """Arena bytes one simulation of `prob` takes in a batch (host only)."""
    lib = load_library()
    p = make_params(prob, rk4=True, dt_mode=dt_mode, dt0=dt0, precision=precision)
    out = ctypes.c_size_t()
    rc = lib.smaug_batch_footprint(ctypes.byref(p), ctypes.byref(out))
    if rc != SMAUG_OK:
        raise SmaugError(f"smaug_batch_footprint failed ({rc})")
    return int(out.value)


class Batch:
    """Many simulations resident on one GPU, stepped together."""

    def __init__(self, ndim: int, precision: int = PREC_FP64, arena_bytes: int = 1 << 30, max_sims: int = 256,
                 device: int = 0):
        self.lib = load_library()
        self.ndim = ndim
        self.precision = precision
        self.max_sims = max_sims
        self.h = ctypes.c_void_p()
        rc = self.lib.smaug_batch_create(ndim, precision, device, arena_bytes, max_sims, ctypes.byref(self.h))
        self._check(rc, "smaug_batch_create")
        self.probs: dict[int, object] = {}

    def _check(self, rc, what):
        if rc != SMAUG_OK:
            msg = self.lib.smaug_batch_last_error(self.h).decode() if self.h else ""
            raise SmaugError(f"{what} failed ({rc}): {msg}")

    def add(self, prob, nsteps: int, dt_mode: int = 1, dt0: float = 0.0, w=None, delx=None) -> int | None:
        """Admit a simulation; its slot, or None when the batch is full.  w:
        the initial state (default prob.w), e.g. a view of pinned memory;
        delx: the metric, ndim grid-shaped arrays back to back (default
        prob.delx())."""
        p = make_params(prob, rk4=True, dt_mode=dt_mode, dt0=dt0, precision=self.precision)
        if delx is None:
            delx = np.concatenate([a.ravel() for a in prob.delx()])
        delx = _f64(delx)
        if delx.size != prob.ndim * prob.w[0].size:
            raise SmaugError("metric size does not match the problem")
        w = _f64(prob.w if w is None else w)
        if w.size != prob.w.size:
            raise SmaugError("state size does not match the problem")
        slot = ctypes.c_int(-1)
        rc = self.lib.smaug_batch_add(self.h, ctypes.byref(p), delx.ctypes.data_as(_PD), w.ctypes.data_as(_PD),
                                      int(nsteps), ctypes.byref(slot))
        if rc == SMAUG_ERR_FULL:
            return None
        self._check(rc, "smaug_batch_add")
        self.probs[slot.value] = prob
        return slot.value

    def remove(self, slot: int):
        self._check(self.lib.smaug_batch_remove(self.h, slot), "smaug_batch_remove")
        self.probs.pop(slot, None)

    def step(self, n: int = 1):
        self._check(self.lib.smaug_batch_step(self.h, n), "smaug_batch_step")

    def poll(self) -> np.ndarray:
        """Steps left per slot (-1: free slot)."""
        out = (ctypes.c_longlong * self.max_sims)()
        self._check(self.lib.smaug_batch_poll(self.h, out, self.max_sims), "smaug_batch_poll")
        return np.frombuffer(out, dtype=np.int64).copy()

    def poll_begin(self) -> int:
        """Snapshot the steps left per slot behind the steps queued so far
        (does not wait); returns its ticket."""
        t = ctypes.c_longlong(-1)
        self._check(self.lib.smaug_batch_poll_begin(self.h, ctypes.byref(t)), "smaug_batch_poll_begin")
        return t.value

    def poll_end(self, ticket: int) -> np.ndarray:
        """Wait for snapshot `ticket` only: steps left per slot (-1: free)."""
        out = (ctypes.c_longlong * self.max_sims)()
        self._check(self.lib.smaug_batch_poll_end(self.h, ticket, out, self.max_sims), "smaug_batch_poll_end")
        return np.frombuffer(out, dtype=np.int64).copy()

    def state_async(self, slot: int, out: np.ndarray):
        """Queue the read of a simulation that had finished in the last snapshot
        poll_end returned; out (best pinned) is filled by io_wait()."""
        prob = self.probs[slot]
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != prob.w.size:
            raise SmaugError("out must be a C-contiguous float64 array of the problem's size")
        self._check(self.lib.smaug_batch_get_state_async(self.h, slot, out.ctypes.data_as(_PD), out.size),
                    "smaug_batch_get_state_async")
        return out

    def io_wait(self):
        self._check(self.lib.smaug_batch_io_wait(self.h), "smaug_batch_io_wait")

    def sync(self):
        bad = ctypes.c_int(-1)
        self._check(self.lib.smaug_batch_sync(self.h, ctypes.byref(bad)), "smaug_batch_sync")

    def status(self) -> tuple[int, int, str]:
        """Wait, then (status, slot, message): the first simulation error
        (SMAUG_ERR_NONFINITE when a simulation's dt or wave speeds became
        non-finite; that simulation stops, the others go on) and its slot, or
        (0, -1, "")."""
        bad = ctypes.c_int(-1)
        rc = self.lib.smaug_batch_sync(self.h, ctypes.byref(bad))
        msg = self.lib.smaug_batch_last_error(self.h).decode() if rc != SMAUG_OK else ""
        return rc, bad.value, msg

    def state(self, slot: int, out: np.ndarray | None = None) -> np.ndarray:
        prob = self.probs[slot]
        if out is None:
            out = np.empty(prob.w.shape, dtype=np.float64)
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != prob.w.size:
            raise SmaugError("out must be a C-contiguous float64 array of the problem's size")
        self._check(self.lib.smaug_batch_get_state(self.h, slot, out.ctypes.data_as(_PD), out.size),
                    "smaug_batch_get_state")
        return out

    def scalars(self, slot: int) -> dict:
        out = (ctypes.c_double * 8)()
        self._check(self.lib.smaug_batch_get_scalars(self.h, slot, out), "smaug_batch_get_scalars")
        nd = self.ndim
        return {"dt": out[0], "maxcourant": out[1], "maxviscoef": out[2], "dtdiffvisc": out[3],
                "cmax": list(out[4:4 + nd]), "steps": int(out[7])}

    def tune(self, reps: int = 5):
        """Autotune the tile shape; returns (chosen variant, ms per variant)."""
        v = ctypes.c_int(-1)
        ms = (ctypes.c_double * 16)()
        self._check(self.lib.smaug_batch_tune(self.h, reps, ctypes.byref(v), ms, 16), "smaug_batch_tune")
        nv = 11 if self.ndim == 2 else 10
        return v.value, list(ms[:nv])

    def set_variant(self, v: int):
        self._check(self.lib.smaug_batch_set_variant(self.h, v), "smaug_batch_set_variant")

    def profile_stages(self, enable: bool = True):
        self._check(self.lib.smaug_batch_profile_stages(self.h, int(enable)), "smaug_batch_profile_stages")

    def stage_times(self):
        """(total ms, launches) of the stage kernels timed since the last call."""
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        self._check(self.lib.smaug_batch_stage_times(self.h, ctypes.byref(ms), ctypes.byref(n)),
                    "smaug_batch_stage_times")
        return ms.value, n.value

    def info(self) -> dict:
        f, big, n = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_int()
        self._check(self.lib.smaug_batch_info(self.h, ctypes.byref(f), ctypes.byref(big), ctypes.byref(n)),
                    "smaug_batch_info")
        return {"free_bytes": int(f.value), "largest_free": int(big.value), "sims": int(n.value)}

    @property
    def stream(self) -> int:
        return self.lib.smaug_batch_stream(self.h) or 0

    @property
    def launches(self) -> int:
        return int(self.lib.smaug_batch_launch_count(self.h))

    def close(self):
        if self.h:
            self.lib.smaug_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
