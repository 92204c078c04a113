"""Seeded synthetic initial states for the benchmark configurations.

The reference builds its initial states with per-model code
(``models/init_user.cu.*``, ``models/initialisation_user.h.*``) or reads VAC
config files; these generators produce the same kind of state directly, in the
reference's storage layout:

    w[f, k, j, i]   field-major, x fastest, 2 ghost layers per side,
    2-D fields  rho m1 m2 e b1 b2 eb rhob b1b b2b          (iotypes.h:213-215)
    3-D fields  rho m1 m2 m3 e b1 b2 b3 eb rhob b1b b2b b3b (iotypes.h:217-219)

Energies follow the synthetic-config convention e = p/(gamma-1) + rho v^2/2 +
B^2/2 (the reference OT model divides B^2/2 by rho, models/init_user.cu.ot).
Cell centres sit at xmin + (c - 2 + 1/2) dx for the blast wave and at
(c - 2) dx for Orszag-Tang (so the periodic images of the ghosts are exact).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

NG = 2  # ghost layers per side (ngi = 2, models/iosmaugparams.h.ot:1-3)


def nvar(ndim: int) -> int:
    return 4 + 3 * ndim


def field_ids(ndim: int) -> dict:
    D = ndim
    ids = {"rho": 0, "e": 1 + D, "eb": 2 + 2 * D, "rhob": 3 + 2 * D}
    for k in range(D):
        ids[f"m{k+1}"] = 1 + k
        ids[f"b{k+1}"] = 2 + D + k
        ids[f"b{k+1}b"] = 4 + 2 * D + k
    return ids


@dataclass
class Problem:
    """A fully specified run: grid, physics constants and initial state."""

    name: str
    ndim: int
    n: tuple            # cells per dim INCLUDING ghosts (x first)
    dx: tuple           # uniform spacing per dim
    xmin: tuple         # coordinate of cell 0 (a ghost) per dim
    gamma: float
    chyp: np.ndarray    # per field id
    btype: tuple        # per dim: 0 periodic, 3 cont, 4 contcd4, 5 fixed, 6 symm, 7 asymm
    courant: float
    w: np.ndarray       # (NVAR, [n2,] n1, n0) float64
    g: tuple = (0.0, 0.0, 0.0)
    hyperdif: int = 1
    meta: dict = field(default_factory=dict)
    # momentum driver: {"dir", "amp", "period", "center", "width"} (None: off)
    driver: dict | None = None
    # per dim: evolved fields (bit f) that take asymm where btype is symm
    bmask: tuple = (0, 0, 0)
    # 2-D: divergence-of-B source terms (the reference's divbon / divbfix)
    divb: int = 0

    @property
    def ncells(self) -> int:
        return int(np.prod(self.n))

    @property
    def interior(self) -> int:
        return int(np.prod([m - 2 * NG for m in self.n]))

    def delx(self):
        """Per-cell metric arrays (one per dim, grid-shaped), see metric()."""
        return metric(self.n, self.xmin, self.dx)


def metric(n, xmin, dx):
    """Cell widths exactly as the reference derives them (initgrid,
    init.cu:1118-1670): positions xmin + c*dx on every cell (init_parallel,
    init.cu:128-140) go into a padded copy, every position component is
    linearly extrapolated over the two outer layers of each direction in turn
    (q(ix) = (1+|ixe-ix|) q(ixe) - |ixe-ix| q(ixf)), and
    delx_d = (x_d[c+1] - x_d[c-1]) / 2 along d (0 replaced by dx).

    Returns a list of ndim arrays shaped like one field ([k,] j, i).  Inside
    the grid delx_d depends on the d coordinate only; the extrapolation
    perturbs the last bits in the ghost layers of the other directions."""
    D = len(n)
    nn = list(n) + [1] * (3 - D)
    shp = tuple(m + 2 for m in nn[:D]) + (1,) * (3 - D)   # (x, y, z) order
    T = []
    for d1 in range(D):
        t = np.zeros(shp)
        pos = xmin[d1] + np.arange(nn[d1]) * dx[d1]
        sl = [slice(1, nn[e] + 1) if e < D else slice(0, 1) for e in range(3)]
        view = [1, 1, 1]
        view[d1] = nn[d1]
        t[tuple(sl)] = pos.reshape(view)
        T.append(t)
    for d in range(D):
        m = nn[d]
        for (lo, hi, e, f) in ((m - 1, m + 1, m - 2, m - 3), (0, 2, 3, 4)):
            for d1 in range(D):
                t = np.moveaxis(T[d1], d, 0)
                for ix in range(lo, hi + 1):
                    a = abs(e - ix)
                    t[ix] = (1 + a) * t[e] - a * t[f]
    out = []
    for d in range(D):
        t = np.moveaxis(T[d], d, 0)
        dd = 0.5 * (t[2:nn[d] + 2] - t[0:nn[d]])
        dd = np.moveaxis(dd, 0, d)
        inner = tuple(slice(1, nn[e] + 1) if (e < D and e != d) else slice(None) for e in range(3))
        dd = dd[inner]
        dd = np.where(dd == 0, dx[d], dd)
        # (x, y, z) -> storage order ([z,] y, x)
        dd = np.transpose(dd, (2, 1, 0))[(0,) if D == 2 else slice(None)]
        out.append(np.ascontiguousarray(dd, dtype=np.float64))
    return out


def _chyp(ndim: int) -> np.ndarray:
    """chyp values of models/iosmaugparams.h.ot:171-179 (sedov3d uses the same
    per-kind values for its extra components)."""
    ids = field_ids(ndim)
    c = np.zeros(nvar(ndim))
    c[ids["rho"]] = 0.045
    c[ids["e"]] = 0.02
    for k in range(ndim):
        c[ids[f"m{k+1}"]] = 0.4
        c[ids[f"b{k+1}"]] = 0.02
    return c


def orszag_tang(nx: int = 256, ny: int | None = None, b0_scale: float = 1.0,
                rho_noise: float = 0.0, seed: int | None = None) -> Problem:
    """2-D Orszag-Tang vortex on [0,1]^2, periodic, zero background fields."""
    ny = nx if ny is None else ny
    n = (nx + 2 * NG, ny + 2 * NG)
    dx = (1.0 / nx, 1.0 / ny)
    x = (np.arange(n[0]) - NG) * dx[0]
    y = (np.arange(n[1]) - NG) * dx[1]
    X, Y = np.meshgrid(x, y, indexing="xy")
    gam = 5.0 / 3.0
    rho = np.full(X.shape, 25.0 / (36.0 * np.pi))
    if rho_noise:
        rng = np.random.default_rng(seed)
        inner = rho[NG:-NG, NG:-NG] * (1.0 + rho_noise * rng.standard_normal((ny, nx)))
        rho[NG:-NG, NG:-NG] = inner
        rho = _periodic_fill(rho)
    p = 5.0 / (12.0 * np.pi)
    B0 = b0_scale / np.sqrt(4.0 * np.pi)
    vx = -np.sin(2 * np.pi * Y)
    vy = np.sin(2 * np.pi * X)
    bx = -B0 * np.sin(2 * np.pi * Y)
    by = B0 * np.sin(4 * np.pi * X)
    w = np.zeros((nvar(2),) + X.shape)
    w[0] = rho
    w[1] = rho * vx
    w[2] = rho * vy
    w[3] = p / (gam - 1) + 0.5 * rho * (vx * vx + vy * vy) + 0.5 * (bx * bx + by * by)
    w[4] = bx
    w[5] = by
    w = np.stack([_periodic_fill(f) for f in w])
    return Problem("orszag_tang", 2, n, dx, (-NG * dx[0], -NG * dx[1]), gam, _chyp(2), (0, 0),
                   0.3, w, meta={"nx": nx, "ny": ny, "b0_scale": b0_scale, "rho_noise": rho_noise,
                                 "seed": seed})


# Stratified solar atmosphere (SI units; B in units where the magnetic
# pressure is B^2/2, i.e. tesla / sqrt(mu0), as dervfields.cu:119-120 use it).
R_GAS = 8.31e3           # J / (kg K), mu = 1 (initialisation_user.h.spicule1_mpi:378)
G_SUN = -274.0           # m / s^2 along the vertical (dim 0)
MU0 = 4.0e-7 * np.pi


def temperature_profile(z, t_ch=6.0e3, t_co=1.0e6, z_tr=2.0e6, w_tr=0.2e6):
    """T(z) = T_ch + (T_co - T_ch) (1 + tanh((z - z_tr) / w_tr)) / 2, evaluated
    in the form and operation order of the reference's temp()
    (models/initialisation_user.h.spicule1_mpi:345-360):
    0.5 T_co (1 + r + (1 - r) tanh((z - z_tr) / w_tr)) with r = T_ch / T_co,
    and the C library's tanh (math.tanh), so that it gives the reference's bits."""
    r = t_ch / t_co
    return np.array([0.5 * t_co * (1 + r + (1.0 - r) * math.tanh((float(zi) - z_tr) / w_tr)) for zi in np.ravel(z)])


def trapezoid_up(f, i0, dx):
    """Running trapezoid integral of f from index i0 upwards on a uniform grid:
    out[i0] = 0, out[i] = out[i-1] + 0.5 (f[i-1] + f[i]) dx -- the sum and its
    operation order of the reference's inte() (models/initialisation_user.h.
    spicule1_mpi:326-343), whose inte(f, i + 1 - i0, 1, ., dx) over f[i0:] is out[i]."""
    out = np.zeros(len(f))
    for i in range(i0 + 1, len(f)):
        out[i] = out[i - 1] + 0.5 * (f[i - 1] + f[i]) * dx
    return out


def hydrostatic_density(z, T, rho0, dz, g=G_SUN, R=R_GAS):
    """rho_b(z) of an ideal gas (p = rho R T) in hydrostatic equilibrium,
    dp/dz = rho g, with rho = rho0 at z = 0: p = p0 exp(-int_0^z dz'/lambda),
    lambda = -R T / g (the reference's scale height, lambda[i] = -R T[i] / ggg,
    models/initialisation_user.h.spicule1_mpi:403-404), the integral by the
    reference's trapezoid rule (trapezoid_up) on the grid points z of spacing
    dz (FP64) from the grid point at z = 0 upwards, and mirrored below it
    (the ghost layers under the surface)."""
    inv = 1.0 / (-R * T / g)
    i0 = int(np.argmin(np.abs(z)))
    if z[i0] != 0.0:
        raise ValueError("the grid needs a point at z = 0")
    integ = trapezoid_up(inv, i0, dz)
    for i in range(i0 - 1, -1, -1):
        integ[i] = integ[i + 1] - 0.5 * (inv[i + 1] + inv[i]) * dz
    p0 = rho0 * R * T[i0]
    p = p0 * np.exp(-integ)
    return p / (R * T), p


def atmosphere(nz: int = 256, nx: int = 128, ny: int | None = None, lz: float = 6.0e6, lx: float = 4.0e6,
               ly: float = 4.0e6, rho0: float = 2.7e-4, b_gauss: float = 10.0, gamma: float = 5.0 / 3.0,
               driver: dict | None = "default", noise: float = 0.0, seed: int | None = None) -> Problem:
    """Stratified solar atmosphere, vertical = dim 0 (z from 0 at the first
    inner cell), 2-D (z, x) when ny is None, else 3-D (z, x, y).  Split
    background: T(z) tanh profile, rho_b hydrostatic, p_b = rho_b R T, uniform
    vertical B_b, e_b = p_b / (gamma - 1) + B_b^2 / 2; perturbations zero (or
    seeded density noise of relative size `noise`).  Vertical boundaries
    contcd4, lateral periodic, gravity along -z.  driver "default": vertical
    velocity driver at the lower boundary, 300 s period, 200 m/s, 0.5 Mm
    horizontal width."""
    D = 2 if ny is None else 3
    cells = (nz, nx) if D == 2 else (nz, nx, ny)
    L = (lz, lx) if D == 2 else (lz, lx, ly)
    n = tuple(c + 2 * NG for c in cells)
    dx = tuple(L[d] / cells[d] for d in range(D))
    xmin = tuple(-NG * dx[d] for d in range(D))
    z = xmin[0] + np.arange(n[0]) * dx[0]
    T = temperature_profile(z)
    rhob, pb = hydrostatic_density(z, T, rho0, dx[0])
    bz = b_gauss * 1.0e-4 / np.sqrt(MU0)
    ids = field_ids(D)
    shape = tuple(reversed(n))  # arrays are indexed [.., dim1, dim0]
    w = np.zeros((nvar(D),) + shape)
    prof = lambda a: np.broadcast_to(a, shape)  # noqa: E731  (dim 0 is the last axis)
    w[ids["rhob"]] = prof(rhob)
    w[ids["b1b"]] = bz
    w[ids["eb"]] = prof(pb / (gamma - 1.0) + 0.5 * bz * bz)
    if noise:
        rng = np.random.default_rng(seed)
        w[ids["rho"]] = noise * prof(rhob) * rng.standard_normal(shape)
    drv = None
    if driver == "default":
        drv = {"dir": 0, "amp": 200.0, "period": 300.0,
               "center": (2.0 * dx[0],) + tuple(L[d] / 2 for d in range(1, D)),
               "width": (2.0 * dx[0],) + (0.5e6,) * (D - 1)}
    elif driver:
        drv = dict(driver)
    prob = Problem("atmosphere", D, n, dx, xmin, gamma, _chyp(D), (4,) + (0,) * (D - 1), 0.3, w,
                   g=(G_SUN, 0.0, 0.0), meta={"nz": nz, "nx": nx, "ny": ny, "noise": noise, "seed": seed},
                   driver=drv)
    if noise:
        prob.w = _boundary_fill(prob)
    return prob


def _boundary_fill(prob: Problem) -> np.ndarray:
    """Ghost fill of the evolved fields: periodic or contcd4 per dim (the
    state handed to the library gets this fill again on load)."""
    w = prob.w.copy()
    nw = 2 + 2 * prob.ndim
    for d in range(prob.ndim):
        ax = w.ndim - 1 - d
        m = w.shape[ax]
        idx = np.arange(m)
        if prob.btype[d] == 0:
            src = np.where(idx < NG, idx + m - 2 * NG, np.where(idx >= m - NG, idx - (m - 2 * NG), idx))
        else:  # contcd4: 0 <- 4, 1 <- 3, n-1 <- n-5, n-2 <- n-4
            src = idx.copy()
            src[0], src[1], src[m - 1], src[m - 2] = 4, 3, m - 5, m - 4
        w[:nw] = np.take(w[:nw], src, axis=ax)
    return w


def driver_slab(n: int = 24) -> Problem:
    """2-D (z, x) uniform slab in metres around the driver of the reference's
    spicule model (models/usersource.cu.spicule1: centre z = 0.0174 Mm,
    x = 1.998046 Mm, widths 1 km, 200 m/s, constant in time), 250 m cells, so
    that its Gaussian spans several cells.  rho = 1e-3, p = 1e3, B = (1e-2, 0)."""
    D = 2
    N = (n + 2 * NG,) * 2
    dx = (250.0, 250.0)
    c = (0.0174e6, 1.998046e6)
    xmin = tuple(c[d] - (N[d] // 2) * dx[d] + 0.3 * dx[d] for d in range(D))
    gam = 5.0 / 3.0
    ids = field_ids(D)
    w = np.zeros((nvar(D),) + tuple(reversed(N)))
    w[ids["rho"]] = 1.0e-3
    w[ids["b1"]] = 1.0e-2
    w[ids["e"]] = 1.0e3 / (gam - 1.0) + 0.5 * 1.0e-4
    drv = {"dir": 0, "amp": 200.0, "period": 0.0, "center": c, "width": (1.0e3, 1.0e3)}
    return Problem("driver_slab", D, N, dx, xmin, gam, _chyp(D), (0, 0), 0.3, w, driver=drv)


ENSEMBLE_SIDES = (128, 192, 256, 384, 512, 768)


def ensemble(count: int = 96, seed: int = 4242, sides=ENSEMBLE_SIDES) -> list:
    """Batched ensemble of independent 2-D Orszag-Tang vortices: side drawn
    uniformly from `sides`, B0 scaled by U[0.5, 1.5], 1 % Gaussian density
    noise per cell (noise seed = seed + instance id)."""
    rng = np.random.default_rng(seed)
    n = rng.choice(np.asarray(sides), size=count)
    b0 = rng.uniform(0.5, 1.5, size=count)
    return [orszag_tang(int(n[i]), b0_scale=float(b0[i]), rho_noise=0.01, seed=seed + i) for i in range(count)]


def _periodic_fill(a: np.ndarray) -> np.ndarray:
    out = a.copy()
    for ax in range(a.ndim):
        m = a.shape[ax]
        idx = np.arange(m)
        src = np.where(idx < NG, idx + m - 2 * NG, np.where(idx >= m - NG, idx - (m - 2 * NG), idx))
        out = np.take(out, src, axis=ax)
    return out


def blast_wave(n: int = 128, seed: int = 1234) -> Problem:
    """3-D blast wave on [-0.5, 0.5]^3, periodic: rho=1, p=0.1,
    B=(1/sqrt2, 1/sqrt2, 0), p=10 inside r<0.1 about a centre jittered by
    U(-dx/2, dx/2)^3 (PCG64 seeded)."""
    N = (n + 2 * NG,) * 3
    d = 1.0 / n
    rng = np.random.default_rng(seed)
    c0 = rng.uniform(-d / 2, d / 2, size=3)
    ax = -0.5 + (np.arange(N[0]) - NG + 0.5) * d
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")  # arrays indexed [k, j, i]
    r = np.sqrt((X - c0[0]) ** 2 + (Y - c0[1]) ** 2 + (Z - c0[2]) ** 2)
    gam = 5.0 / 3.0
    p = np.where(r < 0.1, 10.0, 0.1)
    bx = by = 1.0 / np.sqrt(2.0)
    w = np.zeros((nvar(3),) + X.shape)
    w[0] = 1.0
    w[4] = p / (gam - 1) + 0.5 * (bx * bx + by * by)
    w[5] = bx
    w[6] = by
    w = np.stack([_periodic_fill(f) for f in w])
    return Problem("blast_wave", 3, N, (d, d, d), (-0.5 - (NG - 0.5) * d,) * 3, gam, _chyp(3),
                   (0, 0, 0), 0.3, w, meta={"n": n, "seed": seed, "centre": c0.tolist()})
