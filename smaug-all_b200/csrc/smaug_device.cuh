// smaug_device.cuh -- device side of the fused ideal-MHD stage (sm_100a).
//
// One thread advances one interior cell through one Runge-Kutta stage:
//   out = base + h * L(in)
// where L is the SMAUG/SAC single-step operator (fluxes + divergence, the
// background energy terms, gravity, hyperdiffusive viscosity/resistivity).
// The reference runs L as ~300 separate kernels that round-trip every
// intermediate through HBM (dev/smaug/src/iosmaug.cpp:904-1166); here the
// whole operator is evaluated in registers from the state of the cell's
// neighbourhood and written once, together with the ghost copies of the
// cell (the on-device replacement for cuboundary / the MPI halo exchange).
//
// Each increment is applied in the order the reference applies it to its
// output slot, and with the same expression shapes; built without FMA
// contraction this reproduces the oracle (and so the reference) bit for bit.
//
// Field ids follow iotypes.h:213-219; evolved fields live in the state
// buffers, the static background fields (eb, rhob, bb...) in `bg`.
#pragma once
#include <cstdint>
#include <cstring>

namespace smaug {

constexpr int kMaxD = 3;

struct Reduce {  // maxima over all cells of one state (as uint64 bit patterns of non-negative doubles)
  unsigned long long v[8];  // [0..2] cmax per dim, [3] maxcourant, [4] courant over idx >= K, [5] max nu
};

struct DevScalars {
  double dt;
  double dtdiffvisc;
  double maxviscoef;  // running maximum over all steps
  double maxcourant;
  double minsq[3];    // min over the first K cells of delx_d^2 (viscous dt), set with the metric
  int step;
  int status;
  int go;         // batch only: this simulation takes the current step
  int bg_live;    // set on load: the state has a nonzero energy background (e_b, B_b)
  double t;       // simulation time at the start of the current step (driver)
  double hst[5];  // RK stage sizes of the current step: [1..4] = dt/2, dt/2, dt, dt/6 (set with dt)
  Reduce red[5];  // [0] state at step start, [1..3] RK stage outputs, [4] state at step end
  // maxima over the ghost cells that keep their loaded values (fixed
  // boundaries): the stage kernels never rewrite those cells, so each step's
  // stage maxima start from these
  Reduce floor;
};

struct Geo {
  int n[3];
  long long st[3];
  long long N;
  int btype[3];               // per dim: 0 periodic, 3 cont, 4 contcd4, 5 fixed, 6 symm, 7 asymm
  int bmask[3];               // per dim: evolved fields (bit f) that take asymm where btype is symm
  int outer_frozen[3];        // 1: a later dim is fixed, so the outermost ghost layer keeps its loaded values
  int has_const;              // some ghost cells keep their loaded values (a fixed dim)
  long long K;                // courant cells below K are excluded from the viscous-dt maximum
  const double *dx1[3];       // metric along d at inner cells (depends on c_d only)
  const double *rdx1[3];      // its reciprocals 1 / dx1 (IEEE division, once per grid line)
  const double *dxlast;       // full per-cell metric of the last dim (courant reduction)
  const double *drvf[3];      // driver: Gaussian factor per cell index along each dim
};

struct Phys {
  double gamma;
  double courant;
  double chyp[13];
  double g[3];
  int hyperdif;
  int has_bgb;                // any background B or eb != 0 (energy background terms)
  int has_grav;
  int dt_mode;
  int divb;                   // 2-D divergence-of-B source terms (divbon, divbfix)
  double dxs[3];              // uniform spacing per dim (p->dx, the divB gradient)
  int drv_on, drv_dir;        // momentum driver: on, driven momentum component
  double drv_amp, drv_period; // amplitude, period (0: constant in time)
};

struct StageArgs {
  // FP64 path
  const double *in;    // NW evolved fields, stage input (read with halo)
  const double *bg;    // NB background fields (FP64 in both paths)
  const double *base;  // NW evolved fields, RK base (read at the cell)
  double *out;         // NW evolved fields, stage output
  double *acc;         // RK accumulator (stage 3 writes (w1+2w2+w3-4w)/3, stage 4 adds it)
  // mixed-precision path: FP32 stage states, the RK base as an FP32 value plus
  // an FP32 compensation (w32 + c32 carries ~48 bits), FP32 RK increment sum
  const float *in32;
  float *out32, *acc32, *w32, *c32;
  DevScalars *sc;
  int kind;            // FP64: 0 plain, 3 = RK stage 3, 4 = RK stage 4; mixed: RK stage 1..4
  int red_in, red_out; // reduction slots: cmax of `in`, maxima of `out`
  double hdiv;         // h = dt / hdiv (dt/2, dt/2, dt, dt/6 as the oracle divides)
  int hslot;           // > 0: h is sc->hst[hslot], the same division done once per step
  double tfrac;        // stage input time = t + tfrac * dt (0, 1/2, 1/2, 1; driver)
};

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *slot, double v) {
  // IEEE order of non-negative doubles equals the order of their bit patterns;
  // a NaN (positive quiet NaN) compares above +inf and so is always kept.
  atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

__host__ __device__ __forceinline__ double red_get(const Reduce &r, int i) {
  double x;
  memcpy(&x, &r.v[i], sizeof(double));
  return x;
}

template <int D>
struct Lay {
  static constexpr int RHO = 0, M0 = 1, EN = 1 + D, B0 = 2 + D, NW = 2 + 2 * D;
  static constexpr int EB = 2 + 2 * D, RHOB = 3 + 2 * D, BB0 = 4 + 2 * D, NVAR = 4 + 3 * D;
};

template <int D>
struct Cell {
  const double *__restrict__ in;
  const double *__restrict__ bg;
  long long N;
  __device__ __forceinline__ double v(int f, long long i) const {
    return f < Lay<D>::NW ? __ldg(in + (long long)f * N + i) : __ldg(bg + (long long)(f - Lay<D>::NW) * N + i);
  }
};

// ----------------------------------------------------------- derived fields

// computept3_MODID, dervfields.cu:107-153
template <int D>
__device__ __forceinline__ double pt_at(const Cell<D> &c, long long i, double gam) {
  using L = Lay<D>;
  double bb = 0, b2 = 0, m2 = 0;
#pragma unroll
  for (int k = 0; k < D; ++k) bb += c.v(L::B0 + k, i) * c.v(L::BB0 + k, i);
#pragma unroll
  for (int k = 0; k < D; ++k) b2 += c.v(L::B0 + k, i) * c.v(L::B0 + k, i);
#pragma unroll
  for (int k = 0; k < D; ++k) m2 += c.v(L::M0 + k, i) * c.v(L::M0 + k, i);
  double t = ((gam)-2.0) * ((bb) + 0.5 * (b2));
  return ((gam)-1.0) * (c.v(L::EN, i) - 0.5 * (m2) / (c.v(L::RHO, i) + c.v(L::RHOB, i))) - t;
}

// computec3_MODID, dervfields.cu:241-309, from explicit field values
template <int D>
__device__ __forceinline__ double cfast_vals(const double *w, const double *b, int dir, double gam) {
  // w: NW evolved values, b: NB background values (eb, rhob, bb0..)
  using L = Lay<D>;
  double m2 = 0, b2 = 0, bbb = 0, bb2 = 0;
#pragma unroll
  for (int k = 0; k < D; ++k) m2 += w[L::M0 + k] * w[L::M0 + k];
#pragma unroll
  for (int k = 0; k < D; ++k) b2 += w[L::B0 + k] * w[L::B0 + k];
#pragma unroll
  for (int k = 0; k < D; ++k) bbb += b[2 + k] * w[L::B0 + k];
#pragma unroll
  for (int k = 0; k < D; ++k) bb2 += b[2 + k] * b[2 + k];
  const double rt = w[L::RHO] + b[1];
  double pk = ((gam)-1) * (w[L::EN] - 0.5 * ((m2) / (rt)) - 0.5 * (b2) - (bbb));
  double cs2 = (((gam)) * (pk + (((gam)) - 1) * (b[0] - 0.5 * (bb2))) / (rt));
  double cf = ((b2) + (bb2) + 2.0 * (bbb)) / (rt) + (cs2);
  double bd = b[2 + dir] + w[L::B0 + dir];
  double cfasti = 0.5 * (cf + sqrt(cf * cf - 4.0 * cs2 * ((bd) * (bd)) / (rt)));
  return sqrt(cfasti) + fabs(w[L::M0 + dir] / (rt));
}

// Fluxes of all evolved fields along dir at cell i:
// computefluxrho/computefluxmom* (centdiff1.cu:51-256), computefluxe/fluxe1
// and computefluxb* (centdiff2.cu:189-340).
template <int D>
__device__ __forceinline__ void fluxes_at(const Cell<D> &c, long long i, int dir, double gam, double *F) {
  using L = Lay<D>;
  const double rho = c.v(L::RHO, i), rhob = c.v(L::RHOB, i);
  const double rt = rho + rhob;
  const double md = c.v(L::M0 + dir, i);
  const double pt = pt_at<D>(c, i, gam);
  F[L::RHO] = md * rho / (rho + rhob) + (rhob * md) / (rhob + rho);
  const double bd = c.v(L::B0 + dir, i), bbd = c.v(L::BB0 + dir, i);
#pragma unroll
  for (int k = 0; k < D; ++k) {
    const double bf = c.v(L::B0 + k, i), bbf = c.v(L::BB0 + k, i);
    double tr = md * c.v(L::M0 + k, i) / (rt);
    double mg = (k == dir) ? pt - (bf * bbd + bbf * bd) - bf * bd : -(bf * bbd + bbf * bd) - bf * bd;
    F[L::M0 + k] = tr + mg;
  }
  double bbm = 0, bm = 0;
#pragma unroll
  for (int k = 0; k < D; ++k) bbm += c.v(L::BB0 + k, i) * c.v(L::M0 + k, i);
#pragma unroll
  for (int k = 0; k < D; ++k) bm += c.v(L::B0 + k, i) * c.v(L::M0 + k, i);
  {
    double tr = md * c.v(L::EN, i) / (rt);
    double fl = md * (pt);
    fl -= bd * (bbm);
    fl -= bbd * (bm);
    fl /= (rt);
    fl += md * c.v(L::EB, i) / (rt);
    fl -= bd * (bm) / (rt);
    F[L::EN] = tr + fl;
  }
#pragma unroll
  for (int k = 0; k < D; ++k) {
    if (k == dir) {
      F[L::B0 + k] = 0.0;
    } else {
      F[L::B0 + k] = md * c.v(L::B0 + k, i) / (rt) - (bd + bbd) * c.v(L::M0 + k, i) / (rt) +
                     (c.v(L::BB0 + k, i)) * md / (rt);
    }
  }
}

// 4th-order central difference (grad3dn_MODID, gradops.cu:437-606) of values
// at offsets -2,-1,+1,+2; zero within two cells of a non-periodic edge.
__device__ __forceinline__ double d4(double am2, double am1, double ap1, double ap2, double dx, bool zero) {
  double g = (((8 * ap1 - 8 * am1 + am2 - ap2) / 6.0)) / (2.0 * (dx));
  return zero ? 0.0 : g;
}

// --------------------------------------------------------- hyperviscosity

// q of the hyperviscosity chain for one field at cell i (hyperdifvisc1r.cu:1222-1262)
enum { Q_RHO = 0, Q_EN = 1, Q_VEL = 2, Q_B = 3 };

template <int D, int QK>
__device__ __forceinline__ double q_at(const Cell<D> &c, long long i, int f) {
  using L = Lay<D>;
  if (QK == Q_RHO) return c.v(L::RHO, i);
  if (QK == Q_B) return c.v(L::B0 + f, i);
  if (QK == Q_VEL) return c.v(L::M0 + f, i) / (c.v(L::RHO, i) + c.v(L::RHOB, i));
  double b2 = 0, m2 = 0;
#pragma unroll
  for (int k = 0; k < D; ++k) b2 += c.v(L::B0 + k, i) * c.v(L::B0 + k, i);
#pragma unroll
  for (int k = 0; k < D; ++k) m2 += c.v(L::M0 + k, i) * c.v(L::M0 + k, i);
  return c.v(L::EN, i) - 0.5 * ((b2) + (m2) / (c.v(L::RHO, i) + c.v(L::RHOB, i)));
}

// Right and left hyperviscosity of q along d at an inner cell
// (hyperdifvisc2r/3r/4r, hyperdifvisc1r.cu:426-845; 2l/3l/4l,
// hyperdifvisc1l.cu:436-855).  The padded copy of q has right pad 0 and left
// pad q(5) (bc_hyperdifl, hyperdifvisc1l.cu:17-66).
template <int D, int QK>
__device__ __forceinline__ void visc_at(const Cell<D> &c, const Geo &g, long long i, int cd, int d, int f,
                                        double cmax, double chyp, double dx, double &nur, double &nul) {
  double q[7];
  const long long s = g.st[d];
#pragma unroll
  for (int o = -3; o <= 3; ++o) {
    const int x = cd + o;
    if (x >= g.n[d])
      q[o + 3] = 0.0;
    else if (x < 0)
      q[o + 3] = q_at<D, QK>(c, i + (long long)(5 - cd) * s, f);
    else
      q[o + 3] = q_at<D, QK>(c, i + (long long)o * s, f);
  }
#define QQ(o) q[(o) + 3]
  double maxt1 = 0, maxt2 = 0;
#pragma unroll
  for (int t = -1; t <= 1; ++t) {
    double v = fabs(3.0 * (QQ(t + 1) - QQ(t)) - (QQ(t + 2) - QQ(t - 1)));
    if (v > maxt1) maxt1 = v;
  }
#pragma unroll
  for (int t = -2; t <= 2; ++t) {
    double v = fabs((QQ(t + 1) - QQ(t)));
    if (v > maxt2) maxt2 = v;
  }
  nur = (maxt2 > 0) ? ((dx)) * (cmax) * (chyp)*maxt1 / maxt2 : 0.0;
  maxt1 = 0;
  maxt2 = 0;
#pragma unroll
  for (int t = -1; t <= 1; ++t) {
    double v = fabs(3.0 * (QQ(t) - QQ(t - 1)) - (QQ(t + 1) - QQ(t - 2)));
    if (v > maxt1) maxt1 = v;
  }
#pragma unroll
  for (int t = -2; t <= 2; ++t) {
    double v = fabs(QQ(t) - (QQ(t - 1)));
    if (v > maxt2) maxt2 = v;
  }
  nul = (maxt2 > 0) ? ((dx)) * (cmax) * (chyp)*maxt1 / maxt2 : 0.0;
#undef QQ
}

// Driver velocity at inner cell c for the stage whose input is at time
// t + tfrac * dt: A * F(c) * tdep, F = f1 * f0 (2-D) or (f1 * f0) * f2 (3-D)
// from the host-computed factor lines, tdep = sin(2 pi t / P) or 1 (P = 0).
// The driven momentum then gains h * vvz * (rho + rhob) of the stage output
// (models/usersource.cu.spicule1:4-137, addsourceterms2).
template <int D>
__device__ __forceinline__ double driver_vvz(const Geo &g, const Phys &p, const DevScalars *sc, double tfrac,
                                             const int *c) {
  double f = g.drvf[1][c[1]] * g.drvf[0][c[0]];
  if (D == 3) f = f * g.drvf[2][c[2]];
  double tdep = 1.0;
  if (p.drv_period > 0.0) tdep = sin(2.0 * 3.14159265358979323846 * (sc->t + tfrac * sc->dt) / p.drv_period);
  return p.drv_amp * f * tdep;
}

// ------------------------------------------------------------- boundaries
// The reference fills the ghosts field by field and, per field, direction by
// direction (iosmaug.cpp:1157-1166).  The rule of one direction takes ghost
// coordinate x of n cells from the source coordinate below, along the same
// direction, so corners compose the rules in direction order:
//   0 periodic  x +- (n-4)              (models/boundary.cu.sedov3d)
//   3 cont      0,1 <- 2;  n-2,n-1 <- n-3   (bc3_cont_dir, gradops.cu:1043-1050)
//   4 contcd4   0 <- 4, 1 <- 3, n-1 <- n-5, n-2 <- n-4   (boundary.cu.sedov3d)
//   5 fixed     the loaded values (bc3_setfixed_dir / bc3_fixed_dir,
//               gradops.cu:1201-1269); its tests read `i==0 || i==1 && dir==0`,
//               so the pass also restores the outermost layer (0, n-1) of
//               every earlier direction
//   6 symm      2-D 0 <- 3, 1 <- 2, n-1 <- n-4, n-2 <- n-3; 3-D as contcd4
//               (bc3_symm_dir, gradops.cu:1324-1395)
//   7 asymm     the symm source negated (bc3_asymm_dir); on a symm direction
//               the fields of bmask take this rule
enum { BC_PERIODIC = 0, BC_CONT = 3, BC_CONTCD4 = 4, BC_FIXED = 5, BC_SYMM = 6, BC_ASYMM = 7 };

// Source coordinate of ghost coordinate x along a direction of n cells (-1:
// none, the fixed type).
__host__ __device__ inline int bc_source(int type, int D, int n, int x) {
  switch (type) {
    case BC_PERIODIC: return x < 2 ? x + (n - 4) : x - (n - 4);
    case BC_CONT: return x < 2 ? 2 : n - 3;
    case BC_CONTCD4: return x == 0 ? 4 : x == 1 ? 3 : x == n - 1 ? n - 5 : n - 4;
    case BC_SYMM:
    case BC_ASYMM:
      if (D == 2) return x == 0 ? 3 : x == 1 ? 2 : x == n - 1 ? n - 4 : n - 3;
      return x == 0 ? 4 : x == 1 ? 3 : x == n - 1 ? n - 5 : n - 4;
    default: return -1;
  }
}

// Evolved fields (bit f) negated by the rule along d.
__host__ __device__ inline unsigned bc_neg(const Geo &g, int d) {
  return g.btype[d] == BC_ASYMM ? 0xffu : g.btype[d] == BC_SYMM ? (unsigned)g.bmask[d] : 0u;
}

// Does cell c keep its loaded value under the fill passes?  Walks back from
// the last pass that writes the cell: a fixed pass restores it; another rule
// moves to its source along that direction and continues with the earlier
// passes; an inner cell evolves.
template <int D>
__host__ __device__ inline bool is_const_cell(const Geo &g, const int *c0) {
  int c[3] = {c0[0], c0[1], c0[2]};
  int limit = D - 1;
  while (limit >= 0) {
    int L = -1;
    for (int q = limit; q >= 0 && L < 0; --q) {
      bool covers = c[q] < 2 || c[q] > g.n[q] - 3;
      if (!covers && g.btype[q] == BC_FIXED)
        for (int e = 0; e < q; ++e)
          if (c[e] == 0 || c[e] == g.n[e] - 1) covers = true;
      if (covers) L = q;
    }
    if (L < 0) return false;
    if (g.btype[L] == BC_FIXED) return true;
    c[L] = bc_source(g.btype[L], D, g.n[L], c[L]);
    limit = L - 1;
  }
  return false;
}

}  // namespace smaug
