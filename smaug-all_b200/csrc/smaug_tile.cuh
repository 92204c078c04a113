// smaug_tile.cuh -- production stage kernel: shared-memory tiles, each
// per-cell quantity, flux and hyperviscosity computed once per tile.
//
// Same operator as smaug_stage.cuh (the term-by-term restatement used for
// bit-exact parity), reorganised for throughput:
//  * a block owns a TX x TY (x TZ) tile of inner cells, one thread per cell;
//  * fluxes of every field along `dir` are evaluated once on the tile widened
//    by 2 along dir and kept in shared memory for the 5-point divergence;
//  * for each dimension d the hyperviscosity inputs q (rho, internal energy,
//    velocities, B components) are evaluated once on the tile widened by 3
//    along d and 1 across, then nu_R / nu_L once per cell (and on the +-1
//    ring the off-diagonal terms need), all in shared memory;
//  * divisions become multiplications by per-cell reciprocals.
// Results match the reference operator to rounding (the FMA-free restatement
// in smaug_stage.cuh is the bit-exact one).
//
// The template parameter T is the type of the stage states and of the stencil
// arithmetic: double (the FP64 path) or float (the mixed path).  The mixed
// path keeps FP64 where accuracy needs it: the background fields, the total
// pressure p_T and the internal energy (both recovered by cancellation), the
// RK base state (an FP32 value plus an FP32 compensation), the RK combination
// itself and the dt reductions.  With T = double every expression below is
// the FP64 path's.
#pragma once
#include <type_traits>
#include "smaug_device.cuh"

namespace SMAUG_NS {
using namespace smaug;

// A tile of inner cells, one thread per cell (TZ = 1 in 2-D).
template <int X, int Y, int Z>
struct Tile {
  static constexpr int TX = X, TY = Y, TZ = Z, NT = X * Y * Z;
};
// the single-instance kernels' tiles
template <int D>
struct TileShape;
template <>
struct TileShape<2> : Tile<16, 16, 1> {};
template <>
struct TileShape<3> : Tile<8, 8, 4> {};

template <int D>
struct TileBox {
  // a box in grid coordinates: lo[d] .. lo[d]+ext[d]-1
  int lo[3], ext[3];
  __device__ __forceinline__ int size() const { return ext[0] * ext[1] * (D == 3 ? ext[2] : 1); }
  __device__ __forceinline__ void at(int r, int *c) const {
    c[0] = lo[0] + r % ext[0];
    r /= ext[0];
    c[1] = lo[1] + r % ext[1];
    c[2] = D == 3 ? lo[2] + r / ext[1] : 0;
  }
  __device__ __forceinline__ int index(const int *c) const {
    return (c[0] - lo[0]) + ext[0] * ((c[1] - lo[1]) + (D == 3 ? ext[1] * (c[2] - lo[2]) : 0));
  }
};

template <int D>
__device__ __forceinline__ long long gidx(const Geo &g, const int *c) {
  return c[0] + (long long)c[1] * g.st[1] + (D == 3 ? (long long)c[2] * g.st[2] : 0);
}

__device__ __forceinline__ double vmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double vabs(double a) { return fabs(a); }
__device__ __forceinline__ float vabs(float a) { return fabsf(a); }
// a * b + c with one rounding (never left to contraction)
__device__ __forceinline__ double vfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
// The hyperviscosity ratio a / b (b > 0): IEEE division in FP64; in FP32 the
// reciprocal-based quotient (within 2 ulp), the ratio being a limiter weight.
__device__ __forceinline__ double vratio(double a, double b) { return a / b; }
__device__ __forceinline__ float vratio(float a, float b) { return __fdividef(a, b); }

// Offset of field f at cell i in 32-bit arithmetic (the host rejects grids
// whose NVAR * N does not fit 31 bits): one multiply-add per access instead
// of a 64-bit product.
__device__ __forceinline__ unsigned fo32(int f, long long N, long long i) {
  return (unsigned)f * (unsigned)N + (unsigned)i;
}

// State accessor: evolved fields of type T, background fields FP64.
template <int D, typename T>
struct CellT {
  const T *__restrict__ in;
  const double *__restrict__ bg;
  long long N;
  // field f at cell i in the stencil type
  __device__ __forceinline__ T v(int f, long long i) const {
    return f < Lay<D>::NW ? __ldg(in + fo32(f, N, i)) : (T)__ldg(bg + fo32(f - Lay<D>::NW, N, i));
  }
  // field f at cell i in FP64
  __device__ __forceinline__ double vd(int f, long long i) const {
    return f < Lay<D>::NW ? (double)__ldg(in + fo32(f, N, i)) : __ldg(bg + fo32(f - Lay<D>::NW, N, i));
  }
};

template <int D>
__device__ __forceinline__ bool in_grid(const Geo &g, const int *c) {
#pragma unroll
  for (int d = 0; d < D; ++d)
    if (c[d] < 0 || c[d] >= g.n[d]) return false;
  return true;
}

// Fluxes along dir with reciprocal arithmetic (the same physical fluxes as
// fluxes_at): rho, momentum, energy, induction.  rho_t, its reciprocal and
// the total pressure are formed in FP64.  bgb = 0: e_b and B_b are zero
// everywhere (not read).
template <int D, typename T>
__device__ __forceinline__ void fluxes_fast(const CellT<D, T> &c, long long i, int dir, double gam, bool bgb, T *F) {
  using L = Lay<D>;
  const T rho = c.v(L::RHO, i);
  const double rt = (double)rho + c.vd(L::RHOB, i);
  const double irtd = __drcp_rn(rt);
  const T irt = (T)irtd;
  T m[D], b[D], bb[D];
#pragma unroll
  for (int k = 0; k < D; ++k) {
    m[k] = c.v(L::M0 + k, i);
    b[k] = c.v(L::B0 + k, i);
    bb[k] = bgb ? c.v(L::BB0 + k, i) : T(0);
  }
  const T e = c.v(L::EN, i), eb = bgb ? c.v(L::EB, i) : T(0);
  double bbb = 0, b2 = 0, m2 = 0;
  T bbm = 0, bm = 0;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    bbb += (double)b[k] * (double)bb[k];
    b2 += (double)b[k] * (double)b[k];
    m2 += (double)m[k] * (double)m[k];
    bbm += bb[k] * m[k];
    bm += b[k] * m[k];
  }
  const T pt = (T)((gam - 1.0) * ((double)e - 0.5 * m2 * irtd) - (gam - 2.0) * (bbb + 0.5 * b2));
  const T md = m[dir], vd = md * irt;
  const T bd = b[dir], bbd = bb[dir];
  F[L::RHO] = md;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    T f = vd * m[k] - (b[k] * bbd + bb[k] * bd) - b[k] * bd;
    if (k == dir) f += pt;
    F[L::M0 + k] = f;
  }
  F[L::EN] = vd * (e + eb) + (md * pt - bd * bbm - bbd * bm - bd * bm) * irt;
#pragma unroll
  for (int k = 0; k < D; ++k)
    F[L::B0 + k] = (k == dir) ? T(0) : vd * (b[k] + bb[k]) - (bd + bbd) * m[k] * irt;
}

// q values for the hyperviscosity of all fields of one dimension d:
// slot 0 rho, 1 internal energy q_e (formed in FP64), 2..2+D-1 velocities,
// then B_f (f != d).
template <int D, typename T>
__device__ __forceinline__ void q_all(const CellT<D, T> &c, long long i, int d, T *q) {
  using L = Lay<D>;
  const T rho = c.v(L::RHO, i);
  const double irtd = __drcp_rn((double)rho + c.vd(L::RHOB, i));
  const T irt = (T)irtd;
  double b2 = 0, m2 = 0;
  q[0] = rho;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    const T m = c.v(L::M0 + k, i), b = c.v(L::B0 + k, i);
    b2 += (double)b * (double)b;
    m2 += (double)m * (double)m;
    q[2 + k] = m * irt;
  }
  q[1] = (T)(c.vd(L::EN, i) - 0.5 * (b2 + m2 * irtd));
  int s = 2 + D;
#pragma unroll
  for (int f = 0; f < D; ++f)
    if (f != d) q[s++] = c.v(L::B0 + f, i);
}

// cfast/courant maxima as reduce_cell (computec3, dervfields.cu:241-309), for
// the mixed path: the state is FP32 there, so the wave speeds are formed in
// FP32 from a correctly rounded reciprocal of rho_t (the pressure recovery's
// rounding stays at the level of the FP32 inputs); the courant number divides
// by the metric through a correctly rounded reciprocal too.  Explicitly
// rounded operations, never contracted: every build variant of the stage
// kernel gives the same bits.  b: eb, rho_b, B_b (zeros when the simulation
// has no energy background).  The maxima are FP32 values and kept in FP32.
//
// A fast pass comes first. It takes the square roots and the metric's
// reciprocal from the hardware approximations (x rsqrtf(x), __fdividef); every
// other operation is the same as in the exact pass. That puts each approximate
// speed within about 8 ulp (1e-6 relative) of its correctly rounded value: the
// terms under the roots are identical, and the sums after them add
// non-negative terms. If every approximate speed of the cell stays more than
// 1e-5 below the thread's running maximum, the cell cannot raise it and is
// done. Any other cell, a NaN included, takes the correctly rounded pass. The
// maxima come out the same bits either way.
__device__ __forceinline__ float sqrt_approx(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }

template <int D>
__device__ __forceinline__ void reduce_cell_mixed(const Geo &g, const Phys &p, const float *o, const double *b,
                                                  long long idx, float *r) {
  using L = Lay<D>;
  const float irt = __frcp_rn((float)((double)o[L::RHO] + b[1]));
  float m2 = 0.0f, b2 = 0.0f, bbb = 0.0f, bb2 = 0.0f;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    const float m = o[L::M0 + k], bf = o[L::B0 + k], bb = (float)b[2 + k];
    m2 = __fmaf_rn(m, m, m2);
    b2 = __fmaf_rn(bf, bf, b2);
    bbb = __fmaf_rn(bb, bf, bbb);
    bb2 = __fmaf_rn(bb, bb, bb2);
  }
  const float gm1 = (float)(p.gamma - 1.0), gam = (float)p.gamma;
  // p_k = (gamma-1) (e - m^2/(2 rho_t) - B^2/2 - B.B_b)
  const float ek = __fsub_rn(__fsub_rn(__fsub_rn(o[L::EN], __fmul_rn(__fmul_rn(0.5f, m2), irt)),
                                       __fmul_rn(0.5f, b2)), bbb);
  const float pk = __fmul_rn(gm1, ek);
  // c_s^2 = gamma (p_k + (gamma-1)(e_b - B_b^2/2)) / rho_t
  const float pbg = __fmul_rn(gm1, __fsub_rn((float)b[0], __fmul_rn(0.5f, bb2)));
  const float cs2 = __fmul_rn(__fmul_rn(gam, __fadd_rn(pk, pbg)), irt);
  const float cf = __fadd_rn(__fmul_rn(__fadd_rn(__fadd_rn(b2, bb2), __fmul_rn(2.0f, bbb)), irt), cs2);
  {
    constexpr float kBelow = 1.0f - 1e-5f;
    const float rdx = __fdividef(1.0f, (float)__ldg(g.dxlast + idx));
    bool need = false;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const float bd = (float)(b[2 + d] + (double)o[L::B0 + d]);
      const float disc =
          __fsub_rn(__fmul_rn(cf, cf), __fmul_rn(__fmul_rn(__fmul_rn(4.0f, cs2), __fmul_rn(bd, bd)), irt));
      const float cfi = __fmul_rn(0.5f, __fadd_rn(cf, sqrt_approx(fmaxf(disc, 0.0f))));
      const float cff = __fadd_rn(sqrt_approx(cfi), fabsf(__fmul_rn(o[L::M0 + d], irt)));
      need |= !(cff < r[d] * kBelow);
      if (d == D - 1) {
        const float cour = cff * rdx;
        need |= !(cour < r[3] * kBelow);
        if (idx >= g.K) need |= !(cour < r[4] * kBelow);
      }
    }
    if (!need) return;
  }
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float bd = (float)(b[2 + d] + (double)o[L::B0 + d]);
    const float disc = __fsub_rn(__fmul_rn(cf, cf), __fmul_rn(__fmul_rn(__fmul_rn(4.0f, cs2), __fmul_rn(bd, bd)), irt));
    const float cfi = __fmul_rn(0.5f, __fadd_rn(cf, __fsqrt_rn(fmaxf(disc, 0.0f))));
    const float cff = __fadd_rn(__fsqrt_rn(cfi), fabsf(__fmul_rn(o[L::M0 + d], irt)));
    if (cff > r[d] || cff != cff) r[d] = cff;
    if (d == D - 1) {
      const float cour = __fmul_rn(cff, __frcp_rn((float)__ldg(g.dxlast + idx)));
      if (cour > r[3] || cour != cour) r[3] = cour;
      if (idx >= g.K && (cour > r[4] || cour != cour)) r[4] = cour;
    }
  }
}

// The end of a stage for one cell: the stage output base + h dL with the
// driver, the RK combination of the stage, the write of the cell and the
// wave-speed / viscosity maxima, taken into the
// thread's running maxima red[6] (in the stencil type: FP32 values in the
// mixed path; the caller flushes them to the simulation's reduction slot).
template <int D, typename T>
__device__ __forceinline__ void stage_epilogue(const StageArgs &a, const Geo &g, const Phys &p, const CellT<D, T> &C,
                                               const int *c, bool active, long long idx, double h, const T *dL,
                                               T numax, T *red) {
  using L = Lay<D>;
  constexpr int NW = L::NW, NB = L::NVAR - NW;
  constexpr bool MIXED = sizeof(T) == sizeof(float);
  if (numax > red[5] || numax != numax) red[5] = numax;
  if (active) {
    double o[NW];
    float hi[NW], lo[NW];
    if (!MIXED) {
#pragma unroll
      for (int f = 0; f < NW; ++f) o[f] = a.base[fo32(f, g.N, idx)] + h * (double)dL[f];
      if (p.drv_on) {  // momentum driver on the stage output (before the RK combination)
        const double vvz = driver_vvz<D>(g, p, a.sc, a.tfrac, c);
        const double rb = __ldg(a.bg + (long long)(L::RHOB - NW) * g.N + idx);
        // (unrolled compare: a runtime index would push o to local memory)
#pragma unroll
        for (int k = 0; k < D; ++k)
          if (k == p.drv_dir) o[L::M0 + k] = o[L::M0 + k] + h * vvz * (o[L::RHO] + rb);
      }
      if (a.kind == 3) {
#pragma unroll
        for (int f = 0; f < NW; ++f) {
          const unsigned j = fo32(f, g.N, idx);
          a.acc[j] = (a.acc[j] + 2.0 * C.vd(f, idx) + o[f] - 4.0 * a.base[j]) * (1.0 / 3.0);
        }
      } else if (a.kind == 4) {
#pragma unroll
        for (int f = 0; f < NW; ++f) o[f] += a.acc[fo32(f, g.N, idx)];
      }
    } else {
      // RK4 in increment form, W = w32 + c32:
      //   stages k = 1..3: S_k = W + h_k L_k (FP32), A += c_k h_k L_k with
      //   c = 1/3, 2/3, 1/3, so A = (S1 + 2 S2 + S3 - 4 W) / 3 as the FP64 path;
      //   stage 4: W <- W + h_4 L_4 + A, kept as value + compensation.
      // Stages 1..3 round to FP32 anyway, so they take the base without c32.
      // momentum driver with the stage output's density, added to the
      // increment of m along drv_dir (dm = 0 without a driver)
      double dm = 0.0;
      int dm_f = -1;
      if (p.drv_on) {
        const double wr = a.kind == 4 ? (double)a.w32[idx] + (double)a.c32[idx] : (double)a.w32[idx];
        const double rb = __ldg(a.bg + (long long)(L::RHOB - NW) * g.N + idx);
        dm = h * driver_vvz<D>(g, p, a.sc, a.tfrac, c) * ((wr + h * (double)dL[L::RHO]) + rb);
        dm_f = L::M0 + p.drv_dir;
      }
#pragma unroll
      for (int f = 0; f < NW; ++f) {
        const unsigned j = fo32(f, g.N, idx);
        double inc = h * (double)dL[f];
        if (f == dm_f) inc += dm;
        if (a.kind == 4) {
          const double wn = ((double)a.w32[j] + (double)a.c32[j]) + (inc + (double)a.acc32[j]);
          hi[f] = (float)wn;
          lo[f] = (float)(wn - (double)hi[f]);
        } else {
          hi[f] = (float)((double)a.w32[j] + inc);
          const double prev = a.kind == 1 ? 0.0 : (double)a.acc32[j];
          a.acc32[j] = (float)(prev + (a.kind == 2 ? 2.0 : 1.0) * (1.0 / 3.0) * inc);
        }
      }
    }
    // the cell (its ghost images are written by the ghost pass that follows
    // every stage: ghost_cell below)
    {
      const unsigned j = (unsigned)idx;
      if (!MIXED) {
#pragma unroll
        for (int f = 0; f < NW; ++f) a.out[fo32(f, g.N, j)] = o[f];
      } else if (a.kind == 4) {
#pragma unroll
        for (int f = 0; f < NW; ++f) {
          a.w32[fo32(f, g.N, j)] = hi[f];
          a.c32[fo32(f, g.N, j)] = lo[f];
        }
      } else {
#pragma unroll
        for (int f = 0; f < NW; ++f) a.out32[fo32(f, g.N, j)] = hi[f];
      }
    }
    // backgrounds (e_b and B_b are zero everywhere without an energy
    // background: only rho_b is read then), then the maxima
    double bgv[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b)
      bgv[b] = (b == L::RHOB - NW || p.has_bgb) ? __ldg(a.bg + fo32(b, g.N, (unsigned)idx)) : 0.0;
    if constexpr (MIXED)
      reduce_cell_mixed<D>(g, p, hi, bgv, idx, red);  // what the next stage reads
    else
      reduce_cell<D>(g, p, o, bgv, idx, red);
  }
}

// Divergence-of-B source terms at an inner cell (cudivb, divb.cu:165-336 with
// divbon = divbfix = 1; 2-D): at cells 3..n-3 of both dims, divB from the
// 4th-order difference over the uniform spacing (zero at the first and last
// two inner cells, as grad3d of gradops.cu:132-237), then -divB (0, B, B.v,
// v) per unit time with B.v = B_total . m / rho_t; NaN momentum and field
// sources count as 0 (dbsourcemom, dbsourceb).
template <typename T>
__device__ __forceinline__ void divb_sources(const CellT<2, T> &C, const Geo &g, const Phys &p, const int *c,
                                             long long idx, T *dL) {
  using L = Lay<2>;
  if (c[0] <= 2 || c[1] <= 2) return;
  T divb = 0;
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    const int x = c[d], n = g.n[d];
    if (x == 3 || x == n - 4 || x == n - 3) continue;
    const long long s = g.st[d];
    T b[4];  // B_d + B_bd at -2, -1, +1, +2
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const long long j = idx + (k < 2 ? k - 2 : k - 1) * s;
      b[k] = C.v(L::B0 + d, j) + (p.has_bgb ? C.v(L::BB0 + d, j) : T(0));
    }
    divb += ((T)8 * (b[2] - b[1]) - (b[3] - b[0])) * (T)(1.0 / (12.0 * p.dxs[d]));
  }
  const T irt = (T)(1.0 / (C.vd(L::RHO, idx) + C.vd(L::RHOB, idx)));
  T bdotv = 0;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const T bk = C.v(L::B0 + k, idx), mk = C.v(L::M0 + k, idx);
    bdotv += (bk + (p.has_bgb ? C.v(L::BB0 + k, idx) : T(0))) * mk;
    T sm = divb * bk, sb = divb * mk * irt;
    if (sm != sm) sm = 0;
    if (sb != sb) sb = 0;
    dL[L::M0 + k] += sm;
    dL[L::B0 + k] += sb;
  }
  dL[L::EN] += divb * bdotv * irt;
}

// ------------------------------------------------------------ the ghost pass
// After every stage the ghost cells of the stage output are filled from the
// inner cells just written (the reference's boundary pass after each step,
// iosmaug.cpp:1157-1166), and their wave speeds join the stage's maxima (the
// reference's c_max covers the ghosts).  Each ghost cell gathers its value:
// from the last direction whose pass writes it, back along the chain of
// sources (smaug_device.cuh) to an inner cell, negating the fields of the
// asymm rules on the way; a chain that meets a fixed pass ends at a cell that
// keeps its loaded value, so the ghost is left alone.

// Ghost cells of a grid: the cells with a coordinate outside [2, n-3].
template <int D>
__host__ __device__ inline long long ghost_count(const Geo &g) {
  long long in = 1;
  for (int d = 0; d < D; ++d) in *= g.n[d] - 4;
  return g.N - in;
}

// Coordinates of ghost k: first the four ghost rows (2-D) or planes (3-D) of
// the last dim, then, for each inner coordinate of the last dim, the ring of
// the lower dims.
template <int D>
__device__ __forceinline__ void ghost_coords(const Geo &g, long long k, int *c) {
  const int n0 = g.n[0], n1 = g.n[1];
  if (D == 2) {
    if (k < 4LL * n0) {
      const int r = (int)(k / n0);
      c[0] = (int)(k - (long long)r * n0);
      c[1] = r < 2 ? r : n1 - 4 + r;
    } else {
      const long long q = k - 4LL * n0;
      const int r = (int)(q & 3);
      c[1] = 2 + (int)(q >> 2);
      c[0] = r < 2 ? r : n0 - 4 + r;
    }
    c[2] = 0;
  } else {
    const long long pl = (long long)n0 * n1;
    const int n2 = g.n[2];
    if (k < 4 * pl) {
      const int r = (int)(k / pl);
      const long long q = k - r * pl;
      c[2] = r < 2 ? r : n2 - 4 + r;
      c[1] = (int)(q / n0);
      c[0] = (int)(q - (long long)c[1] * n0);
    } else {
      const long long ring = pl - (long long)(n0 - 4) * (n1 - 4);
      const long long q0 = k - 4 * pl;
      const long long z = q0 / ring;
      const long long q = q0 - z * ring;
      c[2] = 2 + (int)z;
      if (q < 4LL * n0) {
        const int r = (int)(q / n0);
        c[0] = (int)(q - (long long)r * n0);
        c[1] = r < 2 ? r : n1 - 4 + r;
      } else {
        const long long u = q - 4LL * n0;
        const int r = (int)(u & 3);
        c[1] = 2 + (int)(u >> 2);
        c[0] = r < 2 ? r : n0 - 4 + r;
      }
    }
  }
}

// Fill ghost k of the stage output and take its wave speeds into red.
template <int D, typename T>
__device__ __forceinline__ void ghost_cell(const StageArgs &a, const Geo &g, const Phys &p, long long k, T *red) {
  using L = Lay<D>;
  constexpr int NW = L::NW, NB = L::NVAR - NW;
  constexpr bool MIXED = sizeof(T) == sizeof(float);
  if (k >= ghost_count<D>(g)) return;
  int c[3], s[3];
  ghost_coords<D>(g, k, c);
  s[0] = c[0];
  s[1] = c[1];
  s[2] = c[2];
  unsigned neg = 0;
  for (int limit = D - 1; limit >= 0;) {
    int q = limit, L0 = -1;
    for (; q >= 0; --q) {
      bool covers = s[q] < 2 || s[q] > g.n[q] - 3;
      if (!covers && g.btype[q] == BC_FIXED)
        for (int e = 0; e < q; ++e)
          if (s[e] == 0 || s[e] == g.n[e] - 1) covers = true;
      if (covers) {
        L0 = q;
        break;
      }
    }
    if (L0 < 0) break;                      // an inner cell: the source
    if (g.btype[L0] == BC_FIXED) return;    // keeps its loaded value
    neg ^= bc_neg(g, L0);
    s[L0] = bc_source(g.btype[L0], D, g.n[L0], s[L0]);
    limit = L0 - 1;
  }
  const long long j = gidx<D>(g, c), src = gidx<D>(g, s);
  T ov[NW];
  if (!MIXED) {
#pragma unroll
    for (int f = 0; f < NW; ++f) {
      double v = a.out[fo32(f, g.N, src)];
      if ((neg >> f) & 1u) v = -v;
      a.out[fo32(f, g.N, j)] = v;
      ov[f] = v;
    }
  } else if (a.kind == 4) {
#pragma unroll
    for (int f = 0; f < NW; ++f) {
      float v = a.w32[fo32(f, g.N, src)], w = a.c32[fo32(f, g.N, src)];
      if ((neg >> f) & 1u) {
        v = -v;
        w = -w;
      }
      a.w32[fo32(f, g.N, j)] = v;
      a.c32[fo32(f, g.N, j)] = w;
      ov[f] = v;
    }
  } else {
#pragma unroll
    for (int f = 0; f < NW; ++f) {
      float v = a.out32[fo32(f, g.N, src)];
      if ((neg >> f) & 1u) v = -v;
      a.out32[fo32(f, g.N, j)] = v;
      ov[f] = v;
    }
  }
  double bgv[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b)
    bgv[b] = (b == L::RHOB - NW || p.has_bgb) ? __ldg(a.bg + fo32(b, g.N, j)) : 0.0;
  if constexpr (MIXED)
    reduce_cell_mixed<D>(g, p, ov, bgv, j, red);
  else
    reduce_cell<D>(g, p, ov, bgv, j, red);
}

// One RK stage on the tile (bx, by, bz) of one simulation; every thread of
// the block calls it (it synchronises the block).  sm: tile_smem_elems<D, S>()
// elements of T.
template <int D, typename T, typename S>
__device__ __forceinline__ void tile_body(const StageArgs &a, const Geo &g, const Phys &p, int bx, int by, int bz,
                                          T *sm, T *red) {
  using L = Lay<D>;
  constexpr int TX = S::TX, TY = S::TY, TZ = S::TZ, NT = TX * TY * TZ;
  constexpr int NW = L::NW, NB = L::NVAR - NW;
  constexpr int NQ = 2 * D + 1;  // q slots per cell for one dimension
  constexpr bool MIXED = sizeof(T) == sizeof(float);

  const int t = threadIdx.x;
  const int tc[3] = {t % TX, (t / TX) % TY, D == 3 ? t / (TX * TY) : 0};
  const int org[3] = {2 + bx * TX, 2 + by * TY, D == 3 ? 2 + bz * TZ : 0};
  int c[3] = {org[0] + tc[0], org[1] + tc[1], org[2] + tc[2]};
  bool active = true;
#pragma unroll
  for (int d = 0; d < D; ++d)
    if (c[d] > g.n[d] - 3) active = false;
  const long long idx = active ? gidx<D>(g, c) : 0;
  const CellT<D, T> C{MIXED ? (const T *)(const void *)a.in32 : (const T *)(const void *)a.in, a.bg, g.N};
  const double dt = a.sc->dt;
  const double h = a.hslot > 0 ? a.sc->hst[a.hslot] : dt / a.hdiv;
  T cm[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d) cm[d] = (T)red_get(a.sc->red[a.red_in], d);
  int tile_ext[3] = {TX, TY, D == 3 ? TZ : 1};
  T idx1[3] = {0, 0, 0};
  if (active) {
#pragma unroll
    for (int d = 0; d < D; ++d) idx1[d] = (T)__ldg(g.rdx1[d] + c[d]);
  }
  T dL[NW];
#pragma unroll
  for (int f = 0; f < NW; ++f) dL[f] = 0;
  T numax = 0;

  // ------------------------------------------------ flux divergences
#pragma unroll
  for (int dir = 0; dir < D; ++dir) {
    TileBox<D> box;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      box.lo[e] = org[e] - (e == dir ? 2 : 0);
      box.ext[e] = tile_ext[e] + (e == dir ? 4 : 0);
    }
    const int nbox = box.size();
    for (int r = t; r < nbox; r += NT) {
      int cc[3];
      box.at(r, cc);
      T F[NW];
      if (in_grid<D>(g, cc)) {
        fluxes_fast<D, T>(C, gidx<D>(g, cc), dir, p.gamma, p.has_bgb, F);
      } else {
#pragma unroll
        for (int f = 0; f < NW; ++f) F[f] = 0;
      }
#pragma unroll
      for (int f = 0; f < NW; ++f) sm[f * nbox + r] = F[f];
    }
    __syncthreads();
    if (active) {
      const bool zr = z4(g, c, dir);
      int cc[3] = {c[0], c[1], c[2]};
      const int r0 = box.index(cc);
      const int st = dir == 0 ? 1 : dir == 1 ? box.ext[0] : box.ext[0] * box.ext[1];
      const T w12 = idx1[dir] * (T)(1.0 / 12.0);
#pragma unroll
      for (int f = 0; f < NW; ++f) {
        const T *Fp = sm + f * nbox + r0;
        T gr = ((T)8 * (Fp[st] - Fp[-st]) - (Fp[2 * st] - Fp[-2 * st])) * w12;
        if (!zr) dL[f] -= gr;
      }
    }
    __syncthreads();
  }

  // ------------------------------------------------ gravity
  if (active && p.has_grav) {
    const T rho = C.v(L::RHO, idx), irt = (T)__drcp_rn((double)rho + C.vd(L::RHOB, idx));
#pragma unroll
    for (int k = 0; k < D; ++k) {
      dL[L::M0 + k] += (T)p.g[k] * rho;
      dL[L::EN] += rho * (T)p.g[k] * C.v(L::M0 + k, idx) * irt;
    }
  }
  if constexpr (D == 2) {
    if (active && p.divb) divb_sources<T>(C, g, p, c, idx, dL);
  }

  // ------------------------------------------------ per-dimension hyperdiffusion
  // (one call per dimension, d a compile-time constant in each)
  auto dim_pass = [&](auto dc) {
    constexpr int d = decltype(dc)::value;
    // q box: tile widened by 3 along d and 1 across
    TileBox<D> qb;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int w = e >= D ? 0 : (e == d ? 3 : 1);
      qb.lo[e] = org[e] - w;
      qb.ext[e] = tile_ext[e] + 2 * w;
    }
    const int nq = qb.size();
    // face box: the faces along d of the tile (face j between cells j and
    // j+1, j from -1), widened by 1 across d (the off-diagonal terms need nu
    // there); it holds the hyperviscosity ratio max|d3 q| / max|d1 q| per face
    constexpr int TD = d == 0 ? TX : d == 1 ? TY : TZ;
    TileBox<D> fb;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int w = (e >= D || e == d) ? 0 : 1;
      fb.lo[e] = org[e] - (e == d ? 1 : w);
      fb.ext[e] = e == d ? TD + 1 : tile_ext[e] + 2 * w;
    }
    const int nf = fb.size();
    T *Q = sm;            // [NQ][nq]
    T *V = sm + NQ * nq;  // [NQ][nf]
    for (int r = t; r < nq; r += NT) {
      int cc[3];
      qb.at(r, cc);
      T q[NQ];
      const int x = cc[d];
      bool ok = true;
#pragma unroll
      for (int e = 0; e < D; ++e)
        if (e != d && (cc[e] < 0 || cc[e] >= g.n[e])) ok = false;
      if (!ok || x >= g.n[d]) {  // x == n: right pad of the padded q copy (0)
#pragma unroll
        for (int k = 0; k < NQ; ++k) q[k] = 0;
      } else {
        int src[3] = {cc[0], cc[1], cc[2]};
        if (x < 0) src[d] = 5;  // left pad: q(-1) = q(5)
        q_all<D, T>(C, gidx<D>(g, src), d, q);
      }
#pragma unroll
      for (int k = 0; k < NQ; ++k) Q[k * nq + r] = q[k];
    }
    __syncthreads();
    const int sd = d == 0 ? 1 : d == 1 ? qb.ext[0] : qb.ext[0] * qb.ext[1];
    if (p.hyperdif) {
      // runs of SEG faces along d of one q slot on one line: the line's q
      // values are read once, each first and third difference is formed once
      // (explicit FMA), every face takes its windowed maxima; the last run of
      // a line is shifted back to end at the line's last face (shared faces
      // are written twice with the same value)
      constexpr int SEG = TD + 1 < 5 ? TD + 1 : 5;
      constexpr int NS = (TD + 1 + SEG - 1) / SEG;
      const int lines = nf / (TD + 1);
      const int fs = d == 0 ? 1 : d == 1 ? fb.ext[0] : fb.ext[0] * fb.ext[1];  // face stride along d
      for (int u = t; u < NQ * lines * NS; u += NT) {
        const int sg = u % NS, rest = u / NS;
        const int ln = rest % lines, k = rest / lines;
        const int f0 = min(-1 + sg * SEG, TD - SEG);  // first face of the run, tile-relative
        // the line's cross coordinates (tile-relative, -1 .. T_e): decode ln
        int cr[3] = {0, 0, 0}, rem = ln;
#pragma unroll
        for (int e = 0; e < 3; ++e) {
          if (e == d || e >= D) continue;
          const int ex = tile_ext[e] + 2;
          cr[e] = rem % ex - 1;
          rem /= ex;
        }
        // q at the cells f0-2 .. f0+SEG+2 along d
        int qc[3] = {org[0] + cr[0], org[1] + cr[1], org[2] + cr[2]};
        qc[d] = org[d] + f0 - 2;
        const T *qq = Q + k * nq + qb.index(qc);
        T qv[SEG + 5], t1[SEG + 4], t3[SEG + 3];
#pragma unroll
        for (int jx = 0; jx < SEG + 5; ++jx) qv[jx] = qq[jx * sd];
#pragma unroll
        for (int jx = 0; jx < SEG + 4; ++jx) t1[jx] = qv[jx + 1] - qv[jx];
#pragma unroll
        for (int jx = 1; jx <= SEG + 2; ++jx) t3[jx] = vabs(vfma((T)3, t1[jx], -(qv[jx + 2] - qv[jx - 1])));
        int fc[3] = {org[0] + cr[0], org[1] + cr[1], org[2] + cr[2]};
        fc[d] = org[d] + f0;
        T *dst = V + k * nf + fb.index(fc);
#pragma unroll
        for (int m = 0; m < SEG; ++m) {
          T m1 = 0, m3 = 0;
#pragma unroll
          for (int jx = m; jx <= m + 4; ++jx) m1 = vmax(m1, vabs(t1[jx]));
#pragma unroll
          for (int jx = m + 1; jx <= m + 3; ++jx) m3 = vmax(m3, t3[jx]);
          dst[m * fs] = m1 > 0 ? vratio(m3, m1) : T(0);
        }
      }
    }
    __syncthreads();
    if (active) {
      int cc[3] = {c[0], c[1], c[2]};
      const int r0 = qb.index(cc);
      const int fr = fb.index(cc);  // the cell's right face along d; its left face is fr - fs
      const int fs = d == 0 ? 1 : d == 1 ? fb.ext[0] : fb.ext[0] * fb.ext[1];
      const T dxd = (T)__ldg(g.dx1[d] + c[d]);
      // nu_R, nu_L of slot k at the cell shifted by `off` faces across d: dx
      // c_max c_hyp times the face ratios (0 off the inner cells, as the
      // reference's viscosity arrays are)
      auto nu_at = [&](int k, int off, bool in, T &nr, T &nl) {
        int fid = k == 0 ? L::RHO : k == 1 ? L::EN : k < 2 + D ? L::M0 + (k - 2) : 0;
        if (k >= 2 + D) {
          const int ff = k - (2 + D);
          fid = L::B0 + (ff >= d ? ff + 1 : ff);
        }
        const T kk = dxd * cm[d] * (T)p.chyp[fid];
        nr = in ? kk * V[k * nf + fr + off] : T(0);
        nl = in ? kk * V[k * nf + fr - fs + off] : T(0);
      };
      const long long sg = g.st[d];
      const bool zd = z1(g, c, d);
      const T i1 = idx1[d], i2 = idx1[d] * idx1[d];
      if (p.has_bgb) {  // background energy terms along d (addenergyterms_cd2)
        double bb2 = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) bb2 += C.vd(L::BB0 + k, idx) * C.vd(L::BB0 + k, idx);
        const T ptb = (T)((p.gamma - 1) * C.vd(L::EB, idx) - 0.5 * (p.gamma - 2) * bb2);
        const bool z4d = z4(g, c, d);
#pragma unroll
        for (int dir = 0; dir < D; ++dir) {
          const T *v = Q + (2 + dir) * nq + r0;
          T gv = z4d ? T(0) : ((T)8 * (v[sd] - v[-sd]) - (v[2 * sd] - v[-2 * sd])) * (i1 * (T)(1.0 / 12.0));
          if (d == dir) dL[L::EN] -= ptb * gv;
          dL[L::EN] += C.v(L::BB0 + d, idx) * C.v(L::BB0 + dir, idx) * gv;
        }
      }
      if (p.hyperdif) {
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
          T nr, nl;
          nu_at(k, 0, true, nr, nl);
          numax = vmax(numax, vmax(nr, nl));
        }
        // rho and internal energy: f += (nu_R dq+ - nu_L dq-) / dx^2
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const T *q = Q + k * nq + r0;
          T nr, nl;
          nu_at(k, 0, true, nr, nl);
          const T dp = zd ? T(0) : q[sd] - q[0], dm = zd ? T(0) : q[0] - q[-sd];
          dL[k == 0 ? L::RHO : L::EN] += (nr * dp - nl * dm) * i2;
        }
        // momentum
        const T rt0 = C.v(L::RHO, idx) + C.v(L::RHOB, idx);
        const T rtp = C.v(L::RHO, idx + sg) + C.v(L::RHOB, idx + sg);
        const T rtm = C.v(L::RHO, idx - sg) + C.v(L::RHOB, idx - sg);
#pragma unroll
        for (int f = 0; f < D; ++f) {
          const int k = 2 + f;
          const T *v = Q + k * nq + r0;
          T nr, nl;
          nu_at(k, 0, true, nr, nl);
          const T dvp = zd ? T(0) : v[sd] - v[0], dvm = zd ? T(0) : v[0] - v[-sd];
          const T m0 = C.v(L::M0 + f, idx), mp = C.v(L::M0 + f, idx + sg), mm = C.v(L::M0 + f, idx - sg);
          const T fac = (f == d ? (T)1 : (T)0.5) * i2;
          dL[L::M0 + f] += ((rt0 + rtp) * nr * dvp - (rt0 + rtm) * nl * dvm) * (T)0.5 * fac;
          dL[L::EN] += ((m0 + mp) * nr * dvp - (m0 + mm) * nl * dvm) * (T)0.5 * fac;
          if (f != d) {  // off-diagonal: m_d += d_f( rho_t (nu_R+nu_L)/4 d_d v_f )
            const int sf = f == 0 ? 1 : f == 1 ? qb.ext[0] : qb.ext[0] * qb.ext[1];
            const int ff = f == 0 ? 1 : f == 1 ? fb.ext[0] : fb.ext[0] * fb.ext[1];
            const long long gf = g.st[f];
            T t1[2], t2[2];
#pragma unroll
            for (int s = 0; s < 2; ++s) {
              const int o = s ? sf : -sf;
              const int on = s ? ff : -ff;
              const long long go = s ? gf : -gf;
              int cx[3] = {c[0], c[1], c[2]};
              cx[f] += s ? 1 : -1;
              T nr2, nl2;
              nu_at(k, on, cx[f] >= 2 && cx[f] <= g.n[f] - 3, nr2, nl2);
              const T nsum = nr2 + nl2;
              const T tmp5 = z1(g, cx, d) ? T(0) : (v[o + sd] - v[o - sd]) * (T)0.5 * i1;
              const T tmp6 = tmp5 * nsum * (T)0.25;
              t1[s] = (C.v(L::RHO, idx + go) + C.v(L::RHOB, idx + go)) * tmp6;
              t2[s] = tmp6 * C.v(L::M0 + d, idx + go);
            }
            const bool zf = z1(g, c, f);
            const T hf = (T)0.5 * idx1[f];
            if (!zf) {
              dL[L::M0 + d] += (t1[1] - t1[0]) * hf;
              dL[L::EN] += (t2[1] - t2[0]) * hf;
            }
          }
        }
        // magnetic field, f != d
        int ks = 2 + D;
#pragma unroll
        for (int f = 0; f < D; ++f) {
          if (f == d) continue;
          const int k = ks++;
          const T *b = Q + k * nq + r0;
          T nr, nl;
          nu_at(k, 0, true, nr, nl);
          {  // off-diagonal: B_d -= d_f( (nu_L+nu_R)/2 d_d B_f ), e likewise with B_d
            const int sf = f == 0 ? 1 : f == 1 ? qb.ext[0] : qb.ext[0] * qb.ext[1];
            const int ff = f == 0 ? 1 : f == 1 ? fb.ext[0] : fb.ext[0] * fb.ext[1];
            const long long gf = g.st[f];
            T t1[2], t2[2];
#pragma unroll
            for (int s = 0; s < 2; ++s) {
              const int o = s ? sf : -sf;
              const int on = s ? ff : -ff;
              const long long go = s ? gf : -gf;
              int cx[3] = {c[0], c[1], c[2]};
              cx[f] += s ? 1 : -1;
              T nr2, nl2;
              nu_at(k, on, cx[f] >= 2 && cx[f] <= g.n[f] - 3, nr2, nl2);
              const T nsum = nr2 + nl2;
              const T tmp2 = z1(g, cx, d) ? T(0) : (b[o + sd] - b[o - sd]) * (T)0.5 * i1;
              t1[s] = tmp2 * nsum * (T)0.5;
              t2[s] = t1[s] * C.v(L::B0 + d, idx + go);
            }
            if (!z1(g, c, f)) {
              const T hf = (T)0.5 * idx1[f];
              dL[L::B0 + d] -= (t1[1] - t1[0]) * hf;
              dL[L::EN] -= (t2[1] - t2[0]) * hf;
            }
          }
          {  // diagonal: B_f += (nu_R dB+ - nu_L dB-)/dx^2 and Ohmic heating
            const T dbp = zd ? T(0) : b[sd] - b[0], dbm = zd ? T(0) : b[0] - b[-sd];
            dL[L::B0 + f] += (nr * dbp - nl * dbm) * i2;
            dL[L::EN] += ((T)0.5 * (b[0] + b[sd]) * nr * dbp - (T)0.5 * (b[0] + b[-sd]) * nl * dbm) * i2;
          }
        }
      }
    }
    __syncthreads();
  };
  if (p.hyperdif || p.has_bgb) {
    dim_pass(std::integral_constant<int, 0>{});
    dim_pass(std::integral_constant<int, 1>{});
    if constexpr (D == 3) dim_pass(std::integral_constant<int, 2>{});
  }

  stage_epilogue<D, T>(a, g, p, C, c, active, idx, h, dL, numax, red);
}

// One launch = one RK stage of one simulation, one block per tile.
template <int D, typename T>
__global__ void __launch_bounds__(256, 2) tile_stage_kernel(StageArgs a, Geo g, Phys p) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T red[6] = {0, 0, 0, 0, 0, 0};
  tile_body<D, T, TileShape<D>>(a, g, p, blockIdx.x, blockIdx.y, blockIdx.z, reinterpret_cast<T *>(smraw), red);
  block_max_flush<6>(red, &a.sc->red[a.red_out]);
}

// The ghost pass after a tile_stage_kernel launch (grid-stride over the ghosts).
template <int D, typename T>
__global__ void __launch_bounds__(256) ghost_stage_kernel(StageArgs a, Geo g, Phys p) {
  T red[6] = {0, 0, 0, 0, 0, 0};
  const long long ng = ghost_count<D>(g);
  const long long step = (long long)gridDim.x * blockDim.x;
  for (long long k0 = (long long)blockIdx.x * blockDim.x; k0 < ng; k0 += step)
    ghost_cell<D, T>(a, g, p, k0 + threadIdx.x, red);
  block_max_flush<6>(red, &a.sc->red[a.red_out]);
}

// shared memory elements (of the stencil type) the tile body needs
template <int D, typename S = TileShape<D>>
__host__ __device__ constexpr int tile_smem_elems() {
  constexpr int NW = 2 + 2 * D, NQ = 2 * D + 1;
  constexpr int ex[3] = {S::TX, S::TY, D == 3 ? S::TZ : 1};
  // flux box, largest over dir
  int fl = 0, qv = 0;
  for (int dir = 0; dir < D; ++dir) {
    int n = 1, m = 1, u = 1;
    for (int e = 0; e < D; ++e) {
      n *= ex[e] + (e == dir ? 4 : 0);
      m *= ex[e] + (e == dir ? 6 : 2);
      u *= ex[e] + (e == dir ? 1 : 2);  // face box
    }
    fl = fl > NW * n ? fl : NW * n;
    qv = qv > NQ * m + NQ * u ? qv : NQ * m + NQ * u;
  }
  return fl > qv ? fl : qv;
}

}  // namespace SMAUG_NS
