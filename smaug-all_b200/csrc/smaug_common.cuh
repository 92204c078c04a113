// smaug_common.cuh -- host planning and device scalar logic shared by the
// single-simulation context (smaug_capi.cu) and the batch (smaug_batch.cu).
// Everything here has internal linkage in each translation unit.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/smaug_b200.h"
#include "smaug_device.cuh"

// stage kernels of the two builds (stage_exact.cu, stage_fast.cu)
namespace smaug_exact {
void launch_stage(int D, bool mixed, const smaug::StageArgs &a, const smaug::Geo &g, const smaug::Phys &p,
                  cudaStream_t st);
void launch_reduce(int D, const double *w, const double *bg, const smaug::Geo &g, const smaug::Phys &p,
                   smaug::Reduce *r, cudaStream_t st, int const_only = 0);
}  // namespace smaug_exact
namespace smaug_fast {
void launch_stage(int D, bool mixed, const smaug::StageArgs &a, const smaug::Geo &g, const smaug::Phys &p,
                  cudaStream_t st);
void launch_reduce(int D, const double *w, const double *bg, const smaug::Geo &g, const smaug::Phys &p,
                   smaug::Reduce *r, cudaStream_t st, int const_only = 0);
}  // namespace smaug_fast

using namespace smaug;
namespace {

// Sizes, physics and options of one simulation, from its smaug_params.
struct SimPlan {
  int D = 0, NW = 0, NB = 0, NVAR = 0;
  Geo geo{};
  Phys phys{};
  bool rk4 = true, exact = false, mixed = false;
  double dt0 = 0.0;
};

// ndimp of the reference's reductions (computedervfields.cu:1940-1950).
long long ref_ndimp(long long dimp) {
  double fn, fractn, in;
  fn = log((double)dimp) / log(2.0);
  fractn = modf(fn, &in);
  if (fractn > 0) {
    fn += 1;
    return (long long)(int)pow(2, fn);
  }
  return dimp;
}

// Validate params and fill a SimPlan.  Returns an error message or nullptr.
const char *plan_sim(const smaug_params *prm, SimPlan &r) {
  const int D = prm->ndim;
  if (D != 2 && D != 3) return "ndim must be 2 or 3";
  r.D = D;
  r.NW = 2 + 2 * D;
  r.NVAR = 4 + 3 * D;
  r.NB = r.NVAR - r.NW;
  long long N = 1;
  for (int d = 0; d < 3; ++d) {
    const int n = d < D ? prm->n[d] : 1;
    if (d < D && (n < 10 || n > (1 << 20))) return "each dimension needs 10..2^20 cells including ghosts";
    if (d < D) {
      const int t = prm->btype[d];
      if (t != BC_PERIODIC && t != BC_CONT && t != BC_CONTCD4 && t != BC_FIXED && t != BC_SYMM && t != BC_ASYMM)
        return "boundary type must be periodic (0), cont (3), contcd4 (4), fixed (5), symm (6) or asymm (7)";
      if (prm->bmask[d] & ~((1 << (2 + 2 * D)) - 1)) return "bmask may name evolved fields only";
    }
    r.geo.n[d] = n;
    r.geo.btype[d] = d < D ? prm->btype[d] : 0;
    r.geo.bmask[d] = d < D ? prm->bmask[d] : 0;
    N *= n;
  }
  r.geo.has_const = 0;
  for (int d = 0; d < 3; ++d) {
    r.geo.outer_frozen[d] = 0;
    for (int q = d + 1; q < D; ++q)
      if (r.geo.btype[q] == BC_FIXED) r.geo.outer_frozen[d] = d < D;
    if (d < D && r.geo.btype[d] == BC_FIXED) r.geo.has_const = 1;
  }
  if (N * (long long)r.NVAR >= (1LL << 31)) return "grid too large: NVAR * N must stay below 2^31";
  r.geo.st[0] = 1;
  r.geo.st[1] = r.geo.n[0];
  r.geo.st[2] = (long long)r.geo.n[0] * r.geo.n[1];
  r.geo.N = N;
  r.geo.K = ((ref_ndimp(N) + 511) / 512) * 64;
  Phys &p = r.phys;
  p.gamma = prm->gamma;
  p.courant = prm->courant;
  for (int f = 0; f < 13; ++f) p.chyp[f] = prm->chyp[f];
  p.has_grav = 0;
  for (int d = 0; d < 3; ++d) {
    p.g[d] = d < D ? prm->g[d] : 0.0;
    if (p.g[d] != 0.0) p.has_grav = 1;
  }
  p.hyperdif = prm->hyperdif;
  p.dt_mode = prm->dt_mode;
  p.divb = prm->divb != 0;
  for (int d = 0; d < 3; ++d) p.dxs[d] = d < D ? prm->dx[d] : 0.0;
  if (p.divb) {
    if (D != 2) return "divb (divergence-of-B terms) is 2-D only";
    for (int d = 0; d < D; ++d)
      if (!(prm->dx[d] > 0.0)) return "divb needs the grid spacing dx > 0";
  }
  p.drv_on = prm->drv_on != 0;
  p.drv_dir = prm->drv_dir;
  p.drv_amp = prm->drv_amp;
  p.drv_period = prm->drv_period;
  if (p.drv_on) {
    if (prm->drv_dir < 0 || prm->drv_dir >= D) return "drv_dir must name a momentum component (0..ndim-1)";
    if (!(prm->drv_period >= 0.0)) return "drv_period must be >= 0";
    for (int d = 0; d < D; ++d)
      if (!(prm->dx[d] > 0.0) || !(prm->drv_width[d] >= 0.0)) return "driver needs dx > 0 and widths >= 0";
  }
  p.has_bgb = 1;
  r.rk4 = prm->rk4 != 0;
  r.exact = prm->exact != 0;
  r.dt0 = prm->dt0;
  if (prm->precision != SMAUG_PREC_FP64 && prm->precision != SMAUG_PREC_MIXED)
    return "precision must be SMAUG_PREC_FP64 (0) or SMAUG_PREC_MIXED (1)";
  r.mixed = prm->precision == SMAUG_PREC_MIXED;
  if (r.mixed && (!r.rk4 || r.exact)) return "mixed precision needs rk4 = 1 and exact = 0";
  return nullptr;
}

// One direction's pass of the ghost fill of the evolved fields (the rules of
// smaug_device.cuh, field by field, direction by direction as
// iosmaug.cpp:1157-1166): the ghost layers of d from their sources along d,
// which this pass does not write.  Fixed layers, and cells that a later fixed
// pass restores, keep their values.
__global__ void ghost_pass_kernel(double *w, int nw, Geo g, int D, int d) {
  const int n = g.n[d], t = g.btype[d];
  const unsigned neg = bc_neg(g, d);
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < g.N; j += (long long)gridDim.x * blockDim.x) {
    const int x = (int)((j / g.st[d]) % n);
    if (x >= 2 && x <= n - 3) continue;
    if (t == BC_FIXED) continue;
    // a later fixed pass restores this cell (its ghost layers, and the
    // outermost layer of the earlier dims): it keeps its loaded value
    const int c[3] = {(int)(j % g.n[0]), (int)((j / g.n[0]) % g.n[1]), (int)(j / g.st[2])};
    bool later_fixed = false;
    for (int q = d + 1; q < D; ++q) {
      if (g.btype[q] != BC_FIXED) continue;
      if (c[q] < 2 || c[q] > g.n[q] - 3) later_fixed = true;
      for (int e = 0; e < q; ++e)
        if (c[e] == 0 || c[e] == g.n[e] - 1) later_fixed = true;
    }
    if (later_fixed) continue;
    const int xs = bc_source(t, D, n, x);
    const long long src = j + (long long)(xs - x) * g.st[d];
    for (int f = 0; f < nw; ++f) {
      const double v = w[(long long)f * g.N + src];
      w[(long long)f * g.N + j] = ((neg >> f) & 1u) ? -v : v;
    }
  }
}

// Ghost cells of a grid (a coordinate outside [2, n-3]).
inline long long ghost_cells(const Geo &g, int D) {
  long long in = 1;
  for (int d = 0; d < D; ++d) in *= g.n[d] - 4;
  return g.N - in;
}

// The ghost fill of a loaded state, used when a state is loaded
// (iosmaug.cpp:786-794).
void ghost_fill(double *w, int nw, const Geo &g, int D, cudaStream_t s) {
  for (int d = 0; d < D; ++d) ghost_pass_kernel<<<148 * 8, 256, 0, s>>>(w, nw, g, D, d);
}

// The moddton dt block of the reference loop (iosmaug.cpp:855-898):
// dt = courant / maxcourant, then for n > 1 the viscous limit of cugetdtvisc1
// (nushk1.cu:658-790) as that routine actually evaluates it: its buffer holds
// maxviscoef/delx^2 on the first K cells and the courant values c_f/delx of
// the last dimension on the rest.
__device__ __forceinline__ void dt_update(DevScalars *sc, const Phys &p, int D) {
  sc->step += 1;
  const int n = sc->step;
  if (p.dt_mode == 1) {
    const double maxc = red_get(sc->red[0], 3);
    sc->maxcourant = maxc;
    if (((p.courant) / (maxc)) > 1.0e-8) sc->dt = (p.courant) / (maxc);
    if (n > 1) {
      const double cpred = red_get(sc->red[0], 4);
      double dtd = 0.0000000001;
      for (int dir = 0; dir < D; ++dir) {
        double m = cpred;
        double v = ((sc->maxviscoef) + 0.0) / (sc->minsq[dir]);
        if (v > m) m = v;
        if (m > dtd) dtd = m;
        dtd = 0.25 / dtd;
      }
      sc->dtdiffvisc = dtd;
    }
    if ((sc->dtdiffvisc) > 1.0e-8 && (sc->dt) > ((sc->dtdiffvisc))) sc->dt = sc->dtdiffvisc;
  }
  if (!isfinite(sc->dt) || sc->dt <= 0.0) sc->status = SMAUG_ERR_NONFINITE;
  for (int s = 1; s < 5; ++s) sc->red[s] = sc->floor;
  // the RK stage sizes, divided as the oracle divides (dt/2, dt/2, dt, dt/6)
  sc->hst[0] = 0.0;
  sc->hst[1] = sc->dt / 2.0;
  sc->hst[2] = sc->dt / 2.0;
  sc->hst[3] = sc->dt / 1.0;
  sc->hst[4] = sc->dt / 6.0;
}

// End of step: running maximum of the hyperviscosity (the reference's reset
// is undone by cucomputec's params copy, computedervfields.cu:2298-2328) and
// carry the maxima of the new state to slot 0.
__device__ __forceinline__ void finish_update(DevScalars *sc, int last) {
  double nu = 0.0;
  for (int s = 1; s <= last; ++s) nu = fmax(nu, red_get(sc->red[s], 5));
  if (nu > sc->maxviscoef) sc->maxviscoef = nu;
  sc->red[0] = sc->red[last];
  for (int k = 0; k < 6; ++k) {
    double v = red_get(sc->red[0], k);
    if (!isfinite(v)) sc->status = SMAUG_ERR_NONFINITE;
  }
  sc->t += sc->dt;  // simulation time of the next step
}

// Fresh run state: dt0, counters and maxima cleared (minsq kept: it belongs
// to the metric).
__device__ __forceinline__ void reset_update(DevScalars *sc, double dt0) {
  sc->dt = dt0;
  sc->t = 0.0;
  sc->dtdiffvisc = 0.0;
  sc->maxviscoef = 0.0;
  sc->maxcourant = 0.0;
  sc->step = 0;
  sc->status = 0;
  for (int s = 0; s < 5; ++s)
    for (int k = 0; k < 8; ++k) sc->red[s].v[k] = 0ull;
  for (int k = 0; k < 8; ++k) sc->floor.v[k] = 0ull;
}

// FP64 state -> FP32 value + FP32 compensation (w = hi + lo to ~48 bits).
__global__ void split_kernel(const double *__restrict__ w, float *__restrict__ hi, float *__restrict__ lo, long long n) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    const double v = w[j];
    const float h = (float)v;
    hi[j] = h;
    lo[j] = (float)(v - (double)h);
  }
}

// FP32 value + compensation -> FP64 state.
__global__ void combine_kernel(const float *__restrict__ hi, const float *__restrict__ lo, double *__restrict__ w,
                               long long n) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x)
    w[j] = (double)hi[j] + (double)lo[j];
}

// 1-D metric lines, tensor-product check and min delx^2 over the first K
// cells, from a host metric (ndim * N doubles).  Returns an error or nullptr.
// The 1-D metric of each dim along an inner line (n0 + n1 + n2 doubles).
void metric_lines_host(const SimPlan &r, const double *delx, double *d1) {
  const int D = r.D;
  size_t off = 0;
  for (int d = 0; d < D; ++d) {
    const double *m = delx + (size_t)d * r.geo.N;
    for (int x = 0; x < r.geo.n[d]; ++x) {
      int c[3] = {2, 2, D == 3 ? 2 : 0};
      c[d] = x;
      d1[off + x] = m[c[0] + c[1] * r.geo.st[1] + c[2] * r.geo.st[2]];
    }
    off += r.geo.n[d];
  }
}

const char *metric_host(const SimPlan &r, const double *delx, double *d1, double minsq[3]) {
  const int D = r.D;
  const long long N = r.geo.N, K = r.geo.K;
  const int n0 = r.geo.n[0], n1 = r.geo.n[1], n2 = D == 3 ? r.geo.n[2] : 1;
  metric_lines_host(r, delx, d1);
  size_t off = 0;
  for (int d = 0; d < 3; ++d) minsq[d] = INFINITY;
  for (int d = 0; d < D; ++d) {
    const double *m = delx + (size_t)d * N;
    const int n = r.geo.n[d];
    // one pass in storage order (x fastest): inner cells must match the
    // line, every entry must be positive, the first K cells give min delx^2
    const double *line = d1 + off;
    double mn = INFINITY;
    long long j = 0;
    for (int z = 0; z < n2; ++z) {
      const bool zin = D < 3 || (z >= 2 && z <= n2 - 3);
      for (int y = 0; y < n1; ++y) {
        const bool yzin = zin && y >= 2 && y <= n1 - 3;
        const double lyz = d == 1 ? line[y] : line[z];  // the line value when d != 0
        for (int x = 0; x < n0; ++x, ++j) {
          const double v = m[j];
          if (yzin && x >= 2 && x <= n0 - 3 && v != (d == 0 ? line[x] : lyz))
            return "metric is not a tensor-product grid on the inner cells";
          if (!(v > 0.0)) return "metric entries must be positive";
          if (j < K && v * v < mn) mn = v * v;
        }
      }
    }
    minsq[d] = mn;
    off += n;
  }
  return nullptr;
}

// Driver factor lines (n0 + n1 + n2 doubles): along each dim d,
// exp(-(x - c_d)^2 / (w_d * w_d)) at x = xmin_d + i * dx_d, or 1 where w_d = 0
// (usersource.cu.spicule1:77-86; the oracle evaluates the same expression).
void driver_lines(const SimPlan &r, const smaug_params *prm, double *out) {
  size_t off = 0;
  for (int d = 0; d < 3; ++d) {
    const int n = r.geo.n[d];
    for (int i = 0; i < n; ++i) {
      double f = 1.0;
      if (d < r.D && prm->drv_on && prm->drv_width[d] > 0.0) {
        const double x = (prm->xmin[d]) + (((double)i) * (prm->dx[d]));
        const double r2 = (x - prm->drv_center[d]) * (x - prm->drv_center[d]);
        f = exp(-r2 / (prm->drv_width[d] * prm->drv_width[d]));
      }
      out[off + i] = f;
    }
    off += n;
  }
}

// Device-side metric set-up, for a metric in device memory: the 1-D metric of
// each dim along an inner line (into dx1, unless it is null), a tensor-product
// check on the inner cells and a positivity check (status = SMAUG_ERR_ARG on a
// failure), and the minimum of delx_d^2 over the first K cells as an
// order-preserving atomic minimum on the bit patterns of positive doubles
// (minsq must start at +inf).  Cell indices fit 31 bits (plan_sim).
__global__ void metric_kernel(const double *delx, Geo g, int D, double *dx1, DevScalars *sc) {
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nthr = (long long)gridDim.x * blockDim.x;
  long long off = 0;
  const long long nl = (long long)g.n[0] + g.n[1] + g.n[2];  // the reciprocals follow the lines
  for (int d = 0; d < D && dx1; ++d) {
    for (long long x = tid; x < g.n[d]; x += nthr) {
      int c[3] = {2, 2, D == 3 ? 2 : 0};
      c[d] = (int)x;
      const double v = delx[(long long)d * g.N + c[0] + c[1] * g.st[1] + c[2] * g.st[2]];
      dx1[off + x] = v;
      dx1[nl + off + x] = 1.0 / v;
    }
    off += g.n[d];
  }
  // minimum of delx_d^2 over the first K cells: per thread, then per warp,
  // then one atomic per warp (positive doubles order as their bit patterns)
  unsigned long long mn[3] = {~0ull, ~0ull, ~0ull};
  const unsigned n0 = (unsigned)g.n[0], n1 = (unsigned)g.n[1];
  for (long long j = tid; j < g.N; j += nthr) {
    unsigned q = (unsigned)j;
    int c[3];
    c[0] = (int)(q % n0);
    q /= n0;
    c[1] = (int)(q % n1);
    c[2] = (int)(q / n1);
    bool inner = true;
    for (int e = 0; e < D; ++e)
      if (c[e] < 2 || c[e] > g.n[e] - 3) inner = false;
    for (int d = 0; d < D; ++d) {
      const double v = delx[(long long)d * g.N + j];
      if (!(v > 0.0)) atomicExch(&sc->status, (int)SMAUG_ERR_ARG);
      if (inner) {
        int cl[3] = {2, 2, D == 3 ? 2 : 0};
        cl[d] = c[d];
        if (v != delx[(long long)d * g.N + cl[0] + cl[1] * g.st[1] + cl[2] * g.st[2]])
          atomicExch(&sc->status, (int)SMAUG_ERR_ARG);
      }
      if (j < g.K) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(v * v);
        if (b < mn[d]) mn[d] = b;
      }
    }
  }
  for (int d = 0; d < D; ++d) {
    unsigned long long m = mn[d];
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long y = __shfl_xor_sync(0xffffffffu, m, o);
      m = y < m ? y : m;
    }
    if ((threadIdx.x & 31) == 0 && m != ~0ull) atomicMin((unsigned long long *)&sc->minsq[d], m);
  }
}

__global__ void minsq_init_kernel(DevScalars *sc) {
  if (threadIdx.x == 0 && blockIdx.x == 0)
    for (int d = 0; d < 3; ++d) sc->minsq[d] = INFINITY;
}

// Is the energy background live (a nonzero e_b or B_b anywhere)?  OR-ed
// into sc->bg_live, which the caller clears first.
__global__ void bg_scan_kernel(const double *__restrict__ bg, long long N, int D, DevScalars *sc) {
  int any = 0;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < N; j += (long long)gridDim.x * blockDim.x) {
    any |= bg[j] != 0.0;  // e_b
    for (int k = 0; k < D; ++k) any |= bg[(2 + k) * N + j] != 0.0;  // B_b
  }
  if (__syncthreads_or(any) && threadIdx.x == 0) atomicOr(&sc->bg_live, 1);
}

}  // namespace
