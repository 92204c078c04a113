// smaug_cucompat.cu -- the reference's per-operator GPU entry points
// (include/smaug_cukernels.h) over FP64 kernels of this library.
//
// Built once per dimensionality, SMAUG_CU_NDIM = 2 and 3, into
// libsmaug_cu2d.so and libsmaug_cu3d.so, without FMA contraction
// (-fmad=false).  Each kernel is one operator of the reference's single step,
// one thread per cell over a grid-stride loop, with the reference's outputs in
// the reference's arrays (wmod slots, wd derived fields, wtemp temporaries)
// and its arithmetic in its operation order, so that a host loop of the
// reference's shape (iosmaug.cpp:802-1166) gives the reference's bits.  The
// fused production path (smaug_step in libsmaug_b200.so) is the fast way to
// run the same step; these entry points exist so that a host written against
// the reference's interface links and runs unchanged, and so that single
// operators can be compared with the reference one at a time.
//
// Maxima (cmax, maxcourant, the hyperviscosity, the viscous dt) are taken on
// the device as order-preserving atomic maxima of non-negative doubles' bit
// patterns (a NaN is skipped, as the reference's `>` comparisons skip it) and
// copied back into struct params, as the reference's reductions do.
// All calls are synchronous on the legacy default stream, as in the reference.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/smaug_b200.h"
#include "../../include/smaug_cukernels.h"

namespace {

constexpr int kD = SMAUG_CU_NDIM;
// field ids (the reference's enum vars): the evolved fields first
constexpr int kNW = 2 + 2 * kD, kRHO = 0, kM0 = 1, kEN = 1 + kD, kB0 = 2 + kD, kEB = 2 + 2 * kD,
              kRHOB = 3 + 2 * kD, kBB0 = 4 + 2 * kD;

struct Grid {
  int n[3];
  long long N, st[3];
  int bt[3];  // per direction: boundtype[rho][d][0] (0 periodic: no gradient zeroing)
};

struct Shim {
  bool ready = false;
  Grid g{};
  int nslots = 0;
  double maxvisc = 0.0;                // running maximum of the hyperviscosity (p->maxviscoef)
  unsigned long long *d_max = nullptr;  // device maxima (bit patterns of non-negative doubles)
  std::string err;
} S;

int fail(int code, const std::string &m) {
  S.err = m;
  return code;
}

#define CUCK(call)                                                                                   \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess) return fail(SMAUG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// launch, then wait (the reference synchronises after every launch)
#define LAUNCH(kernel, ...)                               \
  do {                                                    \
    kernel<<<blocks(), 256>>>(__VA_ARGS__);                \
    CUCK(cudaGetLastError());                             \
    CUCK(cudaDeviceSynchronize());                        \
  } while (0)

int blocks() {
  const long long b = (S.g.N + 255) / 256;
  return (int)(b < 148 * 16 ? b : 148 * 16);
}

int ready(struct params **p) {
  if (!p || !*p) return fail(SMAUG_ERR_ARG, "null params");
  if (!S.ready) return fail(SMAUG_ERR_STATE, "cuinit must come first");
  return SMAUG_OK;
}

int slot_ok(int order) {
  if (order < 0 || order >= S.nslots) return fail(SMAUG_ERR_ARG, "slot out of range");
  return SMAUG_OK;
}

#define REQUIRE(x)          \
  do {                      \
    const int rc_ = (x);    \
    if (rc_ != SMAUG_OK) return rc_; \
  } while (0)

// ------------------------------------------------------------- device helpers

__device__ __forceinline__ double *fld(double *w, int f, long long N) { return w + (long long)f * N; }

#define GRID_LOOP(i, N) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (N); \
                             i += (long long)gridDim.x * blockDim.x)

__device__ __forceinline__ void coords(const Grid &g, long long i, int *c) {
  c[0] = (int)(i % g.n[0]);
  c[1] = (int)((i / g.n[0]) % g.n[1]);
  c[2] = (int)(i / g.st[2]);
}

__device__ __forceinline__ bool inner(const Grid &g, const int *c) {
  for (int d = 0; d < kD; ++d)
    if (c[d] < 2 || c[d] > g.n[d] - 3) return false;
  return true;
}

// the coordinates other than d within [lo, n-1-lo]
__device__ __forceinline__ bool others_in(const Grid &g, const int *c, int d, int lo) {
  for (int e = 0; e < kD; ++e)
    if (e != d && (c[e] < lo || c[e] > g.n[e] - 1 - lo)) return false;
  return true;
}

// grad3dn (gradops.cu:437-606): 4th-order central difference over the cell
// width dxd; zeroed near non-periodic edges with the reference's operator
// precedence (the n-3 and 2 tests are unconditional)
__device__ double grad3dn(const Grid &g, const double *a, const double *dxd, long long idx, const int *c, int d) {
  double grad = 0;
  const int n = g.n[d];
  const long long s = g.st[d];
  if (c[d] > 1 && c[d] < n - 2)
    grad = (((8 * a[idx + s] - 8 * a[idx - s] + a[idx - 2 * s] - a[idx + 2 * s]) / 6.0)) / (2.0 * (dxd[idx]));
  if (g.bt[d] != 0) {
    if ((c[d] == n - 3) || (c[d] == n - 4 && others_in(g, c, d, 2)))
      grad = 0;
    else if (c[d] == 2 || (c[d] == 3 && others_in(g, c, d, 2)))
      grad = 0;
  }
  return grad;
}

// grad1r3n / grad1l3n (gradops.cu:608-753) at inner cells
__device__ double grad1r(const Grid &g, const double *a, const double *dxd, long long idx, const int *c, int d) {
  const int n = g.n[d];
  double grad = 0;
  if (c[d] < n - 1) grad = ((a[idx + g.st[d]] - a[idx]) / ((dxd[idx])));
  if (g.bt[d] != 0 && (c[d] == n - 2 || c[d] == n - 3 || c[d] == 1 || c[d] == 2)) grad = 0;
  return grad;
}
__device__ double grad1l(const Grid &g, const double *a, const double *dxd, long long idx, const int *c, int d) {
  const int n = g.n[d];
  double grad = 0;
  if (c[d] > 0 && c[d] < n) grad = ((a[idx] - a[idx - g.st[d]]) / ((dxd[idx])));
  if (g.bt[d] != 0 && (c[d] == n - 2 || c[d] == n - 3 || c[d] == 1 || c[d] == 2)) grad = 0;
  return grad;
}

// grad13n (gradops.cu:755-826): 2nd-order central difference on [1, n-2]
__device__ double grad13(const Grid &g, const double *a, const double *dxd, long long idx, const int *c, int d) {
  const int n = g.n[d];
  double grad = 0;
  if (c[d] > 0 && c[d] < n - 1) {
    grad = ((a[idx + g.st[d]] - a[idx - g.st[d]]) / ((dxd[idx])) / 2.0);
    if (g.bt[d] != 0) {
      if ((c[d] == n - 2) || (c[d] == n - 3 && others_in(g, c, d, 1)))
        grad = 0;
      else if (kD == 3 && d == 2) {
        if (c[d] == 1 || (c[d] == 2 && c[0] > 0 && c[0] < g.n[0] - 1 && c[1] > 1 && c[1] < g.n[1] - 1)) grad = 0;
      } else if (c[d] == 1 || (c[d] == 2 && others_in(g, c, d, 1)))
        grad = 0;
    }
  }
  return grad;
}

// grad3d (gradops.cu:132-237, 2-D): 4th-order difference over the uniform
// spacing dxs, zero at the first and last two inner cells
__device__ double grad3d(const Grid &g, const double *a, double dxs, long long idx, const int *c, int dir) {
  const int n = g.n[dir], x = c[dir], o = 1 - dir;
  const long long s = g.st[dir];
  double grad = 0;
  if (x > 1 && x < n - 2) grad = (((8 * a[idx + s] - 8 * a[idx - s] + a[idx - 2 * s] - a[idx + 2 * s]) / 6.0)) / (2.0 * (dxs));
  const bool in_o = c[o] > 1 && c[o] < g.n[o] - 2;
  if ((x == n - 3) || (x == n - 4 && in_o))
    grad = 0;
  else if (x == 2 || (x == 3 && in_o))
    grad = 0;
  return grad;
}

__device__ __forceinline__ void dmax(unsigned long long *slot, double v) {
  if (v > 0.0) atomicMax(slot, (unsigned long long)__double_as_longlong(v));  // NaN and 0 never raise it
}

// ------------------------------------------------------------------ kernels

// cucomputedervfields (computedervfields.cu:1594-1888): with order 0 the
// derived fields vel1..pkb are cleared and the evolved fields of slot 1 become
// slot 0; then B.v of slot `order` (computebdotv3, dervfields.cu:46-52)
__global__ void k_dervfields(Grid g, double *wmod, double *wd, int order) {
  const long long N = g.N, slot = (long long)NVAR * N;
  GRID_LOOP(i, N) {
    if (order == 0) {
      for (int f = vel1; f <= pkb; ++f) wd[f * N + i] = 0;
      for (int f = 0; f < kNW; ++f) wmod[f * N + i] = wmod[f * N + i + slot];
    }
    const double *w = wmod + order * slot;
    double s = 0;
    for (int k = 0; k < kD; ++k) {
      const double t = (w[(kB0 + k) * N + i] + w[(kBB0 + k) * N + i]) * w[(kM0 + k) * N + i];
      s = k == 0 ? t : s + t;
    }
    wd[bdotv * N + i] = s / (w[kRHO * N + i] + w[kRHOB * N + i]);
  }
}

// velocity along dir (computevel3, dervfields.cu:79-98)
__global__ void k_vel(Grid g, const double *w, double *wd, int dir) {
  const long long N = g.N;
  GRID_LOOP(i, N) wd[(vel1 + dir) * N + i] = w[(kM0 + dir) * N + i] / (w[kRHO * N + i] + w[kRHOB * N + i]);
}

// total pressure (computept3, dervfields.cu:107-153)
__global__ void k_pt(Grid g, const double *w, double *wd, double gam) {
  const long long N = g.N;
  GRID_LOOP(i, N) {
    double bb = 0, b2 = 0, m2 = 0;
    for (int k = 0; k < kD; ++k) bb += w[(kB0 + k) * N + i] * w[(kBB0 + k) * N + i];
    for (int k = 0; k < kD; ++k) b2 += w[(kB0 + k) * N + i] * w[(kB0 + k) * N + i];
    for (int k = 0; k < kD; ++k) m2 += w[(kM0 + k) * N + i] * w[(kM0 + k) * N + i];
    const double t = ((gam)-2.0) * ((bb) + 0.5 * (b2));
    wd[pressuret * N + i] = ((gam)-1.0) * (w[kEN * N + i] - 0.5 * (m2) / (w[kRHO * N + i] + w[kRHOB * N + i])) - t;
  }
}

// kinetic-gas pressure (computepk3, dervfields.cu:195-240)
__global__ void k_pk(Grid g, const double *w, double *wd, double gam) {
  const long long N = g.N;
  GRID_LOOP(i, N) {
    double m2 = 0, b2 = 0, bbb = 0;
    for (int k = 0; k < kD; ++k) {
      const double mk = w[(kM0 + k) * N + i], bk = w[(kB0 + k) * N + i];
      m2 = k == 0 ? mk * mk : m2 + mk * mk;
      b2 = k == 0 ? bk * bk : b2 + bk * bk;
      bbb = k == 0 ? bk * w[(kBB0 + k) * N + i] : bbb + bk * w[(kBB0 + k) * N + i];
    }
    double pk = 0.5 * ((m2) / (w[kRHO * N + i] + w[kRHOB * N + i]));
    pk = pk + (0.5 * (b2) + (bbb));
    wd[pressurek * N + i] = ((gam)-1) * w[kEN * N + i] - pk;
  }
}

// background pressure (computepbg3, dervfields.cu:157-191)
__global__ void k_pbg(Grid g, const double *w, double *wd, double gam) {
  const long long N = g.N;
  GRID_LOOP(i, N) {
    double bb2 = 0;
    for (int k = 0; k < kD; ++k) bb2 += w[(kBB0 + k) * N + i] * w[(kBB0 + k) * N + i];
    wd[ptb * N + i] = ((gam)-1) * w[kEB * N + i] - 0.5 * ((gam)-2) * (bb2);
  }
}

// sound and fast speeds along dir (computec3, dervfields.cu:241-309)
__global__ void k_c(Grid g, const double *w, double *wd, double gam, int dir) {
  const long long N = g.N;
  GRID_LOOP(i, N) {
    double m2 = 0, b2 = 0, bbb = 0, bb2 = 0;
    for (int k = 0; k < kD; ++k) m2 += w[(kM0 + k) * N + i] * w[(kM0 + k) * N + i];
    for (int k = 0; k < kD; ++k) b2 += w[(kB0 + k) * N + i] * w[(kB0 + k) * N + i];
    for (int k = 0; k < kD; ++k) bbb += w[(kBB0 + k) * N + i] * w[(kB0 + k) * N + i];
    for (int k = 0; k < kD; ++k) bb2 += w[(kBB0 + k) * N + i] * w[(kBB0 + k) * N + i];
    const double rt = w[kRHO * N + i] + w[kRHOB * N + i];
    const double pk = ((gam)-1) * (w[kEN * N + i] - 0.5 * ((m2) / (rt)) - 0.5 * (b2) - (bbb));
    const double cs2 = (((gam)) * (pk + (((gam)) - 1) * (w[kEB * N + i] - 0.5 * (bb2))) / (rt));
    const double cf = ((b2) + (bb2) + 2.0 * (bbb)) / (rt) + (cs2);
    const double bd = w[(kBB0 + dir) * N + i] + w[(kB0 + dir) * N + i];
    const double cfasti = 0.5 * (cf + sqrt(cf * cf - 4.0 * cs2 * ((bd) * (bd)) / (rt)));
    wd[cfast * N + i] = sqrt(cfasti) + fabs(w[(kM0 + dir) * N + i] / (rt));
    wd[soundspeed * N + i] = sqrt(cs2);
  }
}

// max over all cells of wd[cfast] (cucomputemaxc: ghosts included, from 0)
__global__ void k_max_field(Grid g, const double *a, unsigned long long *out) {
  GRID_LOOP(i, g.N) dmax(out, a[i]);
}

// courant numbers c_fast / delx_dir into temp, and their maximum
// (cucomputemaxcourant, computedervfields.cu:2118-2296)
__global__ void k_courant(Grid g, const double *wd, double *temp, int dir, unsigned long long *out) {
  const long long N = g.N;
  GRID_LOOP(i, N) {
    const double v = wd[cfast * N + i] / (wd[(delx1 + dir) * N + i]);
    temp[i] = v;
    dmax(out, v);
  }
}

// cugetdtvisc1 (nushk1.cu:658-790) as it evaluates: its reduced buffer holds
// maxviscoef / delx^2 on the first K cells and the courant values that
// cucomputemaxcourant left in temp on the rest
__global__ void k_dtvisc(Grid g, const double *wd, const double *temp, long long K, double mv,
                         unsigned long long *out) {
  const long long N = g.N;
  GRID_LOOP(i, N) {
    if (i >= K) {
      dmax(&out[0], temp[i]);
    } else {
      for (int dir = 0; dir < kD; ++dir) {
        const double dx = wd[(delx1 + dir) * N + i];
        dmax(&out[1 + dir], ((mv) + 0.0) / ((dx) * (dx)));
      }
    }
  }
}

// the flux of `field` along dir at every cell (centdiff1.cu:51-256,
// centdiff2.cu:189-340), with the total pressure of wd[pressuret]
__device__ double flux_at(const Grid &g, const double *w, const double *pt, long long i, int f, int dir) {
  const long long N = g.N;
  const double r = w[kRHO * N + i], rb = w[kRHOB * N + i];
  const double rt = r + rb;
  const double md = w[(kM0 + dir) * N + i];
  if (f == kRHO) return md * r / (r + rb) + (rb * md) / (rb + r);
  if (f >= kM0 && f < kM0 + kD) {
    const int k = f - kM0;
    const double tr = md * w[f * N + i] / (rt);
    const double bf = w[(kB0 + k) * N + i], bbf = w[(kBB0 + k) * N + i];
    const double bbd = w[(kBB0 + dir) * N + i], bd = w[(kB0 + dir) * N + i];
    const double mg = (k == dir) ? pt[i] - (bf * bbd + bbf * bd) - bf * bd : -(bf * bbd + bbf * bd) - bf * bd;
    return tr + mg;
  }
  if (f == kEN) {
    double bbm = 0, bm = 0;
    for (int k = 0; k < kD; ++k) bbm += w[(kBB0 + k) * N + i] * w[(kM0 + k) * N + i];
    for (int k = 0; k < kD; ++k) bm += w[(kB0 + k) * N + i] * w[(kM0 + k) * N + i];
    const double tr = md * w[kEN * N + i] / (rt);
    double fl = md * (pt[i]);
    fl -= w[(kB0 + dir) * N + i] * (bbm);
    fl -= w[(kBB0 + dir) * N + i] * (bm);
    fl /= (rt);
    fl += md * w[kEB * N + i] / (rt);
    fl -= w[(kB0 + dir) * N + i] * (bm) / (rt);
    return tr + fl;
  }
  const int k = f - kB0;  // induction; none along dir
  if (k == dir) return 0.0;
  return md * w[f * N + i] / (rt) - (w[(kB0 + dir) * N + i] + w[(kBB0 + dir) * N + i]) * w[(kM0 + k) * N + i] / (rt) +
         (w[(kBB0 + k) * N + i]) * md / (rt);
}

__global__ void k_flux(Grid g, const double *w, double *wd, int f, int dir) {
  const long long N = g.N;
  GRID_LOOP(i, N) wd[flux * N + i] = flux_at(g, w, wd + pressuret * N, i, f, dir);
}

// w_out[f] -= dt * d_dir(flux) at inner cells; for the energy also the
// background energy terms (addenergyterms_cd2, centdiff2.cu:80-115) from
// wd[ptb] and the velocity wd[vel_dir]
__global__ void k_divflux(Grid g, double *wout, const double *wd, double dt, int f, int dir) {
  const long long N = g.N;
  const double *dxd = wd + (delx1 + dir) * N;
  GRID_LOOP(idx, N) {
    int c[3];
    coords(g, idx, c);
    if (!inner(g, c)) continue;
    double *o = wout + f * N;
    o[idx] = o[idx] - dt * grad3dn(g, wd + flux * N, dxd, idx, c, dir);
    if (f == kEN) {
      const double *v = wd + (vel1 + dir) * N;
      o[idx] -= +(dt)*wd[ptb * N + idx] * grad3dn(g, v, dxd, idx, c, dir);
      for (int idim = 0; idim < kD; idim++)
        o[idx] += (dt)*wout[(kBB0 + idim) * N + idx] * wout[(kBB0 + dir) * N + idx] *
                  grad3dn(g, v, wd + (delx1 + idim) * N, idx, c, idim);
    }
  }
}

// gravity (addgrav_cd2, centdiff2.cu:118-150) at inner cells
__global__ void k_grav(Grid g, const double *win, double *wout, double dt, double g0, double g1, double g2) {
  const long long N = g.N;
  const double gg[3] = {g0, g1, g2};
  GRID_LOOP(idx, N) {
    int c[3];
    coords(g, idx, c);
    if (!inner(g, c)) continue;
    for (int k = 0; k < kD; ++k) wout[(kM0 + k) * N + idx] += (dt) * (gg[k]) * win[kRHO * N + idx];
    for (int k = 0; k < kD; ++k)
      wout[kEN * N + idx] += (dt)*win[kRHO * N + idx] * ((gg[k]) * win[(kM0 + k) * N + idx]) /
                             (win[kRHO * N + idx] + win[kRHOB * N + idx]);
  }
}

// divergence-of-B sources (divb_parallel, divb.cu:165-336, divbon = divbfix
// = 1; 2-D): -divB (0, B, B.v, v) at cells 3..n-3, applied as w -= dt * source
// at the inner cells from 2
__global__ void k_divb(Grid g, const double *win, double *wout, double dt, double dxs0, double dxs1) {
  const long long N = g.N;
  GRID_LOOP(idx, N) {
    int c[3];
    coords(g, idx, c);
    if (!(c[0] > 1 && c[1] > 1 && c[0] < g.n[0] - 2 && c[1] < g.n[1] - 2)) continue;
    double dw[kNW];
    for (int f = 0; f < kNW; ++f) dw[f] = 0.0;
    if (c[0] > 2 && c[1] > 2) {
      const double dxs[2] = {dxs0, dxs1};
      double dv = grad3d(g, win + kB0 * N, dxs[0], idx, c, 0) + grad3d(g, win + (kB0 + 1) * N, dxs[1], idx, c, 1);
      dv += grad3d(g, win + kBB0 * N, dxs[0], idx, c, 0) + grad3d(g, win + (kBB0 + 1) * N, dxs[1], idx, c, 1);
      const double rt = win[kRHO * N + idx] + win[kRHOB * N + idx];
      const double bv = ((win[kB0 * N + idx] + win[kBB0 * N + idx]) * win[kM0 * N + idx] +
                         (win[(kB0 + 1) * N + idx] + win[(kBB0 + 1) * N + idx]) * win[(kM0 + 1) * N + idx]) / rt;
      for (int k = 0; k < 2; ++k) {
        const double sm = -dv * win[(kB0 + k) * N + idx];
        dw[kM0 + k] = dw[kM0 + k] + (isnan(sm) ? 0 : sm);
        const double sb = -dv * win[(kM0 + k) * N + idx] / (win[kRHO * N + idx] + win[kRHOB * N + idx]);
        dw[kB0 + k] = dw[kB0 + k] + (isnan(sb) ? 0 : sb);
      }
      dw[kEN] = dw[kEN] + (-dv * bv);
    }
    for (int f = 0; f < kNW; ++f) wout[f * N + idx] = wout[f * N + idx] - dt * dw[f];
  }
}

// the hyperviscosity input q of `field` (hyperdifvisc1r.cu:1222-1262) into
// temp: the density, the internal energy e - (B^2 + m^2/rho_t)/2, a
// velocity m_f / rho_t or a field component B_f
__global__ void k_hyper_q(Grid g, const double *w, double *temp, int field) {
  const long long N = g.N;
  GRID_LOOP(i, N) {
    double q;
    if (field == kEN) {
      double b2 = 0, m2 = 0;
      for (int k = 0; k < kD; ++k) b2 += w[(kB0 + k) * N + i] * w[(kB0 + k) * N + i];
      for (int k = 0; k < kD; ++k) m2 += w[(kM0 + k) * N + i] * w[(kM0 + k) * N + i];
      q = w[kEN * N + i] - 0.5 * ((b2) + (m2) / (w[kRHO * N + i] + w[kRHOB * N + i]));
    } else if (field >= kM0 && field < kM0 + kD) {
      q = w[field * N + i] / (w[kRHO * N + i] + w[kRHOB * N + i]);
    } else {
      q = w[field * N + i];
    }
    temp[i] = q;
  }
}

// q along d at offset `off` from cell c in the padded copies of the chains:
// right pad 0, left pad q(5) (bc_hyperdifl, hyperdifvisc1l.cu:17-66)
__device__ __forceinline__ double qat(const Grid &g, const double *q, long long idx, const int *c, int d, int off) {
  int x = c[d] + off;
  if (x >= g.n[d]) return 0.0;
  if (x < 0) x = 5;
  return q[idx + (long long)(x - c[d]) * g.st[d]];
}

// right (side 0) or left (side 1) hyperviscosity of q along d at inner cells
// (hyperdifvisc2r/3r/4r, hyperdifvisc1r.cu:426-845; 2l/3l/4l,
// hyperdifvisc1l.cu:436-855), 0 elsewhere, into nu; maximum into out
__global__ void k_hyper_nu(Grid g, const double *q, const double *wd, double *nu, int d, double cmax, double chyp,
                           int side, unsigned long long *out) {
  const long long N = g.N;
  GRID_LOOP(idx, N) {
    int c[3];
    coords(g, idx, c);
    double r = 0;
    if (inner(g, c)) {
      const double dx = wd[(delx1 + d) * N + idx];
      double maxt1 = 0, maxt2 = 0;
      for (int s = -1; s <= 1; ++s) {
        const int a = s + 1;
        const double v = side == 0 ? fabs(3.0 * (qat(g, q, idx, c, d, a) - qat(g, q, idx, c, d, a - 1)) -
                                          (qat(g, q, idx, c, d, a + 1) - qat(g, q, idx, c, d, a - 2)))
                                   : fabs(3.0 * (qat(g, q, idx, c, d, a - 1) - qat(g, q, idx, c, d, a - 2)) -
                                          (qat(g, q, idx, c, d, a) - qat(g, q, idx, c, d, a - 3)));
        if (v > maxt1) maxt1 = v;
      }
      for (int s = -2; s <= 2; ++s) {
        const double v = side == 0 ? fabs((qat(g, q, idx, c, d, s + 1) - qat(g, q, idx, c, d, s)))
                                   : fabs(qat(g, q, idx, c, d, s) - (qat(g, q, idx, c, d, s - 1)));
        if (v > maxt2) maxt2 = v;
      }
      if (maxt2 > 0) r = ((dx)) * (cmax) * (chyp)*maxt1 / maxt2;
    }
    nu[idx] = r;
    dmax(out, r);
  }
}

// density / internal-energy hyperdiffusion (hyperdifrhosource1.cu:15-282,
// hyperdifesource1.cu:18-554): f += dt (nu_R dq+ - nu_L dq-) / delx at inner cells
__global__ void k_hyper_scalar(Grid g, const double *q, const double *wd, double *wout, int f, int d, double dt) {
  const long long N = g.N;
  const double *dxd = wd + (delx1 + d) * N;
  GRID_LOOP(idx, N) {
    int c[3];
    coords(g, idx, c);
    if (!inner(g, c)) continue;
    double tp, tm;
    if (f == kRHO) {
      tp = grad1r(g, q, dxd, idx, c, d);
      tm = grad1l(g, q, dxd, idx, c, d);
    } else {
      tm = grad1l(g, q, dxd, idx, c, d);
      tp = grad1r(g, q, dxd, idx, c, d);
    }
    const double rdx = dxd[idx];
    wout[f * N + idx] =
        wout[f * N + idx] + dt * ((wd[hdnur * N + idx] + 0.0) * tp - (wd[hdnul * N + idx] + 0.0) * tm) / rdx;
  }
}

// momentum hyperdiffusion, the diagonal terms (hyperdifmomsource1.cu): m_ii0
// and e from the face-averaged rho_t and m_ii0 and the velocity v along d
__global__ void k_hyper_mom_diag(Grid g, const double *win, const double *v, const double *wd, double *wout, int d,
                                 int ii0, double dt) {
  const long long N = g.N;
  const double *dxd = wd + (delx1 + d) * N;
  GRID_LOOP(idx, N) {
    int c[3];
    coords(g, idx, c);
    if (!inner(g, c)) continue;
    const long long s = g.st[d];
    const double *r = win + kRHO * N, *rb = win + kRHOB * N, *m = win + (kM0 + ii0) * N;
    const double tmp2 = (r[idx] + rb[idx] + r[idx - s] + rb[idx - s]) / 2;
    const double tmp3 = (r[idx] + rb[idx] + r[idx + s] + rb[idx + s]) / 2;
    const double tmp5 = (m[idx] + m[idx - s]) / 2;
    const double tmp6 = (m[idx] + m[idx + s]) / 2;
    const double tmp8 = grad1r(g, v, dxd, idx, c, d);
    const double tmp7 = grad1l(g, v, dxd, idx, c, d);
    const double rdx = dxd[idx];
    const double nur = wd[hdnur * N + idx], nul = wd[hdnul * N + idx];
    const double dm = (tmp3 * (nur + 0.0) * tmp8 - tmp2 * (nul + 0.0) * tmp7) / (rdx) / 2;
    wout[(kM0 + ii0) * N + idx] = wout[(kM0 + ii0) * N + idx] + dt * dm;
    const double de = (tmp6 * (nur + 0.0) * tmp8 - tmp5 * (nul + 0.0) * tmp7) / (rdx) / 2;
    wout[kEN * N + idx] = wout[kEN * N + idx] + dt * de;
  }
}

// momentum hyperdiffusion, the off-diagonal terms (hyperdifmomsourcene1.cu):
// on [1, n-2]^D, t1 = rho_t tmp6 and t2 = tmp6 m_ii0 with
// tmp6 = d_d v (nu_R + nu_L) / 4
__global__ void k_hyper_mom_off_t(Grid g, const double *win, const double *v, const double *wd, double *t1,
                                  double *t2, int d, int ii0) {
  const long long N = g.N;
  GRID_LOOP(idx, N) {
    int c[3];
    coords(g, idx, c);
    bool ok = true;
    for (int e = 0; e < kD; ++e)
      if (c[e] < 1 || c[e] > g.n[e] - 2) ok = false;
    const double tmp5 = ok ? grad13(g, v, wd + (delx1 + d) * N, idx, c, d) : 0.0;
    const double tmp6 = tmp5 * ((wd[hdnur * N + idx] + wd[hdnul * N + idx] + 2.0 * 0.0)) / 4.0;
    t1[idx] = (win[kRHO * N + idx] + win[kRHOB * N + idx]) * tmp6;
    t2[idx] = tmp6 * win[(kM0 + ii0) * N + idx];
  }
}

// the off-diagonal update along ii: target += dt * sb * d_ii(t1), e += dt * sb * d_ii(t2)
__global__ void k_hyper_off_apply(Grid g, const double *t1, const double *t2, const double *wd, double *wout, int tf,
                                  int ii, double sb, int signed_form, double dt) {
  const long long N = g.N;
  const double *dxd = wd + (delx1 + ii) * N;
  GRID_LOOP(idx, N) {
    int c[3];
    coords(g, idx, c);
    if (!inner(g, c)) continue;
    const double a = grad13(g, t1, dxd, idx, c, ii), b = grad13(g, t2, dxd, idx, c, ii);
    const double dm = signed_form ? sb * a : a;
    const double de = signed_form ? sb * b : b;
    wout[tf * N + idx] = wout[tf * N + idx] + dt * dm;
    wout[kEN * N + idx] = wout[kEN * N + idx] + dt * de;
  }
}

// magnetic hyperdiffusion, the diagonal terms (hyperdifbsource1.cu): B_ii0 and
// the Ohmic heating in e from B_f along d and the face-averaged B_jj
__global__ void k_hyper_b_diag(Grid g, const double *win, const double *wd, double *wout, int f, int d, int jj,
                               int ii0, double sb, double dt) {
  const long long N = g.N;
  const double *dxd = wd + (delx1 + d) * N;
  GRID_LOOP(idx, N) {
    int c[3];
    coords(g, idx, c);
    if (!inner(g, c)) continue;
    const long long s = g.st[d];
    const double *b = win + (kB0 + f) * N, *bj = win + (kB0 + jj) * N;
    const double tmp2 = (bj[idx] + bj[idx - s]) / 2;
    const double tmp3 = (bj[idx] + bj[idx + s]) / 2;
    const double tmp4 = grad1l(g, b, dxd, idx, c, d);
    const double tmp5 = grad1r(g, b, dxd, idx, c, d);
    const double rdx = dxd[idx];
    const double nur = wd[hdnur * N + idx], nul = wd[hdnul * N + idx];
    const double db = sb * (tmp5 * nur - tmp4 * nul) / rdx;
    const double de = sb * (tmp3 * tmp5 * nur - tmp2 * tmp4 * nul) / rdx;
    wout[(kB0 + ii0) * N + idx] = wout[(kB0 + ii0) * N + idx] + dt * db;
    wout[kEN * N + idx] = wout[kEN * N + idx] + dt * de;
  }
}

// magnetic hyperdiffusion, the off-diagonal terms (hyperdifbsourcene1.cu): on
// [1, n-2]^D, t1 = d_d B_f (nu_L + nu_R) / 2, t2 = t1 B_jj
__global__ void k_hyper_b_off_t(Grid g, const double *win, const double *wd, double *t1, double *t2, int f, int d,
                                int jj) {
  const long long N = g.N;
  GRID_LOOP(idx, N) {
    int c[3];
    coords(g, idx, c);
    bool ok = true;
    for (int e = 0; e < kD; ++e)
      if (c[e] < 1 || c[e] > g.n[e] - 2) ok = false;
    const double tmp2 = ok ? grad13(g, win + (kB0 + f) * N, wd + (delx1 + d) * N, idx, c, d) : 0.0;
    t1[idx] = tmp2 * (wd[hdnul * N + idx] + wd[hdnur * N + idx]) / 2;
    t2[idx] = t1[idx] * win[(kB0 + jj) * N + idx];
  }
}

// ghost cells of one field along dir (boundary.cu.sedov3d for periodic and
// contcd4, gradops.cu bc3_cont_dir / bc3_symm_dir / bc3_asymm_dir)
__global__ void k_boundary(Grid g, double *a, int dir, int type) {
  const int n = g.n[dir];
  const long long s = g.st[dir];
  GRID_LOOP(idx, g.N) {
    int c[3];
    coords(g, idx, c);
    const int x = c[dir];
    if (x >= 2 && x <= n - 3) continue;
    double sign = 1.0;
    int xs;
    switch (type) {
      case 0: xs = x < 2 ? x + (n - 4) : x - (n - 4); break;
      case 3: xs = x < 2 ? 2 : n - 3; break;
      case 4: xs = x == 0 ? 4 : x == 1 ? 3 : x == n - 1 ? n - 5 : n - 4; break;
      case 7: sign = -1.0;  // fall through: the symm source, negated
      default:
        if (kD == 2) xs = x == 0 ? 3 : x == 1 ? 2 : x == n - 1 ? n - 4 : n - 3;
        else xs = x == 0 ? 4 : x == 1 ? 3 : x == n - 1 ? n - 5 : n - 4;
        break;
    }
    a[idx] = sign * a[idx + (long long)(xs - x) * s];
  }
}

// the Runge-Kutta slot algebra (advance_parallel, advance.cu:18-174) over all
// NVAR fields of every cell
__global__ void k_advance(Grid g, double *wmod, int order, int rkon) {
  const long long N = g.N, sl = (long long)NVAR * N;
  GRID_LOOP(i, sl) {
    if (rkon == 1) {
      switch (order) {
        case 0: wmod[i + 2 * sl] = wmod[i]; break;
        case 1: wmod[i + 3 * sl] = wmod[i]; break;
        case 2: wmod[i + sl] = (wmod[i + sl] + 2.0 * wmod[i + 2 * sl] + wmod[i + 3 * sl] - 4.0 * wmod[i]) / 3; break;
        case 3: wmod[i] = wmod[i] + wmod[i + sl]; break;
        default: break;
      }
    } else {
      wmod[i] = wmod[i + sl];
    }
  }
}

// -------------------------------------------------------------- host helpers

double *slotp(real **d_wmod, int order) { return *d_wmod + (size_t)order * NVAR * S.g.N; }

// device maxima: clear n slots, run, read back as doubles (0 when none > 0)
int max_begin(int n) {
  CUCK(cudaMemset(S.d_max, 0, sizeof(unsigned long long) * n));
  return SMAUG_OK;
}
int max_end(int n, double *out) {
  unsigned long long h[4] = {0, 0, 0, 0};
  CUCK(cudaMemcpy(h, S.d_max, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost));
  for (int k = 0; k < n; ++k) std::memcpy(&out[k], &h[k], sizeof(double));
  return SMAUG_OK;
}

long long ref_ndimp(long long dimp) {  // computedervfields.cu:1940-1950
  double fn, fractn, in;
  fn = log((double)dimp) / log(2.0);
  fractn = modf(fn, &in);
  if (fractn > 0) {
    fn += 1;
    return (long long)(int)pow(2, fn);
  }
  return dimp;
}

int field_ok(int f, int lo, int hi) {
  if (f < lo || f > hi) return fail(SMAUG_ERR_ARG, "field id out of range for this operator");
  return SMAUG_OK;
}
int dim_ok(int d) {
  if (d < 0 || d >= kD) return fail(SMAUG_ERR_ARG, "direction out of range");
  return SMAUG_OK;
}

}  // namespace

extern "C" {

const char *smaug_cu_last_error(void) { return S.err.c_str(); }

int cuinit(struct params **p, struct bparams **bp, real **wmod, real **wnew, real **wd, struct state **state,
           struct params **d_p, struct bparams **d_bp, real **d_wnew, real **d_wmod, real **d_dwn1, real **d_wd,
           struct state **d_state, real **d_wtemp, real **d_wtemp1, real **d_wtemp2) {
  (void)wnew;
  (void)d_wnew;
  if (!p || !*p || !wmod || !*wmod || !wd || !*wd || !state || !*state || !d_p || !d_bp || !d_wmod || !d_dwn1 ||
      !d_wd || !d_state || !d_wtemp || !d_wtemp1 || !d_wtemp2)
    return fail(SMAUG_ERR_ARG, "cuinit: null argument");
  const struct params *P = *p;
  Grid g{};
  g.N = 1;
  long long n1 = 1, n2 = 1;  // cells of the +1 and +2 padded temporaries
  for (int d = 0; d < 3; ++d) {
    g.n[d] = d < kD ? P->n[d] : 1;
    if (d < kD && (g.n[d] < 6 || g.n[d] > (1 << 20))) return fail(SMAUG_ERR_ARG, "cuinit: each n must be 6..2^20");
    g.N *= g.n[d];
    if (d < kD) {
      n1 *= g.n[d] + 1;
      n2 *= g.n[d] + 2;
    }
  }
  g.st[0] = 1;
  g.st[1] = g.n[0];
  g.st[2] = (long long)g.n[0] * g.n[1];
  for (int d = 0; d < 3; ++d) g.bt[d] = d < kD ? P->boundtype[0][d][0] : 0;
  S.g = g;
  S.nslots = P->rkon == 1 ? 6 : 3;
  const size_t N = (size_t)g.N, sl = (size_t)NVAR * N;
  // the reference's allocations (init.cu:903-930)
  CUCK(cudaMalloc((void **)d_wmod, sizeof(real) * S.nslots * sl));
  CUCK(cudaMalloc((void **)d_dwn1, sizeof(real) * sl));
  CUCK(cudaMalloc((void **)d_wd, sizeof(real) * NDERV * N));
  CUCK(cudaMalloc((void **)d_wtemp, sizeof(real) * NTEMP * N));
  CUCK(cudaMalloc((void **)d_wtemp1, sizeof(real) * NTEMP1 * n1));
  CUCK(cudaMalloc((void **)d_wtemp2, sizeof(real) * NTEMP2 * n2));
  CUCK(cudaMalloc((void **)d_bp, sizeof(struct bparams)));
  CUCK(cudaMalloc((void **)d_p, sizeof(struct params)));
  CUCK(cudaMalloc((void **)d_state, sizeof(struct state)));
  CUCK(cudaMemset(*d_wmod, 0, sizeof(real) * S.nslots * sl));
  CUCK(cudaMemset(*d_dwn1, 0, sizeof(real) * sl));
  CUCK(cudaMemset(*d_wtemp, 0, sizeof(real) * NTEMP * N));
  CUCK(cudaMemset(*d_wtemp1, 0, sizeof(real) * NTEMP1 * n1));
  CUCK(cudaMemset(*d_wtemp2, 0, sizeof(real) * NTEMP2 * n2));
  // the host's wmod slots (2, or 4 with rkon), wd, params and state
  CUCK(cudaMemcpy(*d_wmod, *wmod, sizeof(real) * 2 * (1 + (P->rkon == 1)) * sl, cudaMemcpyHostToDevice));
  CUCK(cudaMemcpy(*d_wd, *wd, sizeof(real) * NDERV * N, cudaMemcpyHostToDevice));
  CUCK(cudaMemcpy(*d_p, *p, sizeof(struct params), cudaMemcpyHostToDevice));
  CUCK(cudaMemcpy(*d_state, *state, sizeof(struct state), cudaMemcpyHostToDevice));
  if (bp && *bp) CUCK(cudaMemcpy(*d_bp, *bp, sizeof(struct bparams), cudaMemcpyHostToDevice));
  if (!S.d_max) CUCK(cudaMalloc((void **)&S.d_max, sizeof(unsigned long long) * 4));
  S.maxvisc = P->maxviscoef;
  S.ready = true;
  return SMAUG_OK;
}

int initgrid(struct params **p, struct state **state, real **wd, struct params **d_p, real **d_dwn1, real **d_wd,
             struct state **d_state, real **d_wtemp, real **d_wtemp1, real **d_wtemp2) {
  (void)state;
  (void)d_p;
  (void)d_dwn1;
  (void)d_state;
  (void)d_wtemp;
  (void)d_wtemp1;
  (void)d_wtemp2;
  REQUIRE(ready(p));
  if (!wd || !*wd || !d_wd || !*d_wd) return fail(SMAUG_ERR_ARG, "initgrid: null argument");
  const struct params *P = *p;
  const size_t N = (size_t)S.g.N;
  CUCK(cudaMemcpy(*wd, *d_wd, sizeof(real) * NDERV * N, cudaMemcpyDeviceToHost));
  real *w = *wd;
  if (P->readini == 0) {  // init_parallel's positions (init.cu:128-140): xmin + c dx
    for (size_t i = 0; i < N; ++i) {
      const long long c[3] = {(long long)(i % S.g.n[0]), (long long)((i / S.g.n[0]) % S.g.n[1]),
                              (long long)(i / S.g.st[2])};
      for (int d = 0; d < kD; ++d) w[(pos1 + d) * N + i] = P->xmin[d] + ((double)c[d]) * P->dx[d];
    }
  }
  int n[3] = {S.g.n[0], S.g.n[1], S.g.n[2]};
  double dx[3] = {0, 0, 0};
  for (int d = 0; d < kD; ++d) dx[d] = P->dx[d];
  if (smaug_initgrid(kD, n, w + pos1 * N, dx, w + delx1 * N) != SMAUG_OK)
    return fail(SMAUG_ERR_ARG, std::string("initgrid: ") + smaug_vac_last_error());
  CUCK(cudaMemcpy(*d_wd, *wd, sizeof(real) * NDERV * N, cudaMemcpyHostToDevice));
  return SMAUG_OK;
}

int cuupdate(struct params **p, real **w, real **wmod, real **wtemp2, struct state **state, struct params **d_p,
             real **d_w, real **d_wmod, real **d_wtemp2, struct state **d_state, int step) {
  (void)w;
  (void)wtemp2;
  (void)d_p;
  (void)d_w;
  (void)d_wtemp2;
  REQUIRE(ready(p));
  if (!wmod || !*wmod || !d_wmod || !*d_wmod) return fail(SMAUG_ERR_ARG, "cuupdate: null argument");
  const int every = (*p)->cfgsavefrequency > 0 ? (*p)->cfgsavefrequency : 1;
  if (step % every == 0) {
    CUCK(cudaMemcpy(*wmod, *d_wmod, sizeof(real) * 2 * NVAR * (size_t)S.g.N, cudaMemcpyDeviceToHost));
    if (state && *state && d_state && *d_state)
      CUCK(cudaMemcpy(*state, *d_state, sizeof(struct state), cudaMemcpyDeviceToHost));
  }
  return SMAUG_OK;
}

int cufinish(struct params **p, real **w, real **wnew, struct state **state, struct params **d_p,
             struct bparams **d_bp, real **d_w, real **d_wnew, real **d_wmod, real **d_dwn1, real **d_wd,
             struct state **d_state, real **d_wtemp, real **d_wtemp1, real **d_wtemp2) {
  (void)p;
  (void)w;
  (void)wnew;
  (void)state;
  (void)d_w;
  (void)d_wnew;
  void **bufs[] = {(void **)d_p, (void **)d_bp, (void **)d_wmod, (void **)d_dwn1, (void **)d_wd,
                   (void **)d_state, (void **)d_wtemp, (void **)d_wtemp1, (void **)d_wtemp2};
  for (void **b : bufs)
    if (b && *b) {
      cudaFree(*b);
      *b = nullptr;
    }
  if (S.d_max) cudaFree(S.d_max);
  S.d_max = nullptr;
  S.ready = false;
  return SMAUG_OK;
}

int cusync(struct params **p) {
  (void)p;
  CUCK(cudaDeviceSynchronize());
  return SMAUG_OK;
}

int cuboundary(struct params **p, struct bparams **bp, struct params **d_p, struct bparams **d_bp,
               struct state **d_s, real **d_wmod, int order, int idir, int field) {
  (void)bp;
  (void)d_p;
  (void)d_bp;
  (void)d_s;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(dim_ok(idir));
  REQUIRE(field_ok(field, 0, NVAR - 1));
  const int type = (*p)->boundtype[field][idir][0];
  if (type != 0 && type != 3 && type != 4 && type != 6 && type != 7)
    return fail(SMAUG_ERR_ARG, "cuboundary: boundary type must be 0, 3, 4, 6 or 7 (fixed ghosts: use the fused API)");
  LAUNCH(k_boundary, S.g, slotp(d_wmod, order) + (size_t)field * S.g.N, idir, type);
  return SMAUG_OK;
}

int cuadvance(struct params **p, struct params **d_p, real **d_wmod, real **d_w, int order) {
  (void)d_p;
  (void)d_w;
  REQUIRE(ready(p));
  const int rkon = (*p)->rkon;
  if (rkon == 1 && S.nslots < 6) return fail(SMAUG_ERR_STATE, "cuadvance: rkon = 1 needs the six slots of cuinit");
  const long long sl = (long long)NVAR * S.g.N;
  const int nb = (int)((sl + 255) / 256 < 148 * 16 ? (sl + 255) / 256 : 148 * 16);
  k_advance<<<nb, 256>>>(S.g, *d_wmod, order, rkon);
  CUCK(cudaGetLastError());
  CUCK(cudaDeviceSynchronize());
  return SMAUG_OK;
}

int cucomputedervfields(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order) {
  (void)d_p;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  LAUNCH(k_dervfields, S.g, *d_wmod, *d_wd, order);
  return SMAUG_OK;
}

int cucomputevels(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir) {
  (void)d_p;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(dim_ok(dir));
  LAUNCH(k_vel, S.g, slotp(d_wmod, order), *d_wd, dir);
  return SMAUG_OK;
}

int cucomputept(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir) {
  (void)d_p;
  (void)dir;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  LAUNCH(k_pt, S.g, slotp(d_wmod, order), *d_wd, (*p)->gamma);
  return SMAUG_OK;
}

int cucomputepk(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir) {
  (void)d_p;
  (void)dir;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  LAUNCH(k_pk, S.g, slotp(d_wmod, order), *d_wd, (*p)->gamma);
  return SMAUG_OK;
}

int cucomputepbg(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir) {
  (void)d_p;
  (void)dir;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  LAUNCH(k_pbg, S.g, slotp(d_wmod, order), *d_wd, (*p)->gamma);
  return SMAUG_OK;
}

int cucomputec(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir) {
  (void)d_p;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(dim_ok(dir));
  LAUNCH(k_c, S.g, slotp(d_wmod, order), *d_wd, (*p)->gamma, dir);
  // the reference copies its device params back over the host's here, which
  // restores the running maximum of the hyperviscosity
  (*p)->maxviscoef = S.maxvisc;
  return SMAUG_OK;
}

int cucomputemaxc(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir, real **wd,
                  real **d_wtemp) {
  (void)d_p;
  (void)d_wmod;
  (void)order;
  (void)dir;
  (void)wd;
  (void)d_wtemp;
  REQUIRE(ready(p));
  REQUIRE(max_begin(1));
  LAUNCH(k_max_field, S.g, *d_wd + (size_t)cfast * S.g.N, S.d_max);
  double m = 0;
  REQUIRE(max_end(1, &m));
  (*p)->cmax = m;
  (*p)->maxviscoef = S.maxvisc;
  return SMAUG_OK;
}

int cucomputemaxcourant(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir,
                        real **wd, real **d_wtemp) {
  (void)d_p;
  (void)d_wmod;
  (void)order;
  (void)wd;
  REQUIRE(ready(p));
  REQUIRE(dim_ok(dir));
  REQUIRE(max_begin(1));
  LAUNCH(k_courant, S.g, *d_wd, *d_wtemp, dir, S.d_max);
  double m = 0;
  REQUIRE(max_end(1, &m));
  (*p)->maxcourant = m;  // reset by every call, as the reference's
  return SMAUG_OK;
}

int cugetdtvisc1(struct params **p, struct params **d_p, real **d_wmod, real **wd, real **d_wd, int order,
                 real **d_wtemp, real **d_wtemp1, real **d_wtemp2) {
  (void)d_p;
  (void)d_wmod;
  (void)wd;
  (void)order;
  (void)d_wtemp1;
  (void)d_wtemp2;
  REQUIRE(ready(p));
  const long long K = ((ref_ndimp(S.g.N) + 511) / 512) * 64;
  REQUIRE(max_begin(1 + kD));
  LAUNCH(k_dtvisc, S.g, *d_wd, *d_wtemp, K, (*p)->maxviscoef, S.d_max);
  double m[4] = {0, 0, 0, 0};
  REQUIRE(max_end(1 + kD, m));
  double dtd = 0.0000000001;
  for (int dir = 0; dir < kD; ++dir) {
    double mm = m[0];
    if (m[1 + dir] > mm) mm = m[1 + dir];
    if (mm > dtd) dtd = mm;
    dtd = 0.25 / dtd;
  }
  (*p)->dtdiffvisc = dtd;
  return SMAUG_OK;
}

static int centdiff(struct params **p, real **d_wmod, real **d_wd, int order, int ordero, real dt, int field,
                    int dir) {
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(slot_ok(ordero));
  REQUIRE(dim_ok(dir));
  REQUIRE(field_ok(field, 0, kNW - 1));
  LAUNCH(k_flux, S.g, slotp(d_wmod, order), *d_wd, field, dir);
  LAUNCH(k_divflux, S.g, slotp(d_wmod, ordero), *d_wd, dt, field, dir);
  return SMAUG_OK;
}

int cucentdiff1(struct params **p, struct params **d_p, struct state **d_s, real **d_w, real **d_wmod,
                real **d_dwn1, real **d_wd, int order, int ordero, real dt, int field, int dir) {
  (void)d_p;
  (void)d_s;
  (void)d_w;
  (void)d_dwn1;
  return centdiff(p, d_wmod, d_wd, order, ordero, dt, field, dir);
}

int cucentdiff2(struct params **p, struct params **d_p, struct state **d_s, real **d_w, real **d_wmod,
                real **d_dwn1, real **d_wd, int order, int ordero, real dt, int field, int dir) {
  (void)d_p;
  (void)d_s;
  (void)d_w;
  (void)d_dwn1;
  return centdiff(p, d_wmod, d_wd, order, ordero, dt, field, dir);
}

int cugrav(struct params **p, struct params **d_p, struct state **d_s, real **d_w, real **d_wmod, real **d_dwn1,
           real **d_wd, int order, int ordero, real dt) {
  (void)d_p;
  (void)d_s;
  (void)d_w;
  (void)d_dwn1;
  (void)d_wd;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(slot_ok(ordero));
  const real *gg = (*p)->g;
  LAUNCH(k_grav, S.g, slotp(d_wmod, order), slotp(d_wmod, ordero), dt, gg[0], gg[1], kD == 3 ? gg[kD - 1] : 0.0);
  return SMAUG_OK;
}

int cusource(struct params **p, struct params **d_p, struct state **d_s, real **d_w, real **d_wmod, real **d_dwn1,
             real **d_wd, int order, int ordero, real dt) {
  (void)d_p;
  (void)d_s;
  (void)d_w;
  (void)d_wmod;
  (void)d_dwn1;
  (void)d_wd;
  (void)order;
  (void)ordero;
  (void)dt;
  REQUIRE(ready(p));
  return SMAUG_OK;  // the default model's user source adds nothing
}

int cudivb(struct params **p, struct params **d_p, real **d_w, real **d_wmod, real **d_dwn1, real **d_wd, int order,
           int ordero, real dt) {
  (void)d_p;
  (void)d_w;
  (void)d_dwn1;
  (void)d_wd;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(slot_ok(ordero));
  if (kD != 2) return fail(SMAUG_ERR_ARG, "cudivb: 2-D only (the reference's 3-D kernel reads an uninitialised bound)");
  LAUNCH(k_divb, S.g, slotp(d_wmod, order), slotp(d_wmod, ordero), dt, (*p)->dx[0], (*p)->dx[kD - 1]);
  return SMAUG_OK;
}

int cunushk1(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, real **d_wtemp,
             real **d_wtemp1, real **d_wtemp2) {
  (void)d_p;
  (void)d_wmod;
  (void)d_wd;
  (void)order;
  (void)d_wtemp;
  (void)d_wtemp1;
  (void)d_wtemp2;
  REQUIRE(ready(p));
  return SMAUG_OK;  // the reference's shock viscosity stores nothing (nushk1.cu:339-343)
}

int cuhyperdifvisc1ir(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, real **d_wtemp,
                      real **d_wtemp1, real **d_wtemp2, int field, int dim) {
  (void)d_p;
  (void)d_wd;
  (void)d_wtemp1;
  (void)d_wtemp2;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(dim_ok(dim));
  REQUIRE(field_ok(field, 0, kNW - 1));
  LAUNCH(k_hyper_q, S.g, slotp(d_wmod, order), *d_wtemp + (size_t)tmp1 * S.g.N, field);
  return SMAUG_OK;
}

static int hyper_nu(struct params **p, real **d_wd, real **d_wtemp, int field, int dim, int side) {
  REQUIRE(ready(p));
  REQUIRE(dim_ok(dim));
  REQUIRE(field_ok(field, 0, kNW - 1));
  REQUIRE(max_begin(1));
  LAUNCH(k_hyper_nu, S.g, *d_wtemp + (size_t)tmp1 * S.g.N, *d_wd, *d_wd + (size_t)(side ? hdnul : hdnur) * S.g.N,
         dim, (*p)->cmax, (*p)->chyp[field], side, S.d_max);
  double m = 0;
  REQUIRE(max_end(1, &m));
  if (m > S.maxvisc) S.maxvisc = m;
  (*p)->maxviscoef = S.maxvisc;
  return SMAUG_OK;
}

int cuhyperdifvisc1r(struct params **p, struct params **d_p, real **d_wmod, real **wd, real **d_wd, int order,
                     real **d_wtemp, real **d_wtemp1, real **d_wtemp2, int field, int dim) {
  (void)d_p;
  (void)d_wmod;
  (void)wd;
  (void)order;
  (void)d_wtemp1;
  (void)d_wtemp2;
  return hyper_nu(p, d_wd, d_wtemp, field, dim, 0);
}

int cuhyperdifvisc1l(struct params **p, struct params **d_p, real **d_wmod, real **wd, real **d_wd, int order,
                     real **d_wtemp, real **d_wtemp1, real **d_wtemp2, int field, int dim) {
  (void)d_p;
  (void)d_wmod;
  (void)wd;
  (void)order;
  (void)d_wtemp1;
  (void)d_wtemp2;
  return hyper_nu(p, d_wd, d_wtemp, field, dim, 1);
}

int cuhyperdifrhosource1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd,
                         int order, int ordero, real **d_wtemp, int field, int dim, real dt) {
  (void)d_p;
  (void)d_dwn1;
  (void)d_wtemp;
  (void)field;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(slot_ok(ordero));
  REQUIRE(dim_ok(dim));
  LAUNCH(k_hyper_scalar, S.g, slotp(d_wmod, order) + (size_t)kRHO * S.g.N, *d_wd, slotp(d_wmod, ordero), kRHO,
         dim, dt);
  return SMAUG_OK;
}

int cuhyperdifesource1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd, int order,
                       int ordero, real **d_wtemp, int field, int dim, real dt) {
  (void)d_p;
  (void)d_dwn1;
  (void)order;
  (void)field;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(ordero));
  REQUIRE(dim_ok(dim));
  // q = the internal energy that cuhyperdifvisc1ir left in wtemp
  LAUNCH(k_hyper_scalar, S.g, *d_wtemp + (size_t)tmp1 * S.g.N, *d_wd, slotp(d_wmod, ordero), kEN, dim, dt);
  return SMAUG_OK;
}

int cuhyperdifmomsource1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd,
                         int order, int ordero, real **d_wtemp, int field, int dim, int ii, int ii0, real dt) {
  (void)d_p;
  (void)d_dwn1;
  (void)field;
  (void)ii;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(slot_ok(ordero));
  REQUIRE(dim_ok(dim));
  REQUIRE(dim_ok(ii0));
  // v = the velocity that cuhyperdifvisc1ir left in wtemp
  LAUNCH(k_hyper_mom_diag, S.g, slotp(d_wmod, order), *d_wtemp + (size_t)tmp1 * S.g.N, *d_wd,
         slotp(d_wmod, ordero), dim, ii0, dt);
  return SMAUG_OK;
}

int cuhyperdifmomsourcene1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd,
                           int order, int ordero, real **d_wtemp, int field, int dim, int ii, int ii0, real dt) {
  (void)d_p;
  (void)d_dwn1;
  (void)field;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(slot_ok(ordero));
  REQUIRE(dim_ok(dim));
  REQUIRE(dim_ok(ii));
  REQUIRE(dim_ok(ii0));
  const size_t N = (size_t)S.g.N;
  double *t1 = *d_wtemp + (size_t)tmp2 * N, *t2 = *d_wtemp + (size_t)tmp3 * N;
  LAUNCH(k_hyper_mom_off_t, S.g, slotp(d_wmod, order), *d_wtemp + (size_t)tmp1 * N, *d_wd, t1, t2, dim, ii0);
  LAUNCH(k_hyper_off_apply, S.g, t1, t2, *d_wd, slotp(d_wmod, ordero), kM0 + ii0, ii, 1.0, 0, dt);
  return SMAUG_OK;
}

int cuhyperdifbsource1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd, int order,
                       int ordero, real **d_wtemp, int field, int dim, int jj, int ii0, int mm, real sb, real dt) {
  (void)d_p;
  (void)d_dwn1;
  (void)d_wtemp;
  (void)mm;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(slot_ok(ordero));
  REQUIRE(dim_ok(dim));
  REQUIRE(dim_ok(field));
  REQUIRE(dim_ok(jj));
  REQUIRE(dim_ok(ii0));
  LAUNCH(k_hyper_b_diag, S.g, slotp(d_wmod, order), *d_wd, slotp(d_wmod, ordero), field, dim, jj, ii0, sb, dt);
  return SMAUG_OK;
}

int cuhyperdifbsourcene1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd,
                         int order, int ordero, real **d_wtemp, int field, int dim, int jj, int ii0, int mm, real sb,
                         real dt) {
  (void)d_p;
  (void)d_dwn1;
  REQUIRE(ready(p));
  REQUIRE(slot_ok(order));
  REQUIRE(slot_ok(ordero));
  REQUIRE(dim_ok(dim));
  REQUIRE(dim_ok(field));
  REQUIRE(dim_ok(jj));
  REQUIRE(dim_ok(ii0));
  REQUIRE(dim_ok(mm));
  const size_t N = (size_t)S.g.N;
  double *t1 = *d_wtemp + (size_t)tmp2 * N, *t2 = *d_wtemp + (size_t)tmp3 * N;
  LAUNCH(k_hyper_b_off_t, S.g, slotp(d_wmod, order), *d_wd, t1, t2, field, dim, jj);
  LAUNCH(k_hyper_off_apply, S.g, t1, t2, *d_wd, slotp(d_wmod, ordero), kB0 + ii0, mm, sb, 1, dt);
  return SMAUG_OK;
}

}  // extern "C"
