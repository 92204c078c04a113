// smaug_stage.cuh -- the fused per-stage kernel and the reductions.
//
// Included by stage_exact.cu (compiled with -fmad=false: bit-reproducible
// against the CPU oracle) and stage_fast.cu (FMA contraction on); each
// instantiates the templates in its own namespace SMAUG_NS.
#pragma once
#include "smaug_device.cuh"

namespace SMAUG_NS {
using namespace smaug;

constexpr int kBX = 32, kBY = 4;

// Zero rules of the reference gradients near non-periodic edges, at inner
// cells (gradops.cu:437-826): 4th-order within two cells, 1st/2nd-order at
// the first and last inner cell.
__device__ __forceinline__ bool z4(const Geo &g, const int *c, int d) {
  return g.btype[d] != 0 && (c[d] == 2 || c[d] == 3 || c[d] == g.n[d] - 4 || c[d] == g.n[d] - 3);
}
__device__ __forceinline__ bool z1(const Geo &g, const int *c, int d) {
  return g.btype[d] != 0 && (c[d] == 2 || c[d] == g.n[d] - 3);
}

template <int D>
__device__ __forceinline__ bool inner_at(const Geo &g, const int *c) {
#pragma unroll
  for (int d = 0; d < D; ++d)
    if (c[d] < 2 || c[d] > g.n[d] - 3) return false;
  return true;
}

// grad3d_MODID (gradops.cu:132-237, 2-D branch): 4th-order difference of
// field f along dir over the uniform spacing p->dx, zero at the first and
// last two inner cells whatever the boundary type (its tests read
// `x==2 || x==3 && ...`, the second part true at every inner cell).
template <int D>
__device__ __forceinline__ double grad3d_at(const Cell<D> &C, const Geo &g, const Phys &p, long long idx, const int *c,
                                            int f, int dir) {
  const int n = g.n[dir], x = c[dir], o = 1 - dir;
  const long long s = g.st[dir];
  double grad = 0;
  if (x > 1 && x < n - 2)
    grad = (((8 * C.v(f, idx + s) - 8 * C.v(f, idx - s) + C.v(f, idx - 2 * s) - C.v(f, idx + 2 * s)) / 6.0)) /
           (2.0 * (p.dxs[dir]));
  const bool in_o = c[o] > 1 && c[o] < g.n[o] - 2;
  if ((x == n - 3) || (x == n - 4 && in_o))
    grad = 0;
  else if (x == 2 || (x == 3 && in_o))
    grad = 0;
  return grad;
}

// Block-wide max of v[0..5] then one atomic per value into r.
template <int NV>
__device__ __forceinline__ void block_max_flush(double *v, Reduce *r) {
  __shared__ double sm[NV][32];
  const int lane = (threadIdx.x + threadIdx.y * blockDim.x + threadIdx.z * blockDim.x * blockDim.y) & 31;
  const int warp = (threadIdx.x + threadIdx.y * blockDim.x + threadIdx.z * blockDim.x * blockDim.y) >> 5;
  const int nwarp = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double y = __shfl_xor_sync(0xffffffffu, x, o);
      x = (y > x || y != y) ? y : x;
    }
    if (lane == 0) sm[k][warp] = x;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = lane < nwarp ? sm[k][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        double y = __shfl_xor_sync(0xffffffffu, x, o);
        x = (y > x || y != y) ? y : x;
      }
      if (lane == 0 && x != 0.0) atomic_max_nonneg(&r->v[k], x);
    }
  }
}

// The same for FP32 running maxima (widened exactly to FP64).
template <int NV>
__device__ __forceinline__ void block_max_flush(const float *v, Reduce *r) {
  double w[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) w[k] = (double)v[k];
  block_max_flush<NV>(w, r);
}

// Coordinates along d that take the value of inner coordinate x once the
// ghosts are filled (the per-direction rules above, applied in direction
// order): xs[0] = x itself, then its ghost images (cont gives two); *neg =
// the evolved fields the images take negated.  A fixed direction has no
// images (its ghosts keep their loaded values), and where a later direction
// is fixed the outermost layer is restored by that pass, so it is no image
// either.  Returns the count (1..3).
template <int D>
__device__ __forceinline__ int images(const Geo &g, int d, int x, int *xs, unsigned *neg) {
  // (fixed slots, no runtime index: the arrays stay in registers)
  const int n = g.n[d];
  int k = 1, e1 = 0, e2 = 0;
  switch (g.btype[d]) {
    case BC_PERIODIC:
      if (x == n - 4 || x == n - 3) {
        e1 = x - (n - 4);
        k = 2;
      } else if (x == 2 || x == 3) {
        e1 = x + (n - 4);
        k = 2;
      }
      break;
    case BC_CONT:
      if (x == 2) {
        e1 = 0;
        e2 = 1;
        k = 3;
      } else if (x == n - 3) {
        e1 = n - 1;
        e2 = n - 2;
        k = 3;
      }
      break;
    case BC_SYMM:
    case BC_ASYMM:
      if (D == 2) {
        k = 2;
        if (x == 3) e1 = 0;
        else if (x == 2) e1 = 1;
        else if (x == n - 4) e1 = n - 1;
        else if (x == n - 3) e1 = n - 2;
        else k = 1;
        break;
      }
      // fall through: the 3-D mirror is contcd4's
    case BC_CONTCD4:
      k = 2;
      if (x == 4) e1 = 0;
      else if (x == 3) e1 = 1;
      else if (x == n - 5) e1 = n - 1;
      else if (x == n - 4) e1 = n - 2;
      else k = 1;
      break;
    default:
      break;
  }
  if (g.outer_frozen[d] && k > 1 && (e1 == 0 || e1 == n - 1)) {  // drop images 0 and n-1
    e1 = e2;
    k -= 1;
  }
  xs[0] = x;
  xs[1] = e1;
  xs[2] = e2;
  *neg = bc_neg(g, d);
  return k;
}

// cfast/courant maxima of the state `o` written at cell idx (with that cell's
// background values).
template <int D>
__device__ __forceinline__ void reduce_cell(const Geo &g, const Phys &p, const double *o, const double *bgv,
                                            long long idx, double *r) {
#pragma unroll
  for (int d = 0; d < D; ++d) {
    double cf = cfast_vals<D>(o, bgv, d, p.gamma);
    if (cf > r[d] || cf != cf) r[d] = cf;
    if (d == D - 1) {
      double cour = cf / (__ldg(g.dxlast + idx));
      if (cour > r[3] || cour != cour) r[3] = cour;
      if (idx >= g.K && (cour > r[4] || cour != cour)) r[4] = cour;
    }
  }
}

template <int D>
__global__ void __launch_bounds__(kBX *kBY) stage_kernel(StageArgs a, Geo g, Phys p) {
  using L = Lay<D>;
  constexpr int NW = L::NW;
  constexpr int NB = L::NVAR - NW;
  const int cx = blockIdx.x * blockDim.x + threadIdx.x;
  const int cy = blockIdx.y * blockDim.y + threadIdx.y;
  const int cz = blockIdx.z;
  const bool active = cx < g.n[0] - 4 && cy < g.n[1] - 4 && (D == 2 || cz < g.n[2] - 4);
  double red[6] = {0, 0, 0, 0, 0, 0};
  if (active) {
    int c[3] = {cx + 2, cy + 2, D == 3 ? cz + 2 : 0};
    const long long N = g.N;
    const long long idx = c[0] + (long long)c[1] * g.st[1] + (D == 3 ? (long long)c[2] * g.st[2] : 0);
    const Cell<D> C{a.in, a.bg, N};
    const double dt = a.sc->dt;
    const double h = dt / a.hdiv;
    double cm[3];
#pragma unroll
    for (int d = 0; d < D; ++d) cm[d] = red_get(a.sc->red[a.red_in], d);
    double dxc[3];
#pragma unroll
    for (int d = 0; d < D; ++d) dxc[d] = __ldg(g.dx1[d] + c[d]);
    double o[NW];
#pragma unroll
    for (int f = 0; f < NW; ++f) o[f] = a.base[(long long)f * N + idx];

    // ---- flux divergences (centdiff1.cu / centdiff2.cu), per direction
#pragma unroll 1
    for (int dir = 0; dir < D; ++dir) {
      const long long s = g.st[dir];
      double acc[NW], F[NW];
      fluxes_at<D>(C, idx + s, dir, p.gamma, F);
#pragma unroll
      for (int f = 0; f < NW; ++f) acc[f] = 8 * F[f];
      fluxes_at<D>(C, idx - s, dir, p.gamma, F);
#pragma unroll
      for (int f = 0; f < NW; ++f) acc[f] = acc[f] - 8 * F[f];
      fluxes_at<D>(C, idx - 2 * s, dir, p.gamma, F);
#pragma unroll
      for (int f = 0; f < NW; ++f) acc[f] = acc[f] + F[f];
      fluxes_at<D>(C, idx + 2 * s, dir, p.gamma, F);
      const bool zr = z4(g, c, dir);
#pragma unroll
      for (int f = 0; f < NW; ++f) {
        double gr = ((acc[f] - F[f]) / 6.0) / (2.0 * (dxc[dir]));
        o[f] = o[f] - h * (zr ? 0.0 : gr);
      }
      if (p.has_bgb) {  // addenergyterms_cd2, centdiff2.cu:80-115
        double bb2 = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) bb2 += C.v(L::BB0 + k, idx) * C.v(L::BB0 + k, idx);
        const double ptb = ((p.gamma) - 1) * C.v(L::EB, idx) - 0.5 * ((p.gamma) - 2) * (bb2);
        double gv[3];
#pragma unroll
        for (int idim = 0; idim < D; ++idim) {
          const long long t = g.st[idim];
          double vp1 = C.v(L::M0 + dir, idx + t) / (C.v(L::RHO, idx + t) + C.v(L::RHOB, idx + t));
          double vm1 = C.v(L::M0 + dir, idx - t) / (C.v(L::RHO, idx - t) + C.v(L::RHOB, idx - t));
          double vm2 = C.v(L::M0 + dir, idx - 2 * t) / (C.v(L::RHO, idx - 2 * t) + C.v(L::RHOB, idx - 2 * t));
          double vp2 = C.v(L::M0 + dir, idx + 2 * t) / (C.v(L::RHO, idx + 2 * t) + C.v(L::RHOB, idx + 2 * t));
          gv[idim] = d4(vm2, vm1, vp1, vp2, dxc[idim], z4(g, c, idim));
        }
        o[L::EN] -= +(h)*ptb * gv[dir];
#pragma unroll
        for (int idim = 0; idim < D; idim++)
          o[L::EN] += (h)*C.v(L::BB0 + idim, idx) * C.v(L::BB0 + dir, idx) * gv[idim];
      }
    }

    // ---- gravity, addgrav_cd2 centdiff2.cu:118-150
    if (p.has_grav) {
#pragma unroll
      for (int k = 0; k < D; ++k) o[L::M0 + k] += (h) * (p.g[k]) * C.v(L::RHO, idx);
#pragma unroll
      for (int k = 0; k < D; ++k)
        o[L::EN] += (h)*C.v(L::RHO, idx) * ((p.g[k]) * C.v(L::M0 + k, idx)) / (C.v(L::RHO, idx) + C.v(L::RHOB, idx));
    }

    // ---- divergence of B (cudivb, divb.cu:165-336; iosmaug.cpp:962-963), 2-D:
    // divB at cells 3..n-3, sources -divB (0, B, B.v, v), w -= dt * source
    if (D == 2 && p.divb && c[0] > 2 && c[1] > 2) {
      double divb = grad3d_at<D>(C, g, p, idx, c, L::B0, 0) + grad3d_at<D>(C, g, p, idx, c, L::B0 + 1, 1);
      divb += grad3d_at<D>(C, g, p, idx, c, L::BB0, 0) + grad3d_at<D>(C, g, p, idx, c, L::BB0 + 1, 1);
      const double bdotv = ((C.v(L::B0, idx) + C.v(L::BB0, idx)) * C.v(L::M0, idx) +
                            (C.v(L::B0 + 1, idx) + C.v(L::BB0 + 1, idx)) * C.v(L::M0 + 1, idx)) /
                           (C.v(L::RHO, idx) + C.v(L::RHOB, idx));
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const double sm = -divb * C.v(L::B0 + k, idx);
        o[L::M0 + k] = o[L::M0 + k] - h * (0.0 + (isnan(sm) ? 0 : sm));
        const double sb = -divb * C.v(L::M0 + k, idx) / (C.v(L::RHO, idx) + C.v(L::RHOB, idx));
        o[L::B0 + k] = o[L::B0 + k] - h * (0.0 + (isnan(sb) ? 0 : sb));
      }
      o[L::EN] = o[L::EN] - h * (0.0 + (-divb * bdotv));
    }

    if (p.hyperdif) {
      double nur, nul;
      // ---- density (hyperdifrhosource1.cu:15-282)
#pragma unroll 1
      for (int d = 0; d < D; ++d) {
        visc_at<D, Q_RHO>(C, g, idx, c[d], d, 0, cm[d], p.chyp[L::RHO], dxc[d], nur, nul);
        red[5] = fmax(red[5], fmax(nur, nul));
        const long long s = g.st[d];
        const double r0 = C.v(L::RHO, idx);
        double tp = z1(g, c, d) ? 0.0 : ((C.v(L::RHO, idx + s) - r0) / ((dxc[d])));
        double tm = z1(g, c, d) ? 0.0 : ((r0 - C.v(L::RHO, idx - s)) / ((dxc[d])));
        o[L::RHO] = o[L::RHO] + h * ((nur)*tp - (nul)*tm) / dxc[d];
      }
      // ---- energy (hyperdifesource1.cu:18-554), q = e - (B^2 + m^2/rho_t)/2
#pragma unroll 1
      for (int d = 0; d < D; ++d) {
        visc_at<D, Q_EN>(C, g, idx, c[d], d, 0, cm[d], p.chyp[L::EN], dxc[d], nur, nul);
        red[5] = fmax(red[5], fmax(nur, nul));
        const long long s = g.st[d];
        const double q0 = q_at<D, Q_EN>(C, idx, 0);
        double tm = z1(g, c, d) ? 0.0 : ((q0 - q_at<D, Q_EN>(C, idx - s, 0)) / ((dxc[d])));
        double tp = z1(g, c, d) ? 0.0 : ((q_at<D, Q_EN>(C, idx + s, 0) - q0) / ((dxc[d])));
        o[L::EN] = o[L::EN] + h * ((nur)*tp - (nul)*tm) / dxc[d];
      }
      // ---- momentum (hyperdifmomsource1.cu, hyperdifmomsourcene1.cu)
#pragma unroll 1
      for (int d = 0; d < D; ++d)
#pragma unroll 1
        for (int f = 0; f < D; ++f) {
          visc_at<D, Q_VEL>(C, g, idx, c[d], d, f, cm[d], p.chyp[L::M0 + f], dxc[d], nur, nul);
          red[5] = fmax(red[5], fmax(nur, nul));
          const long long s = g.st[d];
          // diagonal term (ii0 = f), applied twice when f == d
          {
            const double rho0 = C.v(L::RHO, idx), rb0 = C.v(L::RHOB, idx);
            double tmp2 = (rho0 + rb0 + C.v(L::RHO, idx - s) + C.v(L::RHOB, idx - s)) / 2;
            double tmp3 = (rho0 + rb0 + C.v(L::RHO, idx + s) + C.v(L::RHOB, idx + s)) / 2;
            const double m0 = C.v(L::M0 + f, idx);
            double tmp5 = (m0 + C.v(L::M0 + f, idx - s)) / 2;
            double tmp6 = (m0 + C.v(L::M0 + f, idx + s)) / 2;
            const double v0 = q_at<D, Q_VEL>(C, idx, f);
            double tmp8 = z1(g, c, d) ? 0.0 : ((q_at<D, Q_VEL>(C, idx + s, f) - v0) / ((dxc[d])));
            double tmp7 = z1(g, c, d) ? 0.0 : ((v0 - q_at<D, Q_VEL>(C, idx - s, f)) / ((dxc[d])));
            double dm = (tmp3 * (nur)*tmp8 - tmp2 * (nul)*tmp7) / (dxc[d]) / 2;
            double de = (tmp6 * (nur)*tmp8 - tmp5 * (nul)*tmp7) / (dxc[d]) / 2;
            o[L::M0 + f] = o[L::M0 + f] + h * dm;
            o[L::EN] = o[L::EN] + h * de;
            if (f == d) {
              o[L::M0 + f] = o[L::M0 + f] + h * dm;
              o[L::EN] = o[L::EN] + h * de;
            }
          }
          if (f != d) {  // off-diagonal term (ii = f, ii0 = d)
            const long long t = g.st[f];
            double t1[2], t2[2];
#pragma unroll
            for (int sg = 0; sg < 2; ++sg) {
              const long long x = idx + (sg ? t : -t);
              int cxx[3] = {c[0], c[1], c[2]};
              cxx[f] += sg ? 1 : -1;
              t1[sg] = 0.0;
              t2[sg] = 0.0;
              if (inner_at<D>(g, cxx)) {
                double nrx, nlx;
                visc_at<D, Q_VEL>(C, g, x, cxx[d], d, f, cm[d], p.chyp[L::M0 + f], dxc[d], nrx, nlx);
                double tmp5 = z1(g, cxx, d) ? 0.0
                                            : ((q_at<D, Q_VEL>(C, x + s, f) - q_at<D, Q_VEL>(C, x - s, f)) /
                                               ((dxc[d])) / 2.0);
                double tmp6 = tmp5 * ((nrx + nlx + 2.0 * 0.0)) / 4.0;
                t1[sg] = (C.v(L::RHO, x) + C.v(L::RHOB, x)) * tmp6;
                t2[sg] = tmp6 * C.v(L::M0 + d, x);
              }
            }
            const bool zf = z1(g, c, f);
            double dm = zf ? 0.0 : ((t1[1] - t1[0]) / ((dxc[f])) / 2.0);
            o[L::M0 + d] = o[L::M0 + d] + h * dm;
            double de = zf ? 0.0 : ((t2[1] - t2[0]) / ((dxc[f])) / 2.0);
            o[L::EN] = o[L::EN] + h * de;
          }
        }
      // ---- magnetic field (hyperdifbsource1.cu, hyperdifbsourcene1.cu)
#pragma unroll 1
      for (int d = 0; d < D; ++d)
#pragma unroll 1
        for (int f = 0; f < D; ++f) {
          if (f == d) continue;
          visc_at<D, Q_B>(C, g, idx, c[d], d, f, cm[d], p.chyp[L::B0 + f], dxc[d], nur, nul);
          red[5] = fmax(red[5], fmax(nur, nul));
          const long long s = g.st[d];
          {  // off-diagonal (jj = d, mm = f, ii0 = d, sb = -1)
            const double sb = -1.0;
            const long long t = g.st[f];
            double t1[2], t2[2];
#pragma unroll
            for (int sg = 0; sg < 2; ++sg) {
              const long long x = idx + (sg ? t : -t);
              int cxx[3] = {c[0], c[1], c[2]};
              cxx[f] += sg ? 1 : -1;
              t1[sg] = 0.0;
              t2[sg] = 0.0;
              if (inner_at<D>(g, cxx)) {
                double nrx, nlx;
                visc_at<D, Q_B>(C, g, x, cxx[d], d, f, cm[d], p.chyp[L::B0 + f], dxc[d], nrx, nlx);
                double tmp2 = z1(g, cxx, d)
                                  ? 0.0
                                  : ((C.v(L::B0 + f, x + s) - C.v(L::B0 + f, x - s)) / ((dxc[d])) / 2.0);
                t1[sg] = tmp2 * (nlx + nrx) / 2;
                t2[sg] = t1[sg] * C.v(L::B0 + d, x);
              }
            }
            const bool zf = z1(g, c, f);
            double db = sb * (zf ? 0.0 : ((t1[1] - t1[0]) / ((dxc[f])) / 2.0));
            o[L::B0 + d] = o[L::B0 + d] + h * db;
            double de = sb * (zf ? 0.0 : ((t2[1] - t2[0]) / ((dxc[f])) / 2.0));
            o[L::EN] = o[L::EN] + h * de;
          }
          {  // diagonal (jj = f, ii0 = f, sb = +1)
            const double sb = 1.0;
            const double b0 = C.v(L::B0 + f, idx), bm = C.v(L::B0 + f, idx - s), bp = C.v(L::B0 + f, idx + s);
            double tmp2 = (b0 + bm) / 2;
            double tmp3 = (b0 + bp) / 2;
            double tmp4 = z1(g, c, d) ? 0.0 : ((b0 - bm) / ((dxc[d])));
            double tmp5 = z1(g, c, d) ? 0.0 : ((bp - b0) / ((dxc[d])));
            double db = sb * (tmp5 * nur - tmp4 * nul) / dxc[d];
            double de = sb * (tmp3 * tmp5 * nur - tmp2 * tmp4 * nul) / dxc[d];
            o[L::B0 + f] = o[L::B0 + f] + h * db;
            o[L::EN] = o[L::EN] + h * de;
          }
        }
    }

    // ---- momentum driver on the stage output (usersource.cu.spicule1:4-137)
    if (p.drv_on) {
      const double vvz = driver_vvz<D>(g, p, a.sc, a.tfrac, c);
      const double rb = __ldg(a.bg + (long long)(L::RHOB - NW) * N + idx);
#pragma unroll
      for (int k = 0; k < D; ++k)
        if (k == p.drv_dir) o[L::M0 + k] = o[L::M0 + k] + h * vvz * (o[L::RHO] + rb);
    }

    // ---- Runge-Kutta combination (vac.t:447-462)
    if (a.kind == 3) {
#pragma unroll
      for (int f = 0; f < NW; ++f) {
        const long long j = (long long)f * N + idx;
        a.acc[j] = (a.acc[j] + 2 * C.v(f, idx) + o[f] - 4 * a.base[j]) / 3;
      }
    } else if (a.kind == 4) {
#pragma unroll
      for (int f = 0; f < NW; ++f) o[f] = o[f] + a.acc[(long long)f * N + idx];
    }

    // ---- write the cell and its ghost images, reduce wave speeds
    int xs[3][3], nx[3];
    unsigned ng[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (d < D)
        nx[d] = images<D>(g, d, c[d], xs[d], &ng[d]);
      else {
        nx[d] = 1;
        xs[d][0] = 0;
        ng[d] = 0;
      }
    }
    for (int iz = 0; iz < nx[2]; ++iz)
      for (int iy = 0; iy < nx[1]; ++iy)
        for (int ix = 0; ix < nx[0]; ++ix) {
          const long long j = xs[0][ix] + (long long)xs[1][iy] * g.st[1] + (D == 3 ? (long long)xs[2][iz] * g.st[2] : 0);
          const unsigned neg = (ix ? ng[0] : 0u) ^ (iy ? ng[1] : 0u) ^ (iz ? ng[2] : 0u);
          double ov[NW];
#pragma unroll
          for (int f = 0; f < NW; ++f) ov[f] = ((neg >> f) & 1u) ? -o[f] : o[f];
#pragma unroll
          for (int f = 0; f < NW; ++f) a.out[(long long)f * N + j] = ov[f];
          double bgv[NB];
#pragma unroll
          for (int b = 0; b < NB; ++b) bgv[b] = __ldg(a.bg + (long long)b * N + j);
          reduce_cell<D>(g, p, ov, bgv, j, red);
        }
  }
  block_max_flush<6>(red, &a.sc->red[a.red_out]);
}

// Maxima over all cells of a state (used once after the state is loaded);
// const_only: over the cells that keep their loaded values only.
template <int D>
__global__ void reduce_state_kernel(const double *w, const double *bg, Geo g, Phys p, Reduce *r, int const_only) {
  using L = Lay<D>;
  constexpr int NW = L::NW, NB = L::NVAR - L::NW;
  double red[6] = {0, 0, 0, 0, 0, 0};
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < g.N; j += (long long)gridDim.x * blockDim.x) {
    if (const_only) {
      const int c[3] = {(int)(j % g.n[0]), (int)((j / g.n[0]) % g.n[1]), (int)(j / g.st[2])};
      if (!is_const_cell<D>(g, c)) continue;
    }
    double o[NW], bgv[NB];
#pragma unroll
    for (int f = 0; f < NW; ++f) o[f] = w[(long long)f * g.N + j];
#pragma unroll
    for (int b = 0; b < NB; ++b) bgv[b] = bg[(long long)b * g.N + j];
    reduce_cell<D>(g, p, o, bgv, j, red);
  }
  block_max_flush<6>(red, r);
}

}  // namespace SMAUG_NS
