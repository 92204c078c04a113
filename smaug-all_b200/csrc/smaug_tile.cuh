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
#pragma once
#include "smaug_device.cuh"

namespace SMAUG_NS {
using namespace smaug;

template <int D>
struct TileShape;
template <>
struct TileShape<2> {
  static constexpr int TX = 16, TY = 16, TZ = 1;
};
template <>
struct TileShape<3> {
  static constexpr int TX = 8, TY = 8, TZ = 4;
};

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

template <int D>
__device__ __forceinline__ bool in_grid(const Geo &g, const int *c) {
#pragma unroll
  for (int d = 0; d < D; ++d)
    if (c[d] < 0 || c[d] >= g.n[d]) return false;
  return true;
}

// Fluxes along dir with reciprocal arithmetic (the same physical fluxes as
// fluxes_at): rho, momentum, energy, induction.
template <int D>
__device__ __forceinline__ void fluxes_fast(const Cell<D> &c, long long i, int dir, double gam, double *F) {
  using L = Lay<D>;
  const double rho = c.v(L::RHO, i), rt = rho + c.v(L::RHOB, i);
  const double irt = 1.0 / rt;
  double m[D], b[D], bb[D];
#pragma unroll
  for (int k = 0; k < D; ++k) {
    m[k] = c.v(L::M0 + k, i);
    b[k] = c.v(L::B0 + k, i);
    bb[k] = c.v(L::BB0 + k, i);
  }
  const double e = c.v(L::EN, i), eb = c.v(L::EB, i);
  double bbb = 0, b2 = 0, m2 = 0, bbm = 0, bm = 0;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    bbb += b[k] * bb[k];
    b2 += b[k] * b[k];
    m2 += m[k] * m[k];
    bbm += bb[k] * m[k];
    bm += b[k] * m[k];
  }
  const double pt = (gam - 1.0) * (e - 0.5 * m2 * irt) - (gam - 2.0) * (bbb + 0.5 * b2);
  const double md = m[dir], vd = md * irt;
  const double bd = b[dir], bbd = bb[dir];
  F[L::RHO] = md;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    double f = vd * m[k] - (b[k] * bbd + bb[k] * bd) - b[k] * bd;
    if (k == dir) f += pt;
    F[L::M0 + k] = f;
  }
  F[L::EN] = vd * (e + eb) + (md * pt - bd * bbm - bbd * bm - bd * bm) * irt;
#pragma unroll
  for (int k = 0; k < D; ++k)
    F[L::B0 + k] = (k == dir) ? 0.0 : vd * (b[k] + bb[k]) - (bd + bbd) * m[k] * irt;
}

// q values for the hyperviscosity of all fields of one dimension d:
// slot 0 rho, 1 internal energy q_e, 2..2+D-1 velocities, then B_f (f != d).
template <int D>
__device__ __forceinline__ void q_all(const Cell<D> &c, long long i, int d, double *q) {
  using L = Lay<D>;
  const double rho = c.v(L::RHO, i);
  const double irt = 1.0 / (rho + c.v(L::RHOB, i));
  double b2 = 0, m2 = 0;
  q[0] = rho;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    const double m = c.v(L::M0 + k, i), b = c.v(L::B0 + k, i);
    b2 += b * b;
    m2 += m * m;
    q[2 + k] = m * irt;
  }
  q[1] = c.v(L::EN, i) - 0.5 * (b2 + m2 * irt);
  int s = 2 + D;
#pragma unroll
  for (int f = 0; f < D; ++f)
    if (f != d) q[s++] = c.v(L::B0 + f, i);
}

template <int D>
__global__ void __launch_bounds__(256, 2) tile_stage_kernel(StageArgs a, Geo g, Phys p) {
  using L = Lay<D>;
  using S = TileShape<D>;
  constexpr int TX = S::TX, TY = S::TY, TZ = S::TZ, NT = TX * TY * TZ;
  constexpr int NW = L::NW, NB = L::NVAR - NW;
  constexpr int NQ = 2 * D + 1;  // q slots per cell for one dimension
  extern __shared__ double sm[];

  const int t = threadIdx.x;
  const int tc[3] = {t % TX, (t / TX) % TY, D == 3 ? t / (TX * TY) : 0};
  const int org[3] = {2 + (int)blockIdx.x * TX, 2 + (int)blockIdx.y * TY, D == 3 ? 2 + (int)blockIdx.z * TZ : 0};
  int c[3] = {org[0] + tc[0], org[1] + tc[1], org[2] + tc[2]};
  bool active = true;
#pragma unroll
  for (int d = 0; d < D; ++d)
    if (c[d] > g.n[d] - 3) active = false;
  const long long idx = active ? gidx<D>(g, c) : 0;
  const Cell<D> C{a.in, a.bg, g.N};
  const double dt = a.sc->dt;
  const double h = dt / a.hdiv;
  double cm[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d) cm[d] = red_get(a.sc->red[a.red_in], d);
  int tile_ext[3] = {TX, TY, D == 3 ? TZ : 1};
  double idx1[3] = {0, 0, 0}, dxc[3] = {1, 1, 1};
  if (active) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      dxc[d] = __ldg(g.dx1[d] + c[d]);
      idx1[d] = 1.0 / dxc[d];
    }
  }
  double dL[NW];
#pragma unroll
  for (int f = 0; f < NW; ++f) dL[f] = 0.0;
  double numax = 0.0;

  // ------------------------------------------------ flux divergences
#pragma unroll 1
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
      double F[NW];
      if (in_grid<D>(g, cc)) {
        fluxes_fast<D>(C, gidx<D>(g, cc), dir, p.gamma, F);
      } else {
#pragma unroll
        for (int f = 0; f < NW; ++f) F[f] = 0.0;
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
      const double w12 = idx1[dir] * (1.0 / 12.0);
#pragma unroll
      for (int f = 0; f < NW; ++f) {
        const double *Fp = sm + f * nbox + r0;
        double gr = (8.0 * (Fp[st] - Fp[-st]) - (Fp[2 * st] - Fp[-2 * st])) * w12;
        if (!zr) dL[f] -= gr;
      }
    }
    __syncthreads();
  }

  // ------------------------------------------------ gravity
  if (active && p.has_grav) {
    const double rho = C.v(L::RHO, idx), irt = 1.0 / (rho + C.v(L::RHOB, idx));
#pragma unroll
    for (int k = 0; k < D; ++k) {
      dL[L::M0 + k] += p.g[k] * rho;
      dL[L::EN] += rho * p.g[k] * C.v(L::M0 + k, idx) * irt;
    }
  }

  // ------------------------------------------------ per-dimension hyperdiffusion
#pragma unroll 1
  for (int d = 0; d < D; ++d) {
    if (!p.hyperdif && !p.has_bgb) break;
    // q box: tile widened by 3 along d and 1 across
    TileBox<D> qb;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int w = e >= D ? 0 : (e == d ? 3 : 1);
      qb.lo[e] = org[e] - w;
      qb.ext[e] = tile_ext[e] + 2 * w;
    }
    const int nq = qb.size();
    // nu box: the tile widened by 1 across d (off-diagonal terms need nu there)
    TileBox<D> nb;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int w = (e >= D || e == d) ? 0 : 1;
      nb.lo[e] = org[e] - w;
      nb.ext[e] = tile_ext[e] + 2 * w;
    }
    const int nn = nb.size();
    double *Q = sm;             // [NQ][nq]
    double *NU = sm + NQ * nq;  // [2*NQ][nn]: nu_R, nu_L per q slot
    for (int r = t; r < nq; r += NT) {
      int cc[3];
      qb.at(r, cc);
      double q[NQ];
      const int x = cc[d];
      bool ok = true;
#pragma unroll
      for (int e = 0; e < D; ++e)
        if (e != d && (cc[e] < 0 || cc[e] >= g.n[e])) ok = false;
      if (!ok || x >= g.n[d]) {  // x == n: right pad of the padded q copy (0)
#pragma unroll
        for (int k = 0; k < NQ; ++k) q[k] = 0.0;
      } else {
        int src[3] = {cc[0], cc[1], cc[2]};
        if (x < 0) src[d] = 5;  // left pad: q(-1) = q(5)
        q_all<D>(C, gidx<D>(g, src), d, q);
      }
#pragma unroll
      for (int k = 0; k < NQ; ++k) Q[k * nq + r] = q[k];
    }
    __syncthreads();
    const int sd = d == 0 ? 1 : d == 1 ? qb.ext[0] : qb.ext[0] * qb.ext[1];
    if (p.hyperdif) {
      for (int r = t; r < nn; r += NT) {
        int cc[3];
        nb.at(r, cc);
        bool inner = true;
#pragma unroll
        for (int e = 0; e < D; ++e)
          if (cc[e] < 2 || cc[e] > g.n[e] - 3) inner = false;
        double nr[NQ], nl[NQ];
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
          nr[k] = 0.0;
          nl[k] = 0.0;
        }
        if (inner) {
          const int rq = qb.index(cc);
          const double dxd = __ldg(g.dx1[d] + cc[d]);
#pragma unroll
          for (int k = 0; k < NQ; ++k) {
            const double *qq = Q + k * nq + rq;
            double qv[7];
#pragma unroll
            for (int o = -3; o <= 3; ++o) qv[o + 3] = qq[o * sd];
            double m3r = 0, m1r = 0, m3l = 0, m1l = 0;
#pragma unroll
            for (int s2 = -1; s2 <= 1; ++s2) {
              m3r = fmax(m3r, fabs(3.0 * (qv[s2 + 4] - qv[s2 + 3]) - (qv[s2 + 5] - qv[s2 + 2])));
              m3l = fmax(m3l, fabs(3.0 * (qv[s2 + 3] - qv[s2 + 2]) - (qv[s2 + 4] - qv[s2 + 1])));
            }
#pragma unroll
            for (int s2 = -2; s2 <= 2; ++s2) {
              m1r = fmax(m1r, fabs(qv[s2 + 4] - qv[s2 + 3]));
              m1l = fmax(m1l, fabs(qv[s2 + 3] - qv[s2 + 2]));
            }
            int fid = k == 0 ? L::RHO : k == 1 ? L::EN : k < 2 + D ? L::M0 + (k - 2) : 0;
            if (k >= 2 + D) {
              const int ff = k - (2 + D);
              fid = L::B0 + (ff >= d ? ff + 1 : ff);
            }
            const double kk = dxd * cm[d] * p.chyp[fid];
            nr[k] = m1r > 0 ? kk * m3r / m1r : 0.0;
            nl[k] = m1l > 0 ? kk * m3l / m1l : 0.0;
          }
        }
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
          NU[(2 * k) * nn + r] = nr[k];
          NU[(2 * k + 1) * nn + r] = nl[k];
        }
      }
    }
    __syncthreads();
    if (active) {
      int cc[3] = {c[0], c[1], c[2]};
      const int r0 = qb.index(cc);
      const int n0 = nb.index(cc);
      const long long sg = g.st[d];
      const bool zd = z1(g, c, d);
      const double i1 = idx1[d], i2 = idx1[d] * idx1[d];
      if (p.has_bgb) {  // background energy terms along d (addenergyterms_cd2)
        double bb2 = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) bb2 += C.v(L::BB0 + k, idx) * C.v(L::BB0 + k, idx);
        const double ptb = (p.gamma - 1) * C.v(L::EB, idx) - 0.5 * (p.gamma - 2) * bb2;
        const bool z4d = z4(g, c, d);
#pragma unroll
        for (int dir = 0; dir < D; ++dir) {
          const double *v = Q + (2 + dir) * nq + r0;
          double gv = z4d ? 0.0 : (8.0 * (v[sd] - v[-sd]) - (v[2 * sd] - v[-2 * sd])) * (i1 * (1.0 / 12.0));
          if (d == dir) dL[L::EN] -= ptb * gv;
          dL[L::EN] += C.v(L::BB0 + d, idx) * C.v(L::BB0 + dir, idx) * gv;
        }
      }
      if (p.hyperdif) {
#pragma unroll
        for (int k = 0; k < NQ; ++k) numax = fmax(numax, fmax(NU[2 * k * nn + n0], NU[(2 * k + 1) * nn + n0]));
        // rho and internal energy: f += (nu_R dq+ - nu_L dq-) / dx^2
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const double *q = Q + k * nq + r0;
          const double nr = NU[2 * k * nn + n0], nl = NU[(2 * k + 1) * nn + n0];
          const double dp = zd ? 0.0 : q[sd] - q[0], dm = zd ? 0.0 : q[0] - q[-sd];
          dL[k == 0 ? L::RHO : L::EN] += (nr * dp - nl * dm) * i2;
        }
        // momentum
        const double rt0 = C.v(L::RHO, idx) + C.v(L::RHOB, idx);
        const double rtp = C.v(L::RHO, idx + sg) + C.v(L::RHOB, idx + sg);
        const double rtm = C.v(L::RHO, idx - sg) + C.v(L::RHOB, idx - sg);
#pragma unroll
        for (int f = 0; f < D; ++f) {
          const int k = 2 + f;
          const double *v = Q + k * nq + r0;
          const double nr = NU[2 * k * nn + n0], nl = NU[(2 * k + 1) * nn + n0];
          const double dvp = zd ? 0.0 : v[sd] - v[0], dvm = zd ? 0.0 : v[0] - v[-sd];
          const double m0 = C.v(L::M0 + f, idx), mp = C.v(L::M0 + f, idx + sg), mm = C.v(L::M0 + f, idx - sg);
          const double fac = (f == d ? 1.0 : 0.5) * i2;
          dL[L::M0 + f] += ((rt0 + rtp) * nr * dvp - (rt0 + rtm) * nl * dvm) * 0.5 * fac;
          dL[L::EN] += ((m0 + mp) * nr * dvp - (m0 + mm) * nl * dvm) * 0.5 * fac;
          if (f != d) {  // off-diagonal: m_d += d_f( rho_t (nu_R+nu_L)/4 d_d v_f )
            const int sf = f == 0 ? 1 : f == 1 ? qb.ext[0] : qb.ext[0] * qb.ext[1];
            const int nf = f == 0 ? 1 : f == 1 ? nb.ext[0] : nb.ext[0] * nb.ext[1];
            const long long gf = g.st[f];
            double t1[2], t2[2];
#pragma unroll
            for (int s = 0; s < 2; ++s) {
              const int o = s ? sf : -sf;
              const int on = s ? nf : -nf;
              const long long go = s ? gf : -gf;
              int cx[3] = {c[0], c[1], c[2]};
              cx[f] += s ? 1 : -1;
              const double nsum = NU[2 * k * nn + n0 + on] + NU[(2 * k + 1) * nn + n0 + on];
              const double tmp5 = z1(g, cx, d) ? 0.0 : (v[o + sd] - v[o - sd]) * 0.5 * i1;
              const double tmp6 = tmp5 * nsum * 0.25;
              t1[s] = (C.v(L::RHO, idx + go) + C.v(L::RHOB, idx + go)) * tmp6;
              t2[s] = tmp6 * C.v(L::M0 + d, idx + go);
            }
            const bool zf = z1(g, c, f);
            const double hf = 0.5 * idx1[f];
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
          const double *b = Q + k * nq + r0;
          const double nr = NU[2 * k * nn + n0], nl = NU[(2 * k + 1) * nn + n0];
          {  // off-diagonal: B_d -= d_f( (nu_L+nu_R)/2 d_d B_f ), e likewise with B_d
            const int sf = f == 0 ? 1 : f == 1 ? qb.ext[0] : qb.ext[0] * qb.ext[1];
            const int nf = f == 0 ? 1 : f == 1 ? nb.ext[0] : nb.ext[0] * nb.ext[1];
            const long long gf = g.st[f];
            double t1[2], t2[2];
#pragma unroll
            for (int s = 0; s < 2; ++s) {
              const int o = s ? sf : -sf;
              const int on = s ? nf : -nf;
              const long long go = s ? gf : -gf;
              int cx[3] = {c[0], c[1], c[2]};
              cx[f] += s ? 1 : -1;
              const double nsum = NU[2 * k * nn + n0 + on] + NU[(2 * k + 1) * nn + n0 + on];
              const double tmp2 = z1(g, cx, d) ? 0.0 : (b[o + sd] - b[o - sd]) * 0.5 * i1;
              t1[s] = tmp2 * nsum * 0.5;
              t2[s] = t1[s] * C.v(L::B0 + d, idx + go);
            }
            if (!z1(g, c, f)) {
              const double hf = 0.5 * idx1[f];
              dL[L::B0 + d] -= (t1[1] - t1[0]) * hf;
              dL[L::EN] -= (t2[1] - t2[0]) * hf;
            }
          }
          {  // diagonal: B_f += (nu_R dB+ - nu_L dB-)/dx^2 and Ohmic heating
            const double dbp = zd ? 0.0 : b[sd] - b[0], dbm = zd ? 0.0 : b[0] - b[-sd];
            dL[L::B0 + f] += (nr * dbp - nl * dbm) * i2;
            dL[L::EN] += (0.5 * (b[0] + b[sd]) * nr * dbp - 0.5 * (b[0] + b[-sd]) * nl * dbm) * i2;
          }
        }
      }
    }
    __syncthreads();
  }

  // ------------------------------------------------ combine, write, reduce
  double red[6] = {0, 0, 0, 0, 0, numax};
  if (active) {
    double o[NW];
#pragma unroll
    for (int f = 0; f < NW; ++f) o[f] = a.base[(long long)f * g.N + idx] + h * dL[f];
    if (a.kind == 3) {
#pragma unroll
      for (int f = 0; f < NW; ++f) {
        const long long j = (long long)f * g.N + idx;
        a.acc[j] = (a.acc[j] + 2.0 * C.v(f, idx) + o[f] - 4.0 * a.base[j]) * (1.0 / 3.0);
      }
    } else if (a.kind == 4) {
#pragma unroll
      for (int f = 0; f < NW; ++f) o[f] += a.acc[(long long)f * g.N + idx];
    }
    int xs[3][2], nx[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (d < D)
        nx[d] = images(g, d, c[d], xs[d]);
      else {
        nx[d] = 1;
        xs[d][0] = 0;
      }
    }
    for (int iz = 0; iz < nx[2]; ++iz)
      for (int iy = 0; iy < nx[1]; ++iy)
        for (int ix = 0; ix < nx[0]; ++ix) {
          const long long j = xs[0][ix] + (long long)xs[1][iy] * g.st[1] + (D == 3 ? (long long)xs[2][iz] * g.st[2] : 0);
#pragma unroll
          for (int f = 0; f < NW; ++f) a.out[(long long)f * g.N + j] = o[f];
          double bgv[NB];
#pragma unroll
          for (int b = 0; b < NB; ++b) bgv[b] = __ldg(a.bg + (long long)b * g.N + j);
          reduce_cell<D>(g, p, o, bgv, j, red);
        }
  }
  block_max_flush<6>(red, &a.sc->red[a.red_out]);
}

// shared memory bytes the tile kernel needs
template <int D>
__host__ __device__ constexpr int tile_smem_doubles() {
  using S = TileShape<D>;
  constexpr int NW = 2 + 2 * D, NQ = 2 * D + 1;
  constexpr int ex[3] = {S::TX, S::TY, D == 3 ? S::TZ : 1};
  // flux box, largest over dir
  int fl = 0, qv = 0;
  for (int dir = 0; dir < D; ++dir) {
    int n = 1, m = 1, u = 1;
    for (int e = 0; e < D; ++e) {
      n *= ex[e] + (e == dir ? 4 : 0);
      m *= ex[e] + (e == dir ? 6 : 2);
      u *= ex[e] + (e == dir ? 0 : 2);
    }
    fl = fl > NW * n ? fl : NW * n;
    qv = qv > NQ * m + 2 * NQ * u ? qv : NQ * m + 2 * NQ * u;
  }
  return fl > qv ? fl : qv;
}

}  // namespace SMAUG_NS
