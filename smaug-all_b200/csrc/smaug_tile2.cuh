// smaug_tile2.cuh -- the 2-D stage body in three phases.
//
// Same operator as tile_body (smaug_tile.cuh), reorganised for 2-D so that a
// tile needs two block barriers instead of ten and computes every per-cell
// quantity once per tile:
//   phase A  one balanced loop over the union of three boxes: x-fluxes on the
//            tile +-2 along x, y-fluxes on the tile +-2 along y, and the six
//            hyperviscosity inputs q (rho, e_int, v_x, v_y, B_x, B_y) on the
//            tile +-3 in both dimensions;
//   phase B  one loop over runs of cell faces of both dimensions: the ratio
//            max|d3 q| / max|d1 q| of the hyperviscosity once per face
//            (nu_R of a cell and nu_L of its right neighbour share their
//            windows, consecutive faces share their differences), along x on
//            the tile +-1 in y, along y on the tile +-1 in x (the
//            off-diagonal terms need nu there);
//   phase C  per cell: nu = dx c_max c_hyp * ratio on the cell's faces,
//            divergences, gravity, background energy terms, hyperdiffusion,
//            then the shared epilogue.
// A q cell outside the grid along one dimension takes that dimension's pad
// (0 on the right, q(5) on the left, as the reference's padded copies do);
// the corners outside both are never read.
#pragma once
#include <type_traits>

#include "smaug_tile.cuh"

namespace SMAUG_NS {
using namespace smaug;

// The q slots of one cell (2-D): the hyperviscosity inputs, slot 0 rho,
// 1 internal energy (FP64), 2 v_x, 3 v_y, 4 B_x, 5 B_y; then what the
// momentum terms read at the neighbours: 6 rho_t = rho + rho_b, 7 m_x, 8 m_y.
template <typename T>
__device__ __forceinline__ void q_cell(const CellT<2, T> &c, long long i, T *q) {
  using L = Lay<2>;
  const T rho = c.v(L::RHO, i);
  const double rhob = c.vd(L::RHOB, i);
  const double irtd = 1.0 / ((double)rho + rhob);
  const T irt = (T)irtd;
  const T m0 = c.v(L::M0, i), m1 = c.v(L::M0 + 1, i), b0 = c.v(L::B0, i), b1 = c.v(L::B0 + 1, i);
  const double b2 = (double)b0 * (double)b0 + (double)b1 * (double)b1;
  const double m2 = (double)m0 * (double)m0 + (double)m1 * (double)m1;
  q[0] = rho;
  q[1] = (T)(c.vd(L::EN, i) - 0.5 * (b2 + m2 * irtd));
  q[2] = m0 * irt;
  q[3] = m1 * irt;
  q[4] = b0;
  q[5] = b1;
  q[6] = rho + (T)rhob;
  q[7] = m0;
  q[8] = m1;
}

// Box sizes of the three-phase body for a TX x TY tile.
template <typename S>
struct Box2 {
  static constexpr int TX = S::TX, TY = S::TY;
  // flux slots: the evolved fields but B_d (its flux along d is zero)
  static constexpr int NF = Lay<2>::NW - 1;
  static constexpr int NQS = 9;  // q slots per cell (q_cell)
  static constexpr int F0X = TX + 4, F0N = F0X * TY;           // x-fluxes: tile +-2 along x
  static constexpr int F1X = TX, F1N = TX * (TY + 4);          // y-fluxes: tile +-2 along y
  static constexpr int QX = TX + 6, QN = QX * (TY + 6);        // q: tile +-3
  // face ratios along x: faces x+1/2 for x in [-1, TX), rows tile +-1
  static constexpr int V0X = TX + 1, V0N = (TX + 1) * (TY + 2);
  // face ratios along y: faces y+1/2 for y in [-1, TY), columns tile +-1
  static constexpr int V1X = TX + 2, V1N = (TX + 2) * (TY + 1);
  // offsets (elements) of the arrays in shared memory
  static constexpr int OF0 = 0, OF1 = OF0 + NF * F0N, OQ = OF1 + NF * F1N, OV0 = OQ + NQS * QN, OV1 = OV0 + 5 * V0N;
  // flux slot of field f along dir
  static constexpr __host__ __device__ int fslot(int f, int dir) { return f < Lay<2>::B0 + dir ? f : f - 1; }
  static constexpr int ELEMS = OV1 + 5 * V1N;
};

template <typename T, typename S>
__device__ __forceinline__ void tile_body2(const StageArgs &a, const Geo &g, const Phys &p, int bx, int by, T *sm,
                                           T *red) {
  constexpr int D = 2;
  using L = Lay<2>;
  using B = Box2<S>;
  constexpr int TX = S::TX, TY = S::TY, NT = TX * TY;
  constexpr int NW = L::NW;
  constexpr bool MIXED = sizeof(T) == sizeof(float);
  T *F0 = sm + B::OF0, *F1 = sm + B::OF1, *Q = sm + B::OQ, *V0 = sm + B::OV0, *V1 = sm + B::OV1;

  const int t = threadIdx.x;
  const int ox = 2 + bx * TX, oy = 2 + by * TY;
  const int n0 = g.n[0], n1 = g.n[1];
  // the cell of this thread.  With 16-wide tiles a warp takes two rows; they
  // are TY/2 apart rather than adjacent, so that the row offset of the q box
  // (stride TX + 6 = 22) moves the second half-warp by 16 banks: the q reads
  // of phase C are free of bank conflicts.
  constexpr bool PAIRED = TX == 16 && TY == 16;  // 8 rows x 22 = 16 banks mod 32
  int c[3] = {ox + t % TX, oy + (PAIRED ? ((t >> 4) & 1) * (TY / 2) + (t >> 5) : t / TX), 0};
  const bool active = c[0] <= n0 - 3 && c[1] <= n1 - 3;
  const long long idx = active ? c[0] + (long long)c[1] * g.st[1] : 0;
  const CellT<2, T> C{MIXED ? (const T *)(const void *)a.in32 : (const T *)(const void *)a.in, a.bg, g.N};
  const double h = a.sc->dt / a.hdiv;
  const T cm[2] = {(T)red_get(a.sc->red[a.red_in], 0), (T)red_get(a.sc->red[a.red_in], 1)};

  // ------------------------------------------------ phase A: fluxes and q
  // (each branch has its direction as a compile-time constant, so nothing
  // indexes Geo, cm or the flux temporaries dynamically)
  auto flux_item = [=](auto dirc, int rr) {
    constexpr int dir = decltype(dirc)::value;
    const int cx = dir == 0 ? ox - 2 + rr % B::F0X : ox + rr % B::F1X;
    const int cy = dir == 0 ? oy + rr / B::F0X : oy - 2 + rr / B::F1X;
    T F[NW];
    if (cx >= 0 && cx < n0 && cy >= 0 && cy < n1) {
      fluxes_fast<2, T>(C, cx + (long long)cy * g.st[1], dir, p.gamma, p.has_bgb, F);
    } else {
#pragma unroll
      for (int f = 0; f < NW; ++f) F[f] = 0;
    }
    T *dst = (dir == 0 ? F0 : F1) + rr;
    constexpr int stride = dir == 0 ? B::F0N : B::F1N;
#pragma unroll
    for (int f = 0; f < NW; ++f)
      if (f != L::B0 + dir) dst[B::fslot(f, dir) * stride] = F[f];
  };
  for (int r = t; r < B::F0N + B::F1N + B::QN; r += NT) {
    if (r < B::F0N) {
      flux_item(std::integral_constant<int, 0>{}, r);
    } else if (r < B::F0N + B::F1N) {
      flux_item(std::integral_constant<int, 1>{}, r - B::F0N);
    } else {
      const int rr = r - B::F0N - B::F1N;
      int cx = ox - 3 + rr % B::QX, cy = oy - 3 + rr / B::QX;
      T q[B::NQS];
      const bool inx = cx >= 0 && cx < n0, iny = cy >= 0 && cy < n1;
      // pads of the padded copies: right 0, left q(5); corners never read
      // (slots 6..8 are read at the tile +-1 only, always inside the grid)
      if ((!inx && !iny) || cx >= n0 || cy >= n1) {
#pragma unroll
        for (int k = 0; k < B::NQS; ++k) q[k] = 0;
      } else {
        if (cx < 0) cx = 5;
        if (cy < 0) cy = 5;
        q_cell<T>(C, cx + (long long)cy * g.st[1], q);
      }
#pragma unroll
      for (int k = 0; k < B::NQS; ++k) Q[k * B::QN + rr] = q[k];
    }
  }
  __syncthreads();

  // ------------------------------------------------ phase B: face ratios along x and y
  // One work unit: SEG consecutive faces along d of one q slot on one line of
  // the tile.  The line's q values are read once, each first difference
  // |q_j+1 - q_j| and third difference |3 (q_j+1 - q_j) - (q_j+2 - q_j-1)| is
  // formed once, and each face takes the max of the five first and the three
  // third differences around it.  The last run of a line is shifted back to
  // end at the line's last face (faces it shares with the run before are
  // written twice, with the same value).
  constexpr int SEG = 5;
  constexpr int NS0 = (TX + 1 + SEG - 1) / SEG, NS1 = (TY + 1 + SEG - 1) / SEG;
  constexpr int NU0 = 5 * (TY + 2) * NS0, NU1 = 5 * (TX + 2) * NS1;
  static_assert(SEG <= TX + 1 && SEG <= TY + 1, "a run must fit in a line");
  auto face_run = [=](auto dc, int u) {
    constexpr int d = decltype(dc)::value;
    constexpr int NL = d == 0 ? TX : TY;  // faces of a line: -1 .. NL-1 (tile-relative left cell)
    int line, s, k;  // line: the row (d = 0) or column (d = 1) + 1, tile-relative
    if (d == 0) {
      s = u % NS0;
      line = (u / NS0) % (TY + 2);
      k = u / (NS0 * (TY + 2));
    } else {
      line = u % (TX + 2);
      s = (u / (TX + 2)) % NS1;
      k = u / ((TX + 2) * NS1);
    }
    const int f0 = min(-1 + s * SEG, NL - SEG);      // first face of the run
    const int slot = k < 4 ? k : (d == 0 ? 5 : 4);   // B_f, f != d
    constexpr int sd = d == 0 ? 1 : B::QX;
    // q at the cells f0-2 .. f0+SEG+2 along d
    const T *qq = Q + slot * B::QN +
                  (d == 0 ? (f0 + 1) + B::QX * (line + 2) : (line + 2) + B::QX * (f0 + 1));
    T q[SEG + 5], t1[SEG + 4], t3[SEG + 3];
#pragma unroll
    for (int j = 0; j < SEG + 5; ++j) q[j] = qq[j * sd];
#pragma unroll
    for (int j = 0; j < SEG + 4; ++j) t1[j] = q[j + 1] - q[j];
#pragma unroll
    for (int j = 1; j <= SEG + 2; ++j) t3[j] = vabs(vfma((T)3, t1[j], -(q[j + 2] - q[j - 1])));
    T *dst = (d == 0 ? V0 + k * B::V0N : V1 + k * B::V1N);
#pragma unroll
    for (int m = 0; m < SEG; ++m) {
      T m1 = 0, m3 = 0;
#pragma unroll
      for (int j = m; j <= m + 4; ++j) m1 = vmax(m1, vabs(t1[j]));
#pragma unroll
      for (int j = m + 1; j <= m + 3; ++j) m3 = vmax(m3, t3[j]);
      const int fc = f0 + m + 1;
      dst[d == 0 ? fc + B::V0X * line : line + B::V1X * fc] = m1 > 0 ? vratio(m3, m1) : T(0);
    }
  };
  if (p.hyperdif) {
    for (int u = t; u < NU0 + NU1; u += NT) {
      if (u < NU0)
        face_run(std::integral_constant<int, 0>{}, u);
      else
        face_run(std::integral_constant<int, 1>{}, u - NU0);
    }
  }
  __syncthreads();

  // ------------------------------------------------ phase C: the cell's sources
  T dL[NW];
#pragma unroll
  for (int f = 0; f < NW; ++f) dL[f] = 0;
  T numax = 0;
  if (active) {
    const int tx = c[0] - ox, ty = c[1] - oy;
    const T idx1[2] = {(T)(1.0 / __ldg(g.dx1[0] + c[0])), (T)(1.0 / __ldg(g.dx1[1] + c[1]))};
    // flux divergences
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      if (z4(g, c, dir)) continue;
      const T *Fb = dir == 0 ? F0 + (tx + 2) + B::F0X * ty : F1 + tx + B::F1X * (ty + 2);
      const int st = dir == 0 ? 1 : B::F1X;
      const int fs = dir == 0 ? B::F0N : B::F1N;
      const T w12 = idx1[dir] * (T)(1.0 / 12.0);
#pragma unroll
      for (int f = 0; f < NW; ++f) {
        if (f == L::B0 + dir) continue;  // zero flux
        const T *Fp = Fb + B::fslot(f, dir) * fs;
        dL[f] -= ((T)8 * (Fp[st] - Fp[-st]) - (Fp[2 * st] - Fp[-2 * st])) * w12;
      }
    }
    // gravity
    if (p.has_grav) {
      const T rho = C.v(L::RHO, idx), irt = (T)(1.0 / ((double)rho + C.vd(L::RHOB, idx)));
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        dL[L::M0 + k] += (T)p.g[k] * rho;
        dL[L::EN] += rho * (T)p.g[k] * C.v(L::M0 + k, idx) * irt;
      }
    }
    if (p.divb) divb_sources<T>(C, g, p, c, idx, dL);
    const int r0 = (tx + 3) + B::QX * (ty + 3);
    // the terms along dimension d (a compile-time constant in each call, so
    // that nothing indexes Geo, c, cm or idx1 dynamically)
    auto dim_terms = [&](auto dc) {
      constexpr int d = decltype(dc)::value;
      const int sd = d == 0 ? 1 : B::QX;
      const bool zd = z1(g, c, d);
      const T i1 = idx1[d], i2 = idx1[d] * idx1[d];
      if (p.has_bgb) {  // background energy terms along d (addenergyterms_cd2)
        const double bb0 = C.vd(L::BB0, idx), bb1 = C.vd(L::BB0 + 1, idx);
        const double bb2 = bb0 * bb0 + bb1 * bb1;
        const T ptb = (T)((p.gamma - 1) * C.vd(L::EB, idx) - 0.5 * (p.gamma - 2) * bb2);
        const bool z4d = z4(g, c, d);
#pragma unroll
        for (int dir = 0; dir < 2; ++dir) {
          const T *v = Q + (2 + dir) * B::QN + r0;
          const T gv =
              z4d ? T(0) : ((T)8 * (v[sd] - v[-sd]) - (v[2 * sd] - v[-2 * sd])) * (i1 * (T)(1.0 / 12.0));
          if (d == dir) dL[L::EN] -= ptb * gv;
          dL[L::EN] += C.v(L::BB0 + d, idx) * C.v(L::BB0 + dir, idx) * gv;
        }
      }
      if (!p.hyperdif) return;
      // this dimension's face ratios: the cell's right face, its left face,
      // and the face stride across d (the other dim)
      const T *V = d == 0 ? V0 : V1;
      const int vn = d == 0 ? B::V0N : B::V1N;
      const int fr = d == 0 ? (tx + 1) + B::V0X * (ty + 1) : (tx + 1) + B::V1X * (ty + 1);
      const int fl = fr - (d == 0 ? 1 : B::V1X);
      const int fo = 1 - d;                                  // the other dimension
      const int sv = d == 0 ? B::V0X : 1;                    // face stride along fo
      const int sq = fo == 0 ? 1 : B::QX;                    // q stride along fo
      const T dxd = (T)__ldg(g.dx1[d] + c[d]);
      // dx c_max c_hyp of each slot, and whether the neighbours along fo are
      // inner cells (the cell itself is: tiles cover inner cells only)
      T kk[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const int fid = k == 0 ? L::RHO : k == 1 ? L::EN : k < 4 ? L::M0 + (k - 2) : L::B0 + (d == 0 ? 1 : 0);
        kk[k] = dxd * cm[d] * (T)p.chyp[fid];
      }
      const int cfo = c[fo], nfo = fo == 0 ? n0 : n1;
      const bool inm = cfo - 1 >= 2, inp = cfo + 1 <= nfo - 3;
      // nu_R, nu_L of slot k at the cell shifted by s (-1, 0, +1) along fo;
      // 0 off the inner cells, as the reference's viscosity arrays are
      auto nu_at = [&](int k, int s, T &nr, T &nl) {
        const bool in = s == 0 ? true : (s > 0 ? inp : inm);
        nr = in ? kk[k] * V[k * vn + fr + s * sv] : T(0);
        nl = in ? kk[k] * V[k * vn + fl + s * sv] : T(0);
      };
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        T nr, nl;
        nu_at(k, 0, nr, nl);
        numax = vmax(numax, vmax(nr, nl));
      }
      // rho and internal energy: f += (nu_R dq+ - nu_L dq-) / dx^2
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const T *q = Q + k * B::QN + r0;
        T nr, nl;
        nu_at(k, 0, nr, nl);
        const T dp = zd ? T(0) : q[sd] - q[0], dm = zd ? T(0) : q[0] - q[-sd];
        dL[k == 0 ? L::RHO : L::EN] += (nr * dp - nl * dm) * i2;
      }
      // momentum (rho_t and m at the neighbours from the q box)
      const T *qrt = Q + 6 * B::QN + r0;
      const T rt0 = qrt[0], rtp = qrt[sd], rtm = qrt[-sd];
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        const int k = 2 + f;
        const T *v = Q + k * B::QN + r0;
        T nr, nl;
        nu_at(k, 0, nr, nl);
        const T dvp = zd ? T(0) : v[sd] - v[0], dvm = zd ? T(0) : v[0] - v[-sd];
        const T *qm = Q + (7 + f) * B::QN + r0;
        const T m0 = qm[0], mp = qm[sd], mm = qm[-sd];
        const T fac = (f == d ? (T)1 : (T)0.5) * i2;
        dL[L::M0 + f] += ((rt0 + rtp) * nr * dvp - (rt0 + rtm) * nl * dvm) * (T)0.5 * fac;
        dL[L::EN] += ((m0 + mp) * nr * dvp - (m0 + mm) * nl * dvm) * (T)0.5 * fac;
        if (f != d) {  // off-diagonal: m_d += d_f( rho_t (nu_R+nu_L)/4 d_d v_f )
          T t1[2], t2[2];
#pragma unroll
          for (int s = 0; s < 2; ++s) {
            const int o = s ? sq : -sq;
            int cx[3] = {c[0], c[1], 0};
            cx[f] += s ? 1 : -1;
            T nr2, nl2;
            nu_at(k, s ? 1 : -1, nr2, nl2);
            const T nsum = nr2 + nl2;
            const T tmp5 = z1(g, cx, d) ? T(0) : (v[o + sd] - v[o - sd]) * (T)0.5 * i1;
            const T tmp6 = tmp5 * nsum * (T)0.25;
            t1[s] = qrt[o] * tmp6;
            t2[s] = tmp6 * Q[(7 + d) * B::QN + r0 + o];
          }
          if (!z1(g, c, f)) {
            const T hf = (T)0.5 * idx1[f];
            dL[L::M0 + d] += (t1[1] - t1[0]) * hf;
            dL[L::EN] += (t2[1] - t2[0]) * hf;
          }
        }
      }
      // magnetic field B_f, f = the other dimension
      {
        const int f = fo, k = 4;
        const T *b = Q + (4 + f) * B::QN + r0;
        T nr, nl;
        nu_at(k, 0, nr, nl);
        T t1[2], t2[2];
#pragma unroll
        for (int s = 0; s < 2; ++s) {  // off-diagonal: B_d -= d_f( (nu_L+nu_R)/2 d_d B_f ), e with B_d
          const int o = s ? sq : -sq;
          int cx[3] = {c[0], c[1], 0};
          cx[f] += s ? 1 : -1;
          T nr2, nl2;
          nu_at(k, s ? 1 : -1, nr2, nl2);
          const T nsum = nr2 + nl2;
          const T tmp2 = z1(g, cx, d) ? T(0) : (b[o + sd] - b[o - sd]) * (T)0.5 * i1;
          t1[s] = tmp2 * nsum * (T)0.5;
          t2[s] = t1[s] * Q[(4 + d) * B::QN + r0 + o];
        }
        if (!z1(g, c, f)) {
          const T hf = (T)0.5 * idx1[f];
          dL[L::B0 + d] -= (t1[1] - t1[0]) * hf;
          dL[L::EN] -= (t2[1] - t2[0]) * hf;
        }
        // diagonal: B_f += (nu_R dB+ - nu_L dB-)/dx^2 and Ohmic heating
        const T dbp = zd ? T(0) : b[sd] - b[0], dbm = zd ? T(0) : b[0] - b[-sd];
        dL[L::B0 + f] += (nr * dbp - nl * dbm) * i2;
        dL[L::EN] += ((T)0.5 * (b[0] + b[sd]) * nr * dbp - (T)0.5 * (b[0] + b[-sd]) * nl * dbm) * i2;
      }
    };
    if (p.hyperdif || p.has_bgb) {
      dim_terms(std::integral_constant<int, 0>{});
      dim_terms(std::integral_constant<int, 1>{});
    }
  }
  stage_epilogue<2, T>(a, g, p, C, c, active, idx, h, dL, numax, red);
}

// Shared memory (elements of the stencil type) of a stage body: the
// three-phase body in 2-D, the per-dimension body in 3-D.
template <int D, typename S>
__host__ __device__ constexpr int stage_smem_elems() {
  return D == 2 ? Box2<S>::ELEMS : tile_smem_elems<D, S>();
}

}  // namespace SMAUG_NS
