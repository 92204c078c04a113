// smaug_tile2.cuh -- the 2-D stage body in three phases.
//
// Same operator as tile_body (smaug_tile.cuh), reorganised for 2-D so that a
// tile needs two block barriers instead of ten and reads the state from
// global memory once per cell of the tile +-3:
//   phase A  the q slots of every cell of the tile +-3 (q_from: the six
//            hyperviscosity inputs rho, e_int, v_x, v_y, B_x, B_y, and what
//            the fluxes and the momentum terms need at the neighbours);
//   phase B  one loop over runs of cell faces of both dimensions: the ratio
//            max|d3 q| / max|d1 q| of the hyperviscosity once per face
//            (nu_R of a cell and nu_L of its right neighbour share their
//            windows, consecutive faces share their differences), along x on
//            the tile +-1 in y, along y on the tile +-1 in x (the
//            off-diagonal terms need nu there);
//   phase C  per cell: the fluxes at the four neighbours along each
//            dimension from their q slots and their 4th-order divergence,
//            gravity, background energy terms, hyperdiffusion with
//            nu = dx c_max c_hyp * ratio on the cell's faces, then the shared
//            epilogue.
// A q cell outside the grid along one dimension takes that dimension's pad
// (0 on the right, q(5) on the left, as the reference's padded copies do);
// the corners outside both are never read.
#pragma once
#include <type_traits>

#include "smaug_tile.cuh"
#include "smaug_pair.cuh"

namespace SMAUG_NS {
using namespace smaug;

// The q slots of one cell (2-D).  The hyperviscosity inputs: 0 rho,
// 1 internal energy (formed in FP64), 2 v_x, 3 v_y, 4 B_x, 5 B_y.  What the
// momentum terms read at the neighbours: 6 rho_t = rho + rho_b, 7 m_x, 8 m_y.
// What the fluxes read beyond those: 9 e, 10 the total pressure p_T (formed
// in FP64, as the reference's pressure recovery), and with an energy
// background (bgb) 11 B_b,x, 12 B_b,y, 13 e_b (not written without one).
// The raw values of one cell that its q slots are formed from (loaded
// first, so that a thread's loads for all its q cells are in flight together).
template <typename T>
struct QRaw {
  T rho, m0, m1, b0, b1, e, bb0, bb1, eb;
  double rhob;
};

template <typename T>
__device__ __forceinline__ void q_load(const CellT<2, T> &c, long long i, bool bgb, QRaw<T> &r) {
  using L = Lay<2>;
  r.rho = c.v(L::RHO, i);
  r.rhob = c.vd(L::RHOB, i);
  r.m0 = c.v(L::M0, i);
  r.m1 = c.v(L::M0 + 1, i);
  r.b0 = c.v(L::B0, i);
  r.b1 = c.v(L::B0 + 1, i);
  r.e = c.v(L::EN, i);
  r.bb0 = bgb ? c.v(L::BB0, i) : T(0);
  r.bb1 = bgb ? c.v(L::BB0 + 1, i) : T(0);
  r.eb = bgb ? c.v(L::EB, i) : T(0);
}

template <typename T>
__device__ __forceinline__ void q_from(const QRaw<T> &r, double gam, T *q) {
  const T rho = r.rho, m0 = r.m0, m1 = r.m1, b0 = r.b0, b1 = r.b1, e = r.e, bb0 = r.bb0, bb1 = r.bb1;
  const double rhob = r.rhob;
  const double irtd = __drcp_rn((double)rho + rhob);
  const T irt = (T)irtd;
  const double b2 = (double)b0 * (double)b0 + (double)b1 * (double)b1;
  const double m2 = (double)m0 * (double)m0 + (double)m1 * (double)m1;
  const double bbb = (double)b0 * (double)bb0 + (double)b1 * (double)bb1;
  q[0] = rho;
  q[1] = (T)((double)e - 0.5 * (b2 + m2 * irtd));
  q[2] = m0 * irt;
  q[3] = m1 * irt;
  q[4] = b0;
  q[5] = b1;
  q[6] = rho + (T)rhob;
  q[7] = m0;
  q[8] = m1;
  q[9] = e;
  q[10] = (T)((gam - 1.0) * ((double)e - 0.5 * m2 * irtd) - (gam - 2.0) * (bbb + 0.5 * b2));
  q[11] = bb0;
  q[12] = bb1;
  q[13] = r.eb;
}

// The fluxes along dir at the q-box cell r, from its q slots (the physical
// fluxes of fluxes_at: rho, momentum, energy, induction; B_dir has none):
// F[0] rho, F[1] m_x, F[2] m_y, F[3] e, F[4] B_f with f the other dimension.
// In terms of v = m / rho_t, so that no reciprocal is formed here:
//   m_k:  v_d m_k - b_k (b_d + B_b,d) - B_b,k b_d  (+ p_T on k = d)
//   e:    v_d (e + e_b + p_T) - (b_d + B_b,d) (b.v) - b_d (B_b.v)
//   B_f:  v_d (b_f + B_b,f) - (b_d + B_b,d) v_f
// Explicit FMAs: every build variant gives the same bits.
template <int dir, int QN, typename T>
__device__ __forceinline__ void flux_q(const T *Q, int r, bool bgb, T *F) {
  const T v0 = Q[2 * QN + r], v1 = Q[3 * QN + r], b0 = Q[4 * QN + r], b1 = Q[5 * QN + r];
  const T m0 = Q[7 * QN + r], m1 = Q[8 * QN + r], e = Q[9 * QN + r], pt = Q[10 * QN + r];
  T bb0 = 0, bb1 = 0, eb = 0;
  if (bgb) {
    bb0 = Q[11 * QN + r];
    bb1 = Q[12 * QN + r];
    eb = Q[13 * QN + r];
  }
  const T vd = dir == 0 ? v0 : v1, bd = dir == 0 ? b0 : b1, bbd = dir == 0 ? bb0 : bb1;
  const T bdt = bd + bbd;
  F[0] = dir == 0 ? m0 : m1;
  F[1] = vfma(vd, m0, -vfma(b0, bdt, bb0 * bd));
  F[2] = vfma(vd, m1, -vfma(b1, bdt, bb1 * bd));
  if (dir == 0)
    F[1] += pt;
  else
    F[2] += pt;
  const T bv = vfma(b1, v1, b0 * v0), bbv = vfma(bb1, v1, bb0 * v0);
  F[3] = vfma(vd, (e + eb) + pt, -vfma(bdt, bv, bd * bbv));
  const T bf = dir == 0 ? b1 : b0, bbf = dir == 0 ? bb1 : bb0, vf = dir == 0 ? v1 : v0;
  F[4] = vfma(vd, bf + bbf, -(bdt * vf));
}

// flux_q at two q-box cells at once (FP32 only): lane lo at cell ra, lane hi
// at cell rb, each lane the same operations in the same order as flux_q, so
// the same bits.
template <int dir, int QN>
__device__ __forceinline__ void flux_q2(const float *Q, int ra, int rb, bool bgb, f2 *F) {
  auto ld = [&](int slot) { return f2_make(Q[slot * QN + ra], Q[slot * QN + rb]); };
  const f2 v0 = ld(2), v1 = ld(3), b0 = ld(4), b1 = ld(5);
  const f2 m0 = ld(7), m1 = ld(8), e = ld(9), pt = ld(10);
  f2 bb0 = f2_splat(0.0f), bb1 = bb0, eb = bb0;
  if (bgb) {
    bb0 = ld(11);
    bb1 = ld(12);
    eb = ld(13);
  }
  const f2 vd = dir == 0 ? v0 : v1, bd = dir == 0 ? b0 : b1, bbd = dir == 0 ? bb0 : bb1;
  const f2 bdt = bd + bbd;
  F[0] = dir == 0 ? m0 : m1;
  F[1] = pfma(vd, m0, pneg(pfma(b0, bdt, bb0 * bd)));
  F[2] = pfma(vd, m1, pneg(pfma(b1, bdt, bb1 * bd)));
  if (dir == 0)
    F[1] = F[1] + pt;
  else
    F[2] = F[2] + pt;
  const f2 bv = pfma(b1, v1, b0 * v0), bbv = pfma(bb1, v1, bb0 * v0);
  F[3] = pfma(vd, (e + eb) + pt, pneg(pfma(bdt, bv, bd * bbv)));
  const f2 bf = dir == 0 ? b1 : b0, bbf = dir == 0 ? bb1 : bb0, vf = dir == 0 ? v1 : v0;
  F[4] = pfma(vd, bf + bbf, pneg(bdt * vf));
}

// Box sizes of the three-phase body for a TX x TY tile.
template <typename S>
struct Box2 {
  static constexpr int TX = S::TX, TY = S::TY;
  static constexpr int NQS = 14;                        // q slots per cell (q_from)
  static constexpr int QX = TX + 6, QN = QX * (TY + 6);  // q: tile +-3
  // face ratios along x: faces x+1/2 for x in [-1, TX), rows tile +-1
  static constexpr int V0X = TX + 1, V0N = (TX + 1) * (TY + 2);
  // face ratios along y: faces y+1/2 for y in [-1, TY), columns tile +-1
  static constexpr int V1X = TX + 2, V1N = (TX + 2) * (TY + 1);
  // offsets (elements) of the arrays in shared memory
  static constexpr int OQ = 0, OV0 = OQ + NQS * QN, OV1 = OV0 + 5 * V0N;
  static constexpr int ELEMS = OV1 + 5 * V1N;
};

// The rows of the tile that the epilogue reads are prefetched toward L2 at the start
// of the tile, so that their DRAM latency overlaps phases A-C. Those rows are the
// cell's RK base, the accumulator and the compensation where the stage reads them,
// rho_b and the energy backgrounds, and the last dim's metric. Each (array, row)
// segment of TX cells gets a prefetch at its first and its last byte. Every address
// lies in its array: the rows are inner rows, and a row's TX cells from ox run at
// most into the next row.
template <typename T, int TX, int TY, int NT>
__device__ __forceinline__ void prefetch_epilogue_rows(const StageArgs &a, const Geo &g, const Phys &p, int ox,
                                                       int oy) {
  using L = Lay<2>;
  constexpr int NW = L::NW;
  constexpr bool MIXED = sizeof(T) == sizeof(float);
  const int nrow = min(TY, g.n[1] - 2 - oy);
  const bool acc = MIXED ? a.kind >= 2 : (a.kind == 3 || a.kind == 4);
  const bool comp = MIXED && a.kind == 4;
  // arrays: base 0..NW-1, accumulator NW..2NW-1, compensation 2NW..3NW-1,
  // backgrounds 3NW..3NW+3 (rho_b always), the last dim's metric 3NW+4
  constexpr int NA = 3 * NW + 5;
  for (int s = threadIdx.x; s < NA * TY; s += NT) {
    const int arr = s / TY, row = s % TY;
    if (row >= nrow) continue;
    const unsigned cell = (unsigned)(ox + (oy + row) * g.st[1]);
    const char *ptr = nullptr;
    int es = (int)sizeof(T);
    if (arr < NW) {
      ptr = MIXED ? (const char *)(a.w32 + fo32(arr, g.N, cell)) : (const char *)(a.base + fo32(arr, g.N, cell));
    } else if (arr < 2 * NW) {
      if (acc)
        ptr = MIXED ? (const char *)(a.acc32 + fo32(arr - NW, g.N, cell))
                    : (const char *)(a.acc + fo32(arr - NW, g.N, cell));
    } else if (arr < 3 * NW) {
      if (comp) ptr = (const char *)(a.c32 + fo32(arr - 2 * NW, g.N, cell));
    } else if (arr < 3 * NW + 4) {
      const int b = arr - 3 * NW;
      if (b == L::RHOB - NW || p.has_bgb) ptr = (const char *)(a.bg + fo32(b, g.N, cell));
      es = 8;
    } else {
      ptr = (const char *)(g.dxlast + cell);
      es = 8;
    }
    if (!ptr) continue;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr + TX * es - 1));
  }
}

// The q box of tile (nbx, nby) of the same simulation (the block's next work
// item), prefetched toward L2: the stage input's fields and the backgrounds that
// q_load reads, one prefetch per line of each row segment of the box, clamped to
// the grid.
template <typename T, int TX, int TY, int NT>
__device__ __forceinline__ void prefetch_qbox_rows(const StageArgs &a, const Geo &g, const Phys &p, int nbx,
                                                   int nby) {
  using L = Lay<2>;
  constexpr int NW = L::NW;
  constexpr bool MIXED = sizeof(T) == sizeof(float);
  const int x0 = max(2 + nbx * TX - 3, 0), x1 = min(2 + nbx * TX + TX + 2, g.n[0] - 1);
  const int y0 = max(2 + nby * TY - 3, 0), y1 = min(2 + nby * TY + TY + 2, g.n[1] - 1);
  const int nrow = y1 - y0 + 1;
  // arrays: the stage input's NW fields, then rho_b, e_b, B_b
  constexpr int NA = NW + 4;
  for (int s = threadIdx.x; s < NA * (TY + 6); s += NT) {
    const int arr = s / (TY + 6), row = s % (TY + 6);
    if (row >= nrow) continue;
    const unsigned c0 = (unsigned)(x0 + (y0 + row) * g.st[1]), c1 = (unsigned)(x1 + (y0 + row) * g.st[1]);
    const char *p0, *p1;
    if (arr < NW) {
      const T *in = MIXED ? (const T *)(const void *)a.in32 : (const T *)(const void *)a.in;
      p0 = (const char *)(in + fo32(arr, g.N, c0));
      p1 = (const char *)(in + fo32(arr, g.N, c1));
    } else {
      const int b = arr - NW;
      if (!(b == L::RHOB - NW || p.has_bgb)) continue;
      p0 = (const char *)(a.bg + fo32(b, g.N, c0));
      p1 = (const char *)(a.bg + fo32(b, g.N, c1));
    }
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p0));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p1));
  }
}

template <typename T, typename S>
__device__ __forceinline__ void tile_body2(const StageArgs &a, const Geo &g, const Phys &p, int bx, int by, int nbx,
                                           int nby, T *sm, T *red) {
  using L = Lay<2>;
  using B = Box2<S>;
  constexpr int TX = S::TX, TY = S::TY, NT = TX * TY;
  constexpr int NW = L::NW;
  constexpr bool MIXED = sizeof(T) == sizeof(float);
  T *Q = sm + B::OQ, *V0 = sm + B::OV0, *V1 = sm + B::OV1;

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
  const double h = a.hslot > 0 ? a.sc->hst[a.hslot] : a.sc->dt / a.hdiv;
  const T cm[2] = {(T)red_get(a.sc->red[a.red_in], 0), (T)red_get(a.sc->red[a.red_in], 1)};
  prefetch_epilogue_rows<T, TX, TY, NT>(a, g, p, ox, oy);
  if (nbx >= 0) prefetch_qbox_rows<T, TX, TY, NT>(a, g, p, nbx, nby);

  // ------------------------------------------------ phase A: q on the tile +-3
  // A fixed number of q cells per thread (the loop unrolled, so that the
  // compiler may issue a later cell's loads ahead of an earlier cell's math).
  {
    constexpr int NA = (B::QN + NT - 1) / NT;
#pragma unroll
    for (int u = 0; u < NA; ++u) {
      const int rr = t + u * NT;
      if (rr >= B::QN) continue;
      int cx = ox - 3 + rr % B::QX, cy = oy - 3 + rr / B::QX;
      const bool inx = cx >= 0 && cx < n0, iny = cy >= 0 && cy < n1;
      T q[B::NQS];
      // pads of the padded copies: right 0, left q(5); corners never read
      // (slots 6..13 are read at the tile +-2 along one dimension only,
      // always inside the grid)
      if ((!inx && !iny) || cx >= n0 || cy >= n1) {
#pragma unroll
        for (int k = 0; k < B::NQS; ++k) q[k] = 0;
      } else {
        if (cx < 0) cx = 5;
        if (cy < 0) cy = 5;
        QRaw<T> raw;
        q_load<T>(C, cx + (long long)cy * g.st[1], p.has_bgb, raw);
        q_from<T>(raw, p.gamma, q);
      }
#pragma unroll
      for (int k = 0; k < B::NQS; ++k)
        if (k < 11 || p.has_bgb) Q[k * B::QN + rr] = q[k];
    }
  }
  __syncthreads();

  // ------------------------------------------------ phase B: face ratios along x and y
  // One work unit: SEG consecutive faces along d (RUN, or the whole line if
  // it is shorter) of one q slot on one line of the tile.  The line's q
  // values are read once, each first difference |q_j+1 - q_j| and third
  // difference |3 (q_j+1 - q_j) - (q_j+2 - q_j-1)| is
  // formed once, and each face takes the max of the five first and the three
  // third differences around it.  The last run of a line is shifted back to
  // end at the line's last face (faces it shares with the run before are
  // written twice, with the same value).
  constexpr int RUN = 9;  // faces per run, at most a line's
  constexpr int SEG0 = RUN < TX + 1 ? RUN : TX + 1, SEG1 = RUN < TY + 1 ? RUN : TY + 1;
  constexpr int NS0 = (TX + 1 + SEG0 - 1) / SEG0, NS1 = (TY + 1 + SEG1 - 1) / SEG1;
  constexpr int NU0 = 5 * (TY + 2) * NS0, NU1 = 5 * (TX + 2) * NS1;
  auto face_run = [=](auto dc, int u) {
    constexpr int d = decltype(dc)::value;
    constexpr int SEG = d == 0 ? SEG0 : SEG1;
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
    const T idx1[2] = {(T)__ldg(g.rdx1[0] + c[0]), (T)__ldg(g.rdx1[1] + c[1])};
    const int r0 = (tx + 3) + B::QX * (ty + 3);
    // flux divergences: -(8 (F_+1 - F_-1) - (F_+2 - F_-2)) / (12 dx), the
    // fluxes of the neighbours (inside the grid: the cell is an inner cell)
    // from their q slots
    auto div_terms = [&](auto dc) {
      constexpr int dir = decltype(dc)::value;
      if (z4(g, c, dir)) return;
      constexpr int sd = dir == 0 ? 1 : B::QX;
      const T w12 = idx1[dir] * (T)(1.0 / 12.0);
      if constexpr (MIXED) {
        // lanes: the +1 / -1 neighbour (lo) and the +2 / -2 one (hi)
        f2 Fp[5], Fm[5];
        flux_q2<dir, B::QN>((const float *)Q, r0 + sd, r0 + 2 * sd, p.has_bgb, Fp);
        flux_q2<dir, B::QN>((const float *)Q, r0 - sd, r0 - 2 * sd, p.has_bgb, Fm);
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          const int f = k < 4 ? k : L::B0 + 1 - dir;
          const f2 dd = Fp[k] - Fm[k];
          dL[f] = vfma(-vfma((T)8, (T)f2_lo(dd), -(T)f2_hi(dd)), w12, dL[f]);
        }
        return;
      }
      T Fp[5], Fm[5], d1[5];
      flux_q<dir, B::QN>(Q, r0 + sd, p.has_bgb, Fp);
      flux_q<dir, B::QN>(Q, r0 - sd, p.has_bgb, Fm);
#pragma unroll
      for (int k = 0; k < 5; ++k) d1[k] = Fp[k] - Fm[k];
      flux_q<dir, B::QN>(Q, r0 + 2 * sd, p.has_bgb, Fp);
      flux_q<dir, B::QN>(Q, r0 - 2 * sd, p.has_bgb, Fm);
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const int f = k < 4 ? k : L::B0 + 1 - dir;
        dL[f] = vfma(-vfma((T)8, d1[k], -(Fp[k] - Fm[k])), w12, dL[f]);
      }
    };
    div_terms(std::integral_constant<int, 0>{});
    div_terms(std::integral_constant<int, 1>{});
    // gravity
    if (p.has_grav) {
      const T rho = C.v(L::RHO, idx), irt = (T)__drcp_rn((double)rho + C.vd(L::RHOB, idx));
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        dL[L::M0 + k] += (T)p.g[k] * rho;
        dL[L::EN] += rho * (T)p.g[k] * C.v(L::M0 + k, idx) * irt;
      }
    }
    if (p.divb) divb_sources<T>(C, g, p, c, idx, dL);
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
