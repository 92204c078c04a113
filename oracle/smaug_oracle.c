/*
 * smaug_oracle.c -- CPU restatement (FP64) of the SMAUG/SAC ideal-MHD step.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, loaded by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg.  The product path
 * never calls it.
 *
 * Every routine restates the reference code named beside it, term by term and
 * in the same floating-point operation order, so that one single step of this
 * file agrees with the host build of the reference (oracle/ref_shim) to the
 * last bits.  Paths below are relative to dev/smaug/ of the reference.
 *
 * Build: gcc -O2 -ffp-contract=off -fopenmp -fPIC -shared (no FMA contraction,
 * as the reference host build).  The per-cell loops run under OpenMP: every
 * iteration writes only its own cell, and the maxima are taken per thread and
 * then combined with the same comparison, so the results do not depend on the
 * thread count (max is exact).
 */
#include "smaug_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int D, n[3];
  long N, st[3];
  int RHO, EN, EB, RHOB, M0, B0, BB0, NVAR, NW;
} lay_t;

static lay_t mklay(const sm_oracle_grid *g) {
  lay_t L;
  L.D = g->ndim;
  for (int d = 0; d < 3; ++d) L.n[d] = (d < g->ndim) ? g->n[d] : 1;
  L.st[0] = 1;
  L.st[1] = L.n[0];
  L.st[2] = (long)L.n[0] * L.n[1];
  L.N = (long)L.n[0] * L.n[1] * L.n[2];
  /* iotypes.h:213-219 */
  L.RHO = 0;
  L.M0 = 1;
  L.EN = 1 + L.D;
  L.B0 = 2 + L.D;
  L.EB = 2 + 2 * L.D;
  L.RHOB = 3 + 2 * L.D;
  L.BB0 = 4 + 2 * L.D;
  L.NVAR = 4 + 3 * L.D;
  L.NW = 2 + 2 * L.D;
  return L;
}

int sm_oracle_nvar(int ndim) { return 4 + 3 * ndim; }

#define F(w, f) ((w) + (long)(f) * L->N)

static inline void coords(const lay_t *L, long idx, int c[3]) {
  c[0] = (int)(idx % L->n[0]);
  c[1] = (int)((idx / L->n[0]) % L->n[1]);
  c[2] = (int)(idx / L->st[2]);
}

static inline int inner(const lay_t *L, const int c[3]) { /* all coords in [2, n-3] */
  for (int d = 0; d < L->D; ++d)
    if (c[d] < 2 || c[d] > L->n[d] - 3) return 0;
  return 1;
}

/* others (dims != d) within [lo, n-1-lo] */
static inline int others_in(const lay_t *L, const int c[3], int d, int lo) {
  for (int e = 0; e < L->D; ++e)
    if (e != d && (c[e] < lo || c[e] > L->n[e] - 1 - lo)) return 0;
  return 1;
}

/* ---------------------------------------------------------------- gradients
 * grad3dn_MODID, gradops.cu:437-606: 4th-order central difference with the
 * boundary zeroing for non-periodic directions (operator precedence as in the
 * reference: the n-3 and 2 tests are unconditional). */
static double grad3dn(const sm_oracle_grid *g, const lay_t *L, const double *a, long idx,
                      const int c[3], int d) {
  double grad = 0;
  const int n = L->n[d];
  const long s = L->st[d];
  if (c[d] > 1 && c[d] < n - 2)
    grad = (((8 * a[idx + s] - 8 * a[idx - s] + a[idx - 2 * s] - a[idx + 2 * s]) / 6.0)) /
           (2.0 * (g->delx[d][idx]));
  if (g->btype[d] != 0) {
    if ((c[d] == n - 3) || (c[d] == n - 4 && others_in(L, c, d, 2)))
      grad = 0;
    else if (c[d] == 2 || (c[d] == 3 && others_in(L, c, d, 2)))
      grad = 0;
  }
  return grad;
}

/* grad1r3n_MODID / grad1l3n_MODID, gradops.cu:608-753, evaluated at inner cells
 * only (where the reference's zeroing reduces to c_d in {1, 2, n-3, n-2}). */
static double grad1r(const sm_oracle_grid *g, const lay_t *L, const double *a, long idx,
                     const int c[3], int d) {
  const int n = L->n[d];
  double grad = 0;
  if (c[d] < n - 1) grad = ((a[idx + L->st[d]] - a[idx]) / ((g->delx[d][idx])));
  if (g->btype[d] != 0 && (c[d] == n - 2 || c[d] == n - 3 || c[d] == 1 || c[d] == 2)) grad = 0;
  return grad;
}
static double grad1l(const sm_oracle_grid *g, const lay_t *L, const double *a, long idx,
                     const int c[3], int d) {
  const int n = L->n[d];
  double grad = 0;
  if (c[d] > 0 && c[d] < n) grad = ((a[idx] - a[idx - L->st[d]]) / ((g->delx[d][idx])));
  if (g->btype[d] != 0 && (c[d] == n - 2 || c[d] == n - 3 || c[d] == 1 || c[d] == 2)) grad = 0;
  return grad;
}

/* grad13n_MODID, gradops.cu:755-826: 2nd-order central difference on [1, n-2];
 * zeroing at {1, 2, n-3, n-2} for non-periodic directions, including the
 * reference's `j>1` test in the 3-D z branch. */
static double grad13(const sm_oracle_grid *g, const lay_t *L, const double *a, long idx,
                     const int c[3], int d) {
  const int n = L->n[d];
  double grad = 0;
  if (c[d] > 0 && c[d] < n - 1) {
    grad = ((a[idx + L->st[d]] - a[idx - L->st[d]]) / ((g->delx[d][idx])) / 2.0);
    if (g->btype[d] != 0) {
      if ((c[d] == n - 2) || (c[d] == n - 3 && others_in(L, c, d, 1)))
        grad = 0;
      else if (L->D == 3 && d == 2) {
        if (c[d] == 1 || (c[d] == 2 && c[0] > 0 && c[0] < L->n[0] - 1 && c[1] > 1 && c[1] < L->n[1] - 1))
          grad = 0;
      } else if (c[d] == 1 || (c[d] == 2 && others_in(L, c, d, 1)))
        grad = 0;
    }
  }
  return grad;
}

/* -------------------------------------------------------- derived quantities */

/* computept3_MODID, dervfields.cu:107-153 */
static double pt_of(const sm_oracle_grid *g, const lay_t *L, const double *w, long i) {
  double bb = 0, b2 = 0, m2 = 0;
  for (int k = 0; k < L->D; ++k) bb += F(w, L->B0 + k)[i] * F(w, L->BB0 + k)[i];
  for (int k = 0; k < L->D; ++k) b2 += F(w, L->B0 + k)[i] * F(w, L->B0 + k)[i];
  for (int k = 0; k < L->D; ++k) m2 += F(w, L->M0 + k)[i] * F(w, L->M0 + k)[i];
  double t = ((g->gamma) - 2.0) * ((bb) + 0.5 * (b2));
  return ((g->gamma) - 1.0) * (F(w, L->EN)[i] - 0.5 * (m2) / (F(w, L->RHO)[i] + F(w, L->RHOB)[i])) - t;
}

/* computepbg3_MODID, dervfields.cu:157-191 */
static double ptb_of(const sm_oracle_grid *g, const lay_t *L, const double *w, long i) {
  double bb2 = 0;
  for (int k = 0; k < L->D; ++k) bb2 += F(w, L->BB0 + k)[i] * F(w, L->BB0 + k)[i];
  return ((g->gamma) - 1) * F(w, L->EB)[i] - 0.5 * ((g->gamma) - 2) * (bb2);
}

/* computec3_MODID, dervfields.cu:241-309 (returns c_fast along dir) */
static double cfast_of(const sm_oracle_grid *g, const lay_t *L, const double *w, long i, int dir) {
  const double gam = g->gamma;
  double m2 = 0, b2 = 0, bbb = 0, bb2 = 0;
  for (int k = 0; k < L->D; ++k) m2 += F(w, L->M0 + k)[i] * F(w, L->M0 + k)[i];
  for (int k = 0; k < L->D; ++k) b2 += F(w, L->B0 + k)[i] * F(w, L->B0 + k)[i];
  for (int k = 0; k < L->D; ++k) bbb += F(w, L->BB0 + k)[i] * F(w, L->B0 + k)[i];
  for (int k = 0; k < L->D; ++k) bb2 += F(w, L->BB0 + k)[i] * F(w, L->BB0 + k)[i];
  const double rt = F(w, L->RHO)[i] + F(w, L->RHOB)[i];
  double pk = ((gam)-1) * (F(w, L->EN)[i] - 0.5 * ((m2) / (rt)) - 0.5 * (b2) - (bbb));
  double cs2 = (((gam)) * (pk + (((gam)) - 1) * (F(w, L->EB)[i] - 0.5 * (bb2))) / (rt));
  double cf = ((b2) + (bb2) + 2.0 * (bbb)) / (rt) + (cs2);
  double bd = F(w, L->BB0 + dir)[i] + F(w, L->B0 + dir)[i];
  double cfasti = 0.5 * (cf + sqrt(cf * cf - 4.0 * cs2 * ((bd) * (bd)) / (rt)));
  return sqrt(cfasti) + fabs(F(w, L->M0 + dir)[i] / (rt));
}

void sm_oracle_cfast(const sm_oracle_grid *g, const double *w, int dim, double *cf) {
  lay_t L0 = mklay(g);
  const lay_t *L = &L0;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < L->N; ++i) cf[i] = cfast_of(g, L, w, i, dim);
}

/* cucomputemaxc, computedervfields.cu:1922-2116: max of cfast over all cells,
 * starting from 0 (the sound-speed pass reduces zeros, 1997-1999). */
void sm_oracle_cmax(const sm_oracle_grid *g, const double *w, double *cmax) {
  lay_t L0 = mklay(g);
  const lay_t *L = &L0;
  for (int d = 0; d < L->D; ++d) {
    double m = 0.0;
#pragma omp parallel
    {
      double ml = 0.0;
#pragma omp for schedule(static) nowait
      for (long i = 0; i < L->N; ++i) {
        double v = cfast_of(g, L, w, i, d);
        if (v > ml) ml = v;
      }
#pragma omp critical
      if (ml > m) m = ml;
    }
    cmax[d] = m;
  }
}

/* ndimp as computed by cucomputemaxc/cugetdtvisc1 (computedervfields.cu:1940-1950):
 * note fn += 1 is applied to the fractional log2, so ndimp ~ 2 * dimp. */
static long ref_ndimp(long dimp) {
  double fn, fractn, in;
  fn = log((double)dimp) / log(2.0);
  fractn = modf(fn, &in);
  if (fractn > 0) {
    fn += 1;
    return (long)(int)pow(2, fn);
  }
  return dimp;
}

double sm_oracle_select_dt(const sm_oracle_grid *g, const double *w, int step, sm_oracle_state *s) {
  lay_t L0 = mklay(g);
  const lay_t *L = &L0;
  const int dl = L->D - 1;
  /* cucomputemaxcourant (computedervfields.cu:2118-2296) resets maxcourant on
   * every call, so only the last dimension's c_fast/dx survives the dim loop. */
  double *cour = (double *)malloc(sizeof(double) * L->N);
  double maxc = 0.0;
#pragma omp parallel
  {
    double ml = 0.0;
#pragma omp for schedule(static) nowait
    for (long i = 0; i < L->N; ++i) {
      cour[i] = cfast_of(g, L, w, i, dl) / (g->delx[dl][i]);
      if (cour[i] > ml) ml = cour[i];
    }
#pragma omp critical
    if (ml > maxc) maxc = ml;
  }
  s->maxcourant = maxc;
  if (((g->courant) / (maxc)) > 1.0e-8) s->dt = (g->courant) / (maxc); /* iosmaug.cpp:874-875 */
  if (step > 1) {
    /* cugetdtvisc1, nushk1.cu:658-790: zeropadmaxdtvisc runs numBlocks(512)
     * blocks of 64 threads, so only the first K cells receive
     * maxviscoef/dx^2; the rest of the reduced buffer still holds the
     * courant values c_fast/dx left by cucomputemaxcourant. */
    long ndimp = ref_ndimp(L->N);
    long K = ((ndimp + 511) / 512) * 64;
    double cmx = 0.0;
    for (long i = K; i < L->N; ++i)
      if (cour[i] > cmx) cmx = cour[i];
    double dtd = 0.0000000001;
    for (int dir = 0; dir < L->D; ++dir) {
      double m = cmx;
      for (long i = 0; i < K && i < L->N; ++i) {
        double dx = g->delx[dir][i];
        double v = ((s->maxviscoef) + 0.0) / ((dx) * (dx));
        if (v > m) m = v;
      }
      if (m > dtd) dtd = m;
      dtd = 0.25 / dtd;
    }
    s->dtdiffvisc = dtd;
  }
  free(cour);
  if ((s->dtdiffvisc) > 1.0e-8 && (s->dt) > ((s->dtdiffvisc))) s->dt = s->dtdiffvisc;
  return s->dt;
}

/* ---------------------------------------------------------------- fluxes */

/* centdiff1.cu:51-256 (rho, momentum) and centdiff2.cu:189-340 (energy, B) */
static double flux_of(const sm_oracle_grid *g, const lay_t *L, const double *w, const double *pt,
                      long i, int f, int dir) {
  const double rt = F(w, L->RHO)[i] + F(w, L->RHOB)[i];
  const double md = F(w, L->M0 + dir)[i];
  if (f == L->RHO) /* computefluxrho */
    return md * F(w, L->RHO)[i] / (F(w, L->RHO)[i] + F(w, L->RHOB)[i]) +
           (F(w, L->RHOB)[i] * md) / (F(w, L->RHOB)[i] + F(w, L->RHO)[i]);
  if (f >= L->M0 && f < L->M0 + L->D) { /* computefluxmom1/2/3, fluxmom1x */
    const int k = f - L->M0;
    double tr = md * F(w, f)[i] / (rt);
    const double bf = F(w, L->B0 + k)[i], bbf = F(w, L->BB0 + k)[i];
    const double bbd = F(w, L->BB0 + dir)[i], bd = F(w, L->B0 + dir)[i];
    double mg = (k == dir) ? pt[i] - (bf * bbd + bbf * bd) - bf * bd : -(bf * bbd + bbf * bd) - bf * bd;
    return tr + mg;
  }
  if (f == L->EN) { /* computefluxe: transportflux_cd2 + fluxe1 */
    double bbm = 0, bm = 0;
    for (int k = 0; k < L->D; ++k) bbm += F(w, L->BB0 + k)[i] * F(w, L->M0 + k)[i];
    for (int k = 0; k < L->D; ++k) bm += F(w, L->B0 + k)[i] * F(w, L->M0 + k)[i];
    double tr = md * F(w, L->EN)[i] / (rt);
    double fl = md * (pt[i]);
    fl -= F(w, L->B0 + dir)[i] * (bbm);
    fl -= F(w, L->BB0 + dir)[i] * (bm);
    fl /= (rt);
    fl += md * F(w, L->EB)[i] / (rt);
    fl -= F(w, L->B0 + dir)[i] * (bm) / (rt);
    return tr + fl;
  }
  /* computefluxb1/2/3 */
  const int k = f - L->B0;
  if (k == dir) return 0.0;
  return md * F(w, f)[i] / (rt) - (F(w, L->B0 + dir)[i] + F(w, L->BB0 + dir)[i]) * F(w, L->M0 + k)[i] / (rt) +
         (F(w, L->BB0 + k)[i]) * md / (rt);
}

/* ------------------------------------------------------- hyperviscosity */

/* hyperdifvisc1r.cu / hyperdifvisc1l.cu: right and left hyperviscosity of
 * field q along d at every inner cell.  The padded copy of q along d has
 * right pad 0 (what the zeroing in hyperdifvisc1r_parallel leaves) and left
 * pad q(5) (bc_hyperdifl, hyperdifvisc1l.cu:17-66: mirror about cell 2). */
static double qat(const lay_t *L, const double *q, long idx, const int c[3], int d, int off, int side) {
  int x = c[d] + off;
  if (x >= L->n[d]) return 0.0;          /* right pad (right chain only reads it) */
  if (x < 0) x = 5;                      /* left pad: W(0) = W(6) = q(5) */
  (void)side;
  return q[idx + (long)(x - c[d]) * L->st[d]];
}

static void hyperviscosity(const sm_oracle_grid *g, const lay_t *L, const double *q, int field, int d,
                           double cmax, double *nur, double *nul, double *numax) {
  const double chyp = g->chyp[field];
  double numax_all = *numax;
#pragma omp parallel
  {
  double numax_l = 0.0;
  double *numax = &numax_l; /* this thread's maximum, combined below */
#pragma omp for schedule(static) nowait
  for (long idx = 0; idx < L->N; ++idx) {
    int c[3];
    coords(L, idx, c);
    nur[idx] = 0;
    nul[idx] = 0;
    if (!inner(L, c)) continue;
    const double dx = g->delx[d][idx];
    /* right: hyperdifvisc2r/3r/4r (hyperdifvisc1r.cu:426-845) */
    double maxt1 = 0, maxt2 = 0;
    for (int s = -1; s <= 1; ++s) {
      int a = s + 1; /* p1 index A = c+1+s ; q(A) = offset s+1 from c */
      double v = fabs(3.0 * (qat(L, q, idx, c, d, a, 1) - qat(L, q, idx, c, d, a - 1, 1)) -
                      (qat(L, q, idx, c, d, a + 1, 1) - qat(L, q, idx, c, d, a - 2, 1)));
      if (v > maxt1) maxt1 = v;
    }
    for (int s = -2; s <= 2; ++s) {
      double v = fabs((qat(L, q, idx, c, d, s + 1, 1) - qat(L, q, idx, c, d, s, 1)));
      if (v > maxt2) maxt2 = v;
    }
    if (maxt2 > 0) nur[idx] = ((dx)) * (cmax) * (chyp)*maxt1 / maxt2;
    /* left: hyperdifvisc2l/3l/4l (hyperdifvisc1l.cu:436-855) */
    maxt1 = 0;
    maxt2 = 0;
    for (int s = -1; s <= 1; ++s) {
      int a = s + 1; /* q(A-1) = offset s */
      double v = fabs(3.0 * (qat(L, q, idx, c, d, a - 1, 0) - qat(L, q, idx, c, d, a - 2, 0)) -
                      (qat(L, q, idx, c, d, a, 0) - qat(L, q, idx, c, d, a - 3, 0)));
      if (v > maxt1) maxt1 = v;
    }
    for (int s = -2; s <= 2; ++s) {
      double v = fabs(qat(L, q, idx, c, d, s, 0) - (qat(L, q, idx, c, d, s - 1, 0)));
      if (v > maxt2) maxt2 = v;
    }
    if (maxt2 > 0) nul[idx] = ((dx)) * (cmax) * (chyp)*maxt1 / maxt2;
    if (nur[idx] > *numax) *numax = nur[idx];
    if (nul[idx] > *numax) *numax = nul[idx];
  }
#pragma omp critical
  if (numax_l > numax_all) numax_all = numax_l;
  }
  *numax = numax_all;
}

/* ------------------------------------------------------------ boundaries */

/* Ghost fill of the evolved fields, field by field and, for each field,
 * direction by direction (iosmaug.cpp:1157-1166 calls cuboundary in that
 * order), so a corner takes the rule of its last direction applied to the
 * values the earlier directions left.  Per direction d, ghost x of n cells:
 *   0 periodic  x <- x + (n-4) or x - (n-4)   (boundary.cu.sedov3d
 *               boundary{0,1,2}_per_parallel)
 *   3 cont      0,1 <- 2;  n-2,n-1 <- n-3     (gradops.cu:1043-1050,
 *               bc3_cont_dir)
 *   4 contcd4   0 <- 4, 1 <- 3, n-1 <- n-5, n-2 <- n-4
 *               (boundary.cu.sedov3d boundary{0,1,2}_contcd4_parallel)
 *   5 fixed     the values the state was loaded with (bc3_setfixed_dir at
 *               it = -1, iosmaug.cpp:645-654, and bc3_fixed_dir,
 *               gradops.cu:1201-1269).  The helper's tests read
 *               `i==0 || i==1 && dir==0` (gradops.cu:1244-1257), so the pass
 *               along d also restores the outermost ghost layer (0 and n-1)
 *               of every earlier direction; reproduced.
 *   6 symm      2-D: 0 <- 3, 1 <- 2, n-1 <- n-4, n-2 <- n-3;
 *               3-D: 0 <- 4, 1 <- 3, n-1 <- n-5, n-2 <- n-4
 *               (bc3_symm_dir, gradops.cu:1324-1395)
 *   7 asymm     the symm source, negated (bc3_asymm_dir, gradops.cu:1396-1468);
 *               also fields in bmask[d] where btype[d] is symm. */
static int bsrc(int type, int D, int n, int x, double *sign) {
  *sign = 1.0;
  switch (type) {
    case 0: return x < 2 ? x + (n - 4) : x - (n - 4);
    case 3: return x < 2 ? 2 : n - 3;
    case 4: return x == 0 ? 4 : x == 1 ? 3 : x == n - 1 ? n - 5 : n - 4;
    case 7: *sign = -1.0; /* fall through */
    case 6:
      if (D == 2) return x == 0 ? 3 : x == 1 ? 2 : x == n - 1 ? n - 4 : n - 3;
      return x == 0 ? 4 : x == 1 ? 3 : x == n - 1 ? n - 5 : n - 4;
    default: return -1;
  }
}

void sm_oracle_boundary(const sm_oracle_grid *g, double *w) {
  lay_t L0 = mklay(g);
  const lay_t *L = &L0;
  for (int f = 0; f < L->NW; ++f)
    for (int d = 0; d < L->D; ++d) {
      double *a = F(w, f);
      const int n = L->n[d];
      const long s = L->st[d];
      int type = g->btype[d];
      if (type == 6 && ((g->bmask[d] >> f) & 1)) type = 7;
      /* the sources of this pass are inner along d: no cell is both read and written */
#pragma omp parallel for schedule(static)
      for (long idx = 0; idx < L->N; ++idx) {
        int c[3];
        coords(L, idx, c);
        const int x = c[d];
        if (type == 5) {
          int hit = !(x >= 2 && x <= n - 3);
          for (int e = 0; e < d; ++e)
            if (c[e] == 0 || c[e] == L->n[e] - 1) hit = 1;
          if (hit && g->fixed) a[idx] = g->fixed[(long)f * L->N + idx];
          continue;
        }
        if (x >= 2 && x <= n - 3) continue;
        double sign;
        const int xs = bsrc(type, L->D, n, x, &sign);
        if (xs < 0) continue;
        a[idx] = sign * a[idx + (long)(xs - x) * s];
      }
    }
}

/* ------------------------------------------------------------- the stage */

/* grad3d_MODID (gradops.cu:132-237, 2-D branch): 4th-order difference over
 * the uniform spacing p->dx, zero at the first and last two inner cells
 * whatever the boundary type (the tests read `x==2 || x==3 && ...`, the
 * second part always true at inner cells). */
static double grad3d(const sm_oracle_grid *g, const lay_t *L, const double *a, long idx, const int c[3], int dir) {
  const int n = L->n[dir], x = c[dir], o = 1 - dir;
  const long s = L->st[dir];
  double grad = 0;
  if (x > 1 && x < n - 2)
    grad = (((8 * a[idx + s] - 8 * a[idx - s] + a[idx - 2 * s] - a[idx + 2 * s]) / 6.0)) / (2.0 * (g->dxs[dir]));
  const int in_o = c[o] > 1 && c[o] < L->n[o] - 2;
  if ((x == n - 3) || (x == n - 4 && in_o))
    grad = 0;
  else if (x == 2 || (x == 3 && in_o))
    grad = 0;
  return grad;
}

/* divb_parallel (divb.cu:165-336) with divbon = divbfix = 1, 2-D: at cells
 * 3..n-3 of both dims, divB = d_x b1 + d_y b2 + d_x b1b + d_y b2b and the
 * sources -divB (0, b, B.v, v) with B.v = (B_total . m) / rho_t
 * (computebdotv3, dervfields.cu:46-52) and NaN sources taken as 0
 * (dbsourcemom, dbsourceb); then every inner cell (from 2) takes
 * w -= dt * source. */
static void divb_terms(const sm_oracle_grid *g, const lay_t *L, const double *win, double *wout, double h) {
  const long N = L->N;
  const int NW = L->NW;
  double *dw = (double *)calloc((size_t)NW * N, sizeof(double));
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < N; ++idx) {
    int c[3];
    coords(L, idx, c);
    if (!(c[0] > 2 && c[1] > 2 && c[0] < L->n[0] - 2 && c[1] < L->n[1] - 2)) continue;
    double divb = grad3d(g, L, F(win, L->B0), idx, c, 0) + grad3d(g, L, F(win, L->B0 + 1), idx, c, 1);
    divb += grad3d(g, L, F(win, L->BB0), idx, c, 0) + grad3d(g, L, F(win, L->BB0 + 1), idx, c, 1);
    const double rt = F(win, L->RHO)[idx] + F(win, L->RHOB)[idx];
    const double bdotv = ((F(win, L->B0)[idx] + F(win, L->BB0)[idx]) * F(win, L->M0)[idx] +
                          (F(win, L->B0 + 1)[idx] + F(win, L->BB0 + 1)[idx]) * F(win, L->M0 + 1)[idx]) / rt;
    for (int k = 0; k < 2; ++k) {
      double sm = -divb * F(win, L->B0 + k)[idx];
      dw[(long)(L->M0 + k) * N + idx] = dw[(long)(L->M0 + k) * N + idx] + (isnan(sm) ? 0 : sm);
      double sb = -divb * F(win, L->M0 + k)[idx] / (F(win, L->RHO)[idx] + F(win, L->RHOB)[idx]);
      dw[(long)(L->B0 + k) * N + idx] = dw[(long)(L->B0 + k) * N + idx] + (isnan(sb) ? 0 : sb);
    }
    dw[(long)L->EN * N + idx] = dw[(long)L->EN * N + idx] + (-divb * bdotv);
  }
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < N; ++idx) {
    int c[3];
    coords(L, idx, c);
    if (!(c[0] > 1 && c[1] > 1 && c[0] < L->n[0] - 2 && c[1] < L->n[1] - 2)) continue;
    for (int f = 0; f < NW; ++f) F(wout, f)[idx] = F(wout, f)[idx] - h * dw[(long)f * N + idx];
  }
  free(dw);
}

/* Driver (usersource.cu.spicule1:4-137) on every cell of wout; the ghost
 * fill that follows overwrites the ghosts, as cuboundary does after cusource
 * (iosmaug.cpp:1153-1166). */
static void add_driver(const sm_oracle_grid *g, const lay_t *L, double *wout, double h, double t) {
  const sm_oracle_driver *dv = g->drv;
  if (!dv || !dv->on) return;
  const int D = L->D;
  double tdep = 1.0;
  if (dv->period > 0.0) tdep = sin(2.0 * 3.14159265358979323846 * t / dv->period);
  for (long idx = 0; idx < L->N; ++idx) {
    int c[3];
    coords(L, idx, c);
    double f[3] = {1.0, 1.0, 1.0};
    for (int d = 0; d < D; ++d) {
      if (dv->width[d] > 0.0) {
        const double x = (dv->xmin[d]) + (((double)c[d]) * (dv->dx[d]));
        const double r2 = (x - dv->center[d]) * (x - dv->center[d]);
        f[d] = exp(-r2 / (dv->width[d] * dv->width[d]));
      }
    }
    double prod = f[1] * f[0];
    if (D == 3) prod = prod * f[2];
    const double vvz = dv->amp * prod * tdep;
    double *m = F(wout, L->M0 + dv->dir);
    m[idx] = m[idx] + h * vvz * (F(wout, L->RHO)[idx] + F(wout, L->RHOB)[idx]);
  }
}

double sm_oracle_stage(const sm_oracle_grid *g, const double *win, const double *wbase, double *wout,
                       double h, const double *cmax) {
  return sm_oracle_stage_t(g, win, wbase, wout, h, cmax, 0.0);
}

double sm_oracle_stage_t(const sm_oracle_grid *g, const double *win, const double *wbase, double *wout,
                         double h, const double *cmax, double tin) {
  lay_t L0 = mklay(g);
  const lay_t *L = &L0;
  const long N = L->N;
  const int D = L->D;
  double numax = 0.0;
  double *pt = (double *)malloc(sizeof(double) * N);
  double *ptb = (double *)malloc(sizeof(double) * N);
  double *vel = (double *)malloc(sizeof(double) * N * 3);
  double *fl = (double *)malloc(sizeof(double) * N);
  double *q = (double *)malloc(sizeof(double) * N);
  double *nur = (double *)malloc(sizeof(double) * N);
  double *nul = (double *)malloc(sizeof(double) * N);
  double *t1 = (double *)malloc(sizeof(double) * N);
  double *t2 = (double *)malloc(sizeof(double) * N);
  double *t3 = (double *)malloc(sizeof(double) * N);

  if (wout != wbase) memcpy(wout, wbase, sizeof(double) * N * L->NW);
  memcpy(F(wout, L->NW), F(win, L->NW), sizeof(double) * N * (L->NVAR - L->NW));

#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) {
    pt[i] = pt_of(g, L, win, i);
    ptb[i] = ptb_of(g, L, win, i);
    for (int k = 0; k < D; ++k) /* computevel3_MODID, dervfields.cu:79-98 */
      vel[k * N + i] = F(win, L->M0 + k)[i] / (F(win, L->RHO)[i] + F(win, L->RHOB)[i]);
  }

  /* fluxes and divergences, iosmaug.cpp:913-957 */
  for (int dir = 0; dir < D; ++dir) {
    for (int f = 0; f < L->NW; ++f) {
      double *o = F(wout, f);
#pragma omp parallel for schedule(static)
      for (long i = 0; i < N; ++i) fl[i] = flux_of(g, L, win, pt, i, f, dir);
#pragma omp parallel for schedule(static)
      for (long idx = 0; idx < N; ++idx) {
        int c[3];
        coords(L, idx, c);
        if (!inner(L, c)) continue;
        /* centdiff1af / centdiff2b: w = w - dt * div */
        o[idx] = o[idx] - h * grad3dn(g, L, fl, idx, c, dir);
        if (f == L->EN) { /* addenergyterms_cd2, centdiff2.cu:80-115 */
          o[idx] -= +(h)*ptb[idx] * grad3dn(g, L, vel + (long)dir * N, idx, c, dir);
          for (int idim = 0; idim < D; idim++)
            o[idx] += (h)*F(wout, L->BB0 + idim)[idx] * F(wout, L->BB0 + dir)[idx] *
                      grad3dn(g, L, vel + (long)dir * N, idx, c, idim);
        }
      }
    }
  }

  /* gravity, addgrav_cd2 centdiff2.cu:118-150 */
#pragma omp parallel for schedule(static)
  for (long idx = 0; idx < N; ++idx) {
    int c[3];
    coords(L, idx, c);
    if (!inner(L, c)) continue;
    for (int k = 0; k < D; ++k) F(wout, L->M0 + k)[idx] += (h) * (g->g[k]) * F(win, L->RHO)[idx];
    for (int k = 0; k < D; ++k)
      F(wout, L->EN)[idx] += (h)*F(win, L->RHO)[idx] * ((g->g[k]) * F(win, L->M0 + k)[idx]) /
                             (F(win, L->RHO)[idx] + F(win, L->RHOB)[idx]);
  }

  /* divergence of B, cudivb (divb.cu:165-336; iosmaug.cpp:962-963): 2-D */
  if (g->divb && D == 2) divb_terms(g, L, win, wout, h);

  if (g->hyperdif) {
    /* ---- density, hyperdifrhosource1.cu:15-282 */
    for (int d = 0; d < D; ++d) {
      hyperviscosity(g, L, F(win, L->RHO), L->RHO, d, cmax[d], nur, nul, &numax);
#pragma omp parallel for schedule(static)
      for (long idx = 0; idx < N; ++idx) {
        int c[3];
        coords(L, idx, c);
        if (!inner(L, c)) continue;
        double tp = grad1r(g, L, F(win, L->RHO), idx, c, d);
        double tm = grad1l(g, L, F(win, L->RHO), idx, c, d);
        double rdx = g->delx[d][idx];
        F(wout, L->RHO)[idx] = F(wout, L->RHO)[idx] + h * ((nur[idx] + 0.0) * tp - (nul[idx] + 0.0) * tm) / rdx;
      }
    }
    /* ---- energy, hyperdifesource1.cu:18-554 (q = e - (B^2 + m^2/rho)/2) */
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; ++i) {
      double b2 = 0, m2 = 0;
      for (int k = 0; k < D; ++k) b2 += F(win, L->B0 + k)[i] * F(win, L->B0 + k)[i];
      for (int k = 0; k < D; ++k) m2 += F(win, L->M0 + k)[i] * F(win, L->M0 + k)[i];
      q[i] = F(win, L->EN)[i] - 0.5 * ((b2) + (m2) / (F(win, L->RHO)[i] + F(win, L->RHOB)[i]));
    }
    for (int d = 0; d < D; ++d) {
      hyperviscosity(g, L, q, L->EN, d, cmax[d], nur, nul, &numax);
#pragma omp parallel for schedule(static)
      for (long idx = 0; idx < N; ++idx) {
        int c[3];
        coords(L, idx, c);
        if (!inner(L, c)) continue;
        double tm = grad1l(g, L, q, idx, c, d);
        double tp = grad1r(g, L, q, idx, c, d);
        double rdx = g->delx[d][idx];
        F(wout, L->EN)[idx] = F(wout, L->EN)[idx] + h * ((nur[idx] + 0.0) * tp - (nul[idx] + 0.0) * tm) / rdx;
      }
    }
    /* ---- momentum, hyperdifmomsource1.cu / hyperdifmomsourcene1.cu */
    for (int d = 0; d < D; ++d)
      for (int f = 0; f < D; ++f) {
        double *v = vel + (long)f * N; /* q = m_f / rho_t (hyperdifvisc1r.cu:1240-1244) */
        hyperviscosity(g, L, v, L->M0 + f, d, cmax[d], nur, nul, &numax);
        for (int ii1 = 0; ii1 <= 1; ++ii1) {
          const int ii = ii1 == 0 ? d : f, ii0 = ii1 == 0 ? f : d;
          if (ii == d) { /* diagonal: hyperdifmomsource1/2/3/3a */
#pragma omp parallel for schedule(static)
            for (long idx = 0; idx < N; ++idx) {
              int c[3];
              coords(L, idx, c);
              if (!inner(L, c)) continue;
              const long s = L->st[d];
              const double *r = F(win, L->RHO), *rb = F(win, L->RHOB), *m = F(win, L->M0 + ii0);
              double tmp2 = (r[idx] + rb[idx] + r[idx - s] + rb[idx - s]) / 2;
              double tmp3 = (r[idx] + rb[idx] + r[idx + s] + rb[idx + s]) / 2;
              double tmp5 = (m[idx] + m[idx - s]) / 2;
              double tmp6 = (m[idx] + m[idx + s]) / 2;
              double tmp8 = grad1r(g, L, v, idx, c, d);
              double tmp7 = grad1l(g, L, v, idx, c, d);
              double rdx = g->delx[d][idx];
              double dm = (tmp3 * (nur[idx] + 0.0) * tmp8 - tmp2 * (nul[idx] + 0.0) * tmp7) / (rdx) / 2;
              F(wout, L->M0 + ii0)[idx] = F(wout, L->M0 + ii0)[idx] + h * dm;
              double de = (tmp6 * (nur[idx] + 0.0) * tmp8 - tmp5 * (nul[idx] + 0.0) * tmp7) / (rdx) / 2;
              F(wout, L->EN)[idx] = F(wout, L->EN)[idx] + h * de;
            }
          } else { /* off-diagonal: hyperdifmomsourcene1..6a */
            /* t1 = tmp7 = rho_t * tmp6, t2 = tmp8 = tmp6 * m_ii0, on [1,n-2]^D */
#pragma omp parallel for schedule(static)
            for (long idx = 0; idx < N; ++idx) {
              int c[3];
              coords(L, idx, c);
              t1[idx] = 0;
              t2[idx] = 0;
              int ok = 1;
              for (int e = 0; e < D; ++e)
                if (c[e] < 1 || c[e] > L->n[e] - 2) ok = 0;
              double tmp5 = ok ? grad13(g, L, v, idx, c, d) : 0.0;
              double tmp6 = tmp5 * ((nur[idx] + nul[idx] + 2.0 * 0.0)) / 4.0;
              t1[idx] = (F(win, L->RHO)[idx] + F(win, L->RHOB)[idx]) * tmp6;
              t2[idx] = tmp6 * F(win, L->M0 + ii0)[idx];
            }
#pragma omp parallel for schedule(static)
            for (long idx = 0; idx < N; ++idx) {
              int c[3];
              coords(L, idx, c);
              if (!inner(L, c)) continue;
              double dm = grad13(g, L, t1, idx, c, ii);
              F(wout, L->M0 + ii0)[idx] = F(wout, L->M0 + ii0)[idx] + h * dm;
            }
#pragma omp parallel for schedule(static)
            for (long idx = 0; idx < N; ++idx) {
              int c[3];
              coords(L, idx, c);
              if (!inner(L, c)) continue;
              double de = grad13(g, L, t2, idx, c, ii);
              F(wout, L->EN)[idx] = F(wout, L->EN)[idx] + h * de;
            }
          }
        }
      }
    /* ---- magnetic field, hyperdifbsource1.cu / hyperdifbsourcene1.cu */
    for (int d = 0; d < D; ++d)
      for (int f = 0; f < D; ++f) {
        if (f == d) continue;
        hyperviscosity(g, L, F(win, L->B0 + f), L->B0 + f, d, cmax[d], nur, nul, &numax);
        for (int ii1 = 0; ii1 <= 1; ++ii1) {
          const int jj = ii1 == 0 ? d : f, mm = ii1 == 0 ? f : d, ii0 = ii1 == 0 ? d : f;
          const double sb = ii1 == 0 ? -1.0 : 1.0;
          if (mm == d) { /* diagonal: hyperdifbsource1..4 with tmp1 = B_f on [1,n-2]^D */
            const double *b = F(win, L->B0 + f), *bj = F(win, L->B0 + jj);
#pragma omp parallel for schedule(static)
            for (long idx = 0; idx < N; ++idx) {
              int c[3];
              coords(L, idx, c);
              if (!inner(L, c)) continue;
              const long s = L->st[d];
              double tmp2 = (bj[idx] + bj[idx - s]) / 2;
              double tmp3 = (bj[idx] + bj[idx + s]) / 2;
              double tmp4 = grad1l(g, L, b, idx, c, d);
              double tmp5 = grad1r(g, L, b, idx, c, d);
              double rdx = g->delx[d][idx];
              double db = sb * (tmp5 * nur[idx] - tmp4 * nul[idx]) / rdx;
              double de = sb * (tmp3 * tmp5 * nur[idx] - tmp2 * tmp4 * nul[idx]) / rdx;
              F(wout, L->B0 + ii0)[idx] = F(wout, L->B0 + ii0)[idx] + h * db;
              F(wout, L->EN)[idx] = F(wout, L->EN)[idx] + h * de;
            }
          } else { /* off-diagonal: hyperdifbsourcene1..6a */
            const double *b = F(win, L->B0 + f);
#pragma omp parallel for schedule(static)
            for (long idx = 0; idx < N; ++idx) { /* t1 = tmp3, t2 = tmp5 */
              int c[3];
              coords(L, idx, c);
              int ok = 1;
              for (int e = 0; e < D; ++e)
                if (c[e] < 1 || c[e] > L->n[e] - 2) ok = 0;
              double tmp2 = ok ? grad13(g, L, b, idx, c, d) : 0.0;
              t1[idx] = tmp2 * (nul[idx] + nur[idx]) / 2;
              t2[idx] = t1[idx] * F(win, L->B0 + jj)[idx];
            }
#pragma omp parallel for schedule(static)
            for (long idx = 0; idx < N; ++idx) {
              int c[3];
              coords(L, idx, c);
              if (!inner(L, c)) continue;
              double db = sb * grad13(g, L, t1, idx, c, mm);
              F(wout, L->B0 + ii0)[idx] = F(wout, L->B0 + ii0)[idx] + h * db;
            }
#pragma omp parallel for schedule(static)
            for (long idx = 0; idx < N; ++idx) {
              int c[3];
              coords(L, idx, c);
              if (!inner(L, c)) continue;
              double de = sb * grad13(g, L, t2, idx, c, mm);
              F(wout, L->EN)[idx] = F(wout, L->EN)[idx] + h * de;
            }
          }
        }
      }
  }

  add_driver(g, L, wout, h, tin);
  sm_oracle_boundary(g, wout);
  free(pt);
  free(ptb);
  free(vel);
  free(fl);
  free(q);
  free(nur);
  free(nul);
  free(t1);
  free(t2);
  free(t3);
  return numax;
}

/* ------------------------------------------------------------- the step */

int sm_oracle_step(const sm_oracle_grid *g, double *w, int step, int rk4, int dt_mode, sm_oracle_state *s,
                   double *work) {
  lay_t L0 = mklay(g);
  const lay_t *L = &L0;
  const long NV = (long)L->NVAR * L->N;
  const long NW = (long)L->NW * L->N;
  double cm[3];
  if (dt_mode == 1) sm_oracle_select_dt(g, w, step, s);
  const double dt = s->dt;
  double numax = 0.0, v;
  if (!rk4) {
    double *w1 = work;
    sm_oracle_cmax(g, w, cm);
    for (int d = 0; d < L->D; ++d) s->cmax[d] = cm[d];
    v = sm_oracle_stage_t(g, w, w, w1, dt, cm, s->t);
    numax = v;
    memcpy(w, w1, sizeof(double) * NV);
  } else {
    /* SAC fourstep, vac.t:447-462 */
    double *w1 = work, *w2 = work + NV, *w3 = work + 2 * NV;
    sm_oracle_cmax(g, w, cm);
    for (int d = 0; d < L->D; ++d) s->cmax[d] = cm[d];
    v = sm_oracle_stage_t(g, w, w, w1, dt / 2, cm, s->t + 0.0 * dt); /* w1 = w + dt/2 k1 */
    if (v > numax) numax = v;
    sm_oracle_cmax(g, w1, cm);
    v = sm_oracle_stage_t(g, w1, w, w2, dt / 2, cm, s->t + 0.5 * dt); /* w2 = w + dt/2 k2 */
    if (v > numax) numax = v;
    sm_oracle_cmax(g, w2, cm);
    v = sm_oracle_stage_t(g, w2, w, w3, dt, cm, s->t + 0.5 * dt); /* w3 = w + dt k3 */
    if (v > numax) numax = v;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < NW; ++i) w1[i] = (w1[i] + 2 * w2[i] + w3[i] - 4 * w[i]) / 3;
    sm_oracle_cmax(g, w3, cm);
    v = sm_oracle_stage_t(g, w3, w, w2, dt / 6, cm, s->t + 1.0 * dt); /* w + dt/6 k4 */
    if (v > numax) numax = v;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < NW; ++i) w[i] = w2[i] + w1[i];
    sm_oracle_boundary(g, w);
  }
  /* The reference resets p->maxviscoef at the start of its hyperdiffusion
   * block (iosmaug.cpp:973), but the next call, cucomputec
   * (computedervfields.cu:2298-2328), copies the device params back over the
   * host copy, restoring the previous value: the coefficient is a running
   * maximum over all steps. */
  if (numax > s->maxviscoef) s->maxviscoef = numax;
  s->t += dt;
  return 0;
}
