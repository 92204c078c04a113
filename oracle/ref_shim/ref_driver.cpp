/*
 * ref_driver.cpp -- test infrastructure, NOT product code.
 *
 * A small C API around the host build of the SMAUG reference (see
 * build_ref.py).  It replays the reference's own per-step sequence of cu*
 * calls -- the single-step (rkon==0) loop body of dev/smaug/src/iosmaug.cpp --
 * so tests can run the reference on any state and compare.
 *
 *   ref_init        : struct params set-up as models/iosmaugparams.h.ot:13-200
 *                     does, cuinit (init.cu:816-1000) and initgrid
 *                     (init.cu:1118-1670) with readini=0 (uniform grid).
 *   ref_set_state   : load a state into wmod slots 0 and 1 and apply the
 *                     initial boundary pass (iosmaug.cpp:786-794).
 *   ref_step(n)     : one loop iteration n of iosmaug.cpp:802-1166.
 *   ref_get_*       : read back state / derived fields / scalars.
 *
 * Compiled only by build_ref.py, together with the reference sources, with
 * -DUSE_SAC (2-D) or -DUSE_SAC_3D (3-D).
 */
#include "../include/cudapars.h"
#include "../include/iotypes.h"
#include "../include/iobparams.h"
#include "../include/smaugcukernels.h"

shim_uint3 blockIdx, threadIdx, blockDim, gridDim;

namespace {
struct params *p = nullptr, *d_p = nullptr;
struct bparams *bp = nullptr, *d_bp = nullptr;
struct state *st = nullptr, *d_state = nullptr;
real *wmod = nullptr, *wnew = nullptr, *wd = nullptr;
real *d_wnew = nullptr, *d_wmod = nullptr, *d_dwn1 = nullptr, *d_wd = nullptr;
real *d_wtemp = nullptr, *d_wtemp1 = nullptr, *d_wtemp2 = nullptr, *d_w = nullptr;
real cmaxd[3];
int dimp = 0;
}  // namespace

extern "C" {

int ref_ndim(void) { return NDIM; }
int ref_nvar(void) { return NVAR; }
int ref_nderv(void) { return NDERV; }
int ref_params_size(void) { return (int)sizeof(struct params); }

/*
 * n[]      : cells per dim INCLUDING the 2+2 ghost layers (reference convention)
 * xmin/dx  : grid origin (of cell 0, a ghost) and spacing per dim
 * chyp     : NVAR hyperdiffusion coefficients
 * btype    : boundtype per dim (same for all fields and both sides)
 */
int ref_init(const int *n, const double *xmin, const double *dx, double gamma,
             const double *chyp, const int *btype, double courant, int moddton,
             int hyperdifmom, double dt_fixed, const double *g) {
  p = (struct params *)calloc(1, sizeof(struct params));
  st = (struct state *)calloc(1, sizeof(struct state));
  bp = (struct bparams *)calloc(1, sizeof(struct bparams));
  dimp = 1;
  for (int d = 0; d < NDIM; ++d) {
    p->n[d] = n[d];
    p->ng[d] = 2;
    p->npgp[d] = 1;
    p->dx[d] = dx[d];
    p->xmin[d] = xmin[d];
    p->xmax[d] = xmin[d] + n[d] * dx[d];
    p->g[d] = g ? g[d] : 0.0;
    dimp *= n[d];
  }
  p->gamma = gamma;
  p->mu = 1.0;
  p->eta = 0.0;
  p->rkon = 0;
  p->sodifon = 0;
  p->moddton = moddton;
  p->divbon = 0;
  p->divbfix = 0;
  p->hyperdifmom = hyperdifmom;
  p->readini = 0;
  p->cfgsavefrequency = 1;
  p->courant = courant;
  p->maxviscoef = 0;
  p->dtdiffvisc = 0;
  p->chyp3 = 0;
  p->npe = 1;
  p->mode = 0;
  p->cmax = 0.02;
  p->qt = 0;
  p->it = 0;
  for (int f = 0; f < NVAR; ++f) p->chyp[f] = chyp[f];
  for (int f = 0; f < NVAR; ++f)
    for (int d = 0; d < NDIM; ++d)
      for (int s = 0; s < 2; ++s) p->boundtype[f][d][s] = btype[d];
  p->dt = (moddton == 1) ? 1.0e-8 : dt_fixed; /* iosmaug.cpp:327-330 */

  wmod = (real *)calloc((size_t)2 * NVAR * dimp, sizeof(real));
  wd = (real *)calloc((size_t)NDERV * dimp, sizeof(real));
  wnew = (real *)calloc((size_t)NVAR * dimp, sizeof(real));
  cuinit(&p, &bp, &wmod, &wnew, &wd, &st, &d_p, &d_bp, &d_wnew, &d_wmod, &d_dwn1, &d_wd,
         &d_state, &d_wtemp, &d_wtemp1, &d_wtemp2);
  initgrid(&p, &st, &wd, &d_p, &d_dwn1, &d_wd, &d_state, &d_wtemp, &d_wtemp1, &d_wtemp2);
  d_w = d_wmod;
  return 0;
}

/* divbon and divbfix (the divergence-of-B source terms, divb.cu), after ref_init. */
int ref_set_divb(int on) {
  p->divbon = p->divbfix = on;
  d_p->divbon = d_p->divbfix = on;
  return 0;
}

/* Boundary type of one field along one dim (both sides), after ref_init. */
int ref_set_btype(int field, int dim, int type) {
  if (field < 0 || field >= NVAR || dim < 0 || dim >= NDIM) return -1;
  p->boundtype[field][dim][0] = p->boundtype[field][dim][1] = type;
  d_p->boundtype[field][dim][0] = d_p->boundtype[field][dim][1] = type;
  return 0;
}

/* w: NVAR*dimp, field-major, x fastest (the wmod slot layout, iotypes.h:213). */
int ref_set_state(const double *w) {
  memcpy(d_wmod, w, sizeof(real) * NVAR * dimp);
  memcpy(d_wmod + (size_t)NVAR * dimp, w, sizeof(real) * NVAR * dimp);
  /* iosmaug.cpp:645-654: fixed boundaries are captured from slot 0 at it = -1 */
  const int its = p->it;
  p->it = -1;
  d_p->it = -1;
  for (int ii = 0; ii < NVAR; ii++)
    for (int idir = 0; idir < NDIM; idir++)
      if (p->boundtype[ii][idir][0] == 5) cuboundary(&p, &bp, &d_p, &d_bp, &d_state, &d_wmod, 0, idir, ii);
  p->it = its;
  d_p->it = its;
  /* iosmaug.cpp:786-794: boundary on slot 1 for the evolved fields */
  for (int ii = 0; ii <= (b1 + (NDIM - 1)); ii++)
    for (int idir = 0; idir < NDIM; idir++)
      cuboundary(&p, &bp, &d_p, &d_bp, &d_state, &d_wmod, 1, idir, ii);
  return 0;
}

int ref_get_state(double *w, int slot) {
  memcpy(w, d_wmod + (size_t)slot * NVAR * dimp, sizeof(real) * NVAR * dimp);
  return 0;
}

int ref_get_wd(double *out) {
  memcpy(out, d_wd, sizeof(real) * NDERV * dimp);
  return 0;
}

double ref_get_dt(void) { return p->dt; }
void ref_set_dt(double dt) { p->dt = dt; }
double ref_get_scalar(int which) {
  switch (which) {
    case 0: return p->cmax;
    case 1: return p->maxcourant;
    case 2: return p->maxviscoef;
    case 3: return p->dtdiffvisc;
    case 4: return cmaxd[0];
    case 5: return cmaxd[1];
    case 6: return NDIM > 2 ? cmaxd[2] : 0.0;
    default: return 0.0;
  }
}
void ref_set_maxviscoef(double v) { p->maxviscoef = v; }

/* One iteration n of the reference loop, rkon==0 path (iosmaug.cpp:802-1166). */
int ref_step(int n) {
  int order = 0, ordero = 1;
  real dt;
  p->it = n;
  cucomputedervfields(&p, &d_p, &d_wmod, &d_wd, 0); /* 809-812 */

  if (p->moddton == 1.0) { /* 855-898 */
    p->maxcourant = 0.0;
    for (int dim = 0; dim <= (NDIM - 1); dim++) {
      cucomputec(&p, &d_p, &d_wmod, &d_wd, order, dim);
      cucomputemaxc(&p, &d_p, &d_wmod, &d_wd, order, dim, &wd, &d_wtemp);
      cucomputemaxcourant(&p, &d_p, &d_wmod, &d_wd, order, dim, &wd, &d_wtemp);
    }
    if (((p->courant) / (p->maxcourant)) > 1.0e-8) p->dt = (p->courant) / (p->maxcourant);
    if (n > 1) cugetdtvisc1(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2);
    if ((p->dtdiffvisc) > 1.0e-8 && (p->dt) > ((p->dtdiffvisc))) p->dt = (p->dtdiffvisc);
  }

  /* 904-960 */
  for (int dir = 0; dir < NDIM; dir++) cucomputevels(&p, &d_p, &d_wmod, &d_wd, order, dir);
  for (int dir = 0; dir < NDIM; dir++) {
    for (int f = rho; f <= (mom1 + NDIM - 1); f++) {
      if (f == mom1 + dir) {
        cucomputept(&p, &d_p, &d_wmod, &d_wd, order, dir);
        cucomputepbg(&p, &d_p, &d_wmod, &d_wd, order, dir);
      }
      cucentdiff1(&p, &d_p, &d_state, &d_wmod, &d_wmod, &d_dwn1, &d_wd, order, ordero, p->dt, f, dir);
    }
    for (int f = energy; f <= (b1 + (NDIM - 1)); f++) {
      if (f == energy) {
        cucomputevels(&p, &d_p, &d_wmod, &d_wd, order, dir);
        cucomputepbg(&p, &d_p, &d_wmod, &d_wd, ordero, dir);
        cucomputept(&p, &d_p, &d_wmod, &d_wd, order, dir);
      }
      cucentdiff2(&p, &d_p, &d_state, &d_wmod, &d_wmod, &d_dwn1, &d_wd, order, ordero, p->dt, f, dir);
    }
  }
  cugrav(&p, &d_p, &d_state, &d_wmod, &d_wmod, &d_dwn1, &d_wd, order, ordero, p->dt);
  if (p->divbon == 1) cudivb(&p, &d_p, &d_w, &d_wmod, &d_dwn1, &d_wd, order, ordero, p->dt); /* 962-963 */

  if (p->hyperdifmom == 1) { /* 969-1146 */
    dt = (p->dt);
    p->maxviscoef = 0.0;
    for (int dim = 0; dim <= (NDIM - 1); dim++) {
      cucomputec(&p, &d_p, &d_wmod, &d_wd, order, dim);
      cucomputemaxc(&p, &d_p, &d_wmod, &d_wd, order, dim, &wd, &d_wtemp);
      cmaxd[dim] = p->cmax;
      cuhyperdifvisc1ir(&p, &d_p, &d_wmod, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, rho, dim);
      cuhyperdifvisc1r(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, rho, dim);
      cuhyperdifvisc1l(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, rho, dim);
      cuhyperdifrhosource1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, rho, dim, p->dt);
    }
    for (int dim = 0; dim <= (NDIM - 1); dim++) {
      p->cmax = cmaxd[dim];
      cuhyperdifvisc1ir(&p, &d_p, &d_wmod, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, energy, dim);
      cuhyperdifvisc1r(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, energy, dim);
      cuhyperdifvisc1l(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, energy, dim);
      cuhyperdifesource1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, energy, dim, dt);
    }
    for (int dim = 0; dim <= (NDIM - 1); dim++)
      for (int f = 0; f <= (NDIM - 1); f++) {
        p->cmax = cmaxd[dim];
        cuhyperdifvisc1ir(&p, &d_p, &d_wmod, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, mom1 + f, dim);
        cuhyperdifvisc1r(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, mom1 + f, dim);
        cuhyperdifvisc1l(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, mom1 + f, dim);
        for (int ii1 = 0; ii1 <= 1; ii1++) {
          int ii, ii0;
          if (ii1 == 0) {
            ii = dim;
            ii0 = f;
          } else {
            ii = f;
            ii0 = dim;
          }
          if (ii == dim)
            cuhyperdifmomsource1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, f, dim, ii, ii0, p->dt);
          else
            cuhyperdifmomsourcene1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, f, dim, ii, ii0, p->dt);
        }
      }
    for (int dim = 0; dim <= (NDIM - 1); dim++)
      for (int f = 0; f <= (NDIM - 1); f++)
        if (f != dim) {
          p->cmax = cmaxd[dim];
          cuhyperdifvisc1ir(&p, &d_p, &d_wmod, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, b1 + f, dim);
          cuhyperdifvisc1r(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, b1 + f, dim);
          cuhyperdifvisc1l(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, b1 + f, dim);
          for (int ii1 = 0; ii1 <= 1; ii1++) {
            int jj, mm, ii0;
            real sb;
            if (ii1 == 0) {
              jj = dim;
              mm = f;
              sb = -1.0;
              ii0 = dim;
            } else {
              ii0 = f;
              mm = dim;
              sb = 1.0;
              jj = f;
            }
            if (mm == dim)
              cuhyperdifbsource1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, f, dim, jj, ii0, mm, sb, p->dt);
            else
              cuhyperdifbsourcene1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, f, dim, jj, ii0, mm, sb, p->dt);
          }
        }
  }
  cusource(&p, &d_p, &d_state, &d_w, &d_wmod, &d_dwn1, &d_wd, order, ordero, p->dt); /* 1153 */
  for (int ii = 0; ii <= (b1 + (NDIM - 1)); ii++) /* 1157-1166 */
    for (int idir = 0; idir < NDIM; idir++)
      cuboundary(&p, &bp, &d_p, &d_bp, &d_state, &d_wmod, ordero, idir, ii);
  p->it = n + 1;
  return 0;
}

}  // extern "C"
