/*
 * ref_loop.c -- the reference's single-step host loop over the
 * reference-compatible entry points of include/smaug_cukernels.h.
 *
 * The call sequence is the one of dev/smaug/src/iosmaug.cpp: the initial
 * ghost fill (783-790), then per step (802-1166, rkon = 0, moddton = 1)
 * cucomputedervfields, the dt block (cucomputec / cucomputemaxc /
 * cucomputemaxcourant per dimension, cugetdtvisc1 from the second step), the
 * fluxes (cucomputevels, cucomputept, cucomputepbg, cucentdiff1/2 per
 * direction and field), cugrav, cudivb, the hyperdiffusion chains
 * (cuhyperdifvisc1ir/1r/1l and the rho, e, momentum and B sources), cusource
 * and the ghost fill of every evolved field, and cuupdate at the end.  It
 * links against libsmaug_cu2d.so or libsmaug_cu3d.so (build with
 * -DSMAUG_CU_NDIM=2 or 3) as the reference's loop links against its own
 * kernels, and against libsmaug_b200.so for the VAC file reader and writer.
 *
 *   smaug_ref_loop{2d,3d} CONFIG.ini STEPS OUT.out [--btype B0,B1[,B2]] [--no-hyperdif] [--divb]
 *
 * OUT.out is a VAC binary snapshot of the state after STEPS steps (slot 1 of
 * wmod, where the reference's single step leaves it).  Prints the last dt.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "smaug_b200.h"
#include "smaug_cukernels.h"

#define CALL(x)                                                                       \
  do {                                                                                \
    int rc_ = (x);                                                                    \
    if (rc_ != 0) {                                                                   \
      fprintf(stderr, "ref_loop: %s failed (%d): %s\n", #x, rc_, smaug_cu_last_error()); \
      return 1;                                                                       \
    }                                                                                 \
  } while (0)

int main(int argc, char **argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s CONFIG.ini STEPS OUT.out [--btype B0,B1[,B2]] [--no-hyperdif] [--divb]\n", argv[0]);
    return 2;
  }
  const int nt = atoi(argv[2]);
  int bt[3] = {0, 0, 0}, hyperdif = 1, divbon = 0;
  for (int i = 4; i < argc; ++i) {
    if (!strcmp(argv[i], "--no-hyperdif")) hyperdif = 0;
    else if (!strcmp(argv[i], "--divb")) divbon = 1;
    else if (!strcmp(argv[i], "--btype") && i + 1 < argc) {
      char *s = argv[++i];
      for (int d = 0; d < NDIM && *s; ++d) {
        bt[d] = (int)strtol(s, &s, 10);
        if (*s == ',') ++s;
      }
    }
  }

  /* the configuration (readasciivacconfig): positions into wd, the state into wmod */
  smaug_vac_header h;
  if (smaug_vac_read_ascii(argv[1], &h, NULL, 0, NULL, 0) != 0 || h.ndim != NDIM || h.nw != NVAR) {
    fprintf(stderr, "ref_loop: %s is not a %d-D configuration of %d fields: %s\n", argv[1], NDIM, NVAR,
            smaug_vac_last_error());
    return 1;
  }
  size_t N = 1;
  for (int d = 0; d < NDIM; ++d) N *= (size_t)h.n[d];
  double *pos = (double *)malloc(sizeof(double) * NDIM * N), *w = (double *)malloc(sizeof(double) * NVAR * N);
  if (!pos || !w || smaug_vac_read_ascii(argv[1], &h, pos, NDIM * N, w, NVAR * N) != 0) {
    fprintf(stderr, "ref_loop: cannot read %s\n", argv[1]);
    return 1;
  }

  struct params *p = (struct params *)calloc(1, sizeof(struct params));
  struct bparams *bp = NULL;
  struct state *state = (struct state *)calloc(1, sizeof(struct state));
  real *wmod = (real *)calloc(2 * NVAR * N, sizeof(real)), *wd = (real *)calloc(NDERV * N, sizeof(real));
  real *wnew = NULL, *wtemp2 = NULL, *w0 = NULL;
  for (int d = 0; d < NDIM; ++d) {
    const size_t s = d == 0 ? 1 : d == 1 ? (size_t)h.n[0] : (size_t)h.n[0] * h.n[1];
    p->n[d] = h.n[d];
    p->xmin[d] = pos[d * N];
    p->dx[d] = pos[d * N + s] - pos[d * N];
    p->g[d] = h.neqpar > 2 + d ? h.eqpar[2 + d] : 0.0;
    for (int f = 0; f < NVAR; ++f) p->boundtype[f][d][0] = p->boundtype[f][d][1] = bt[d];
  }
  p->gamma = h.eqpar[0];
  p->courant = 0.3;
  p->moddton = 1;
  p->rkon = 0;
  p->hyperdifmom = hyperdif;
  p->divbon = p->divbfix = divbon;
  p->cfgsavefrequency = 1;
  p->readini = 1;
  p->dt = 1.0e-8; /* iosmaug.cpp:327-330 */
  p->chyp[rho] = 0.045;
  p->chyp[energy] = 0.02;
  for (int k = 0; k < NDIM; ++k) {
    p->chyp[mom1 + k] = 0.4;
    p->chyp[b1 + k] = 0.02;
  }
  memcpy(wmod, w, sizeof(real) * NVAR * N);            /* slot 0 */
  memcpy(wmod + NVAR * N, w, sizeof(real) * NVAR * N); /* slot 1 */
  memcpy(wd + pos1 * N, pos, sizeof(real) * NDIM * N);

  struct params *d_p;
  struct bparams *d_bp;
  struct state *d_state;
  real *d_wnew = NULL, *d_wmod, *d_dwn1, *d_wd, *d_wtemp, *d_wtemp1, *d_wtemp2, *d_w = NULL;
  CALL(cuinit(&p, &bp, &wmod, &wnew, &wd, &state, &d_p, &d_bp, &d_wnew, &d_wmod, &d_dwn1, &d_wd, &d_state, &d_wtemp,
              &d_wtemp1, &d_wtemp2));
  CALL(initgrid(&p, &state, &wd, &d_p, &d_dwn1, &d_wd, &d_state, &d_wtemp, &d_wtemp1, &d_wtemp2));
  for (int ii = 0; ii <= (b1 + (NDIM - 1)); ii++)
    for (int idir = 0; idir < NDIM; idir++) CALL(cuboundary(&p, &bp, &d_p, &d_bp, &d_state, &d_wmod, 1, idir, ii));

  int order = 0, ordero = 1;
  double cmax[NDIM];
  for (int n = 1; n <= nt; n++) {
    p->it = n;
    CALL(cucomputedervfields(&p, &d_p, &d_wmod, &d_wd, 0));
    order = 0;
    /* the dt block */
    p->maxcourant = 0.0;
    for (int dim = 0; dim <= (NDIM - 1); dim++) {
      CALL(cucomputec(&p, &d_p, &d_wmod, &d_wd, order, dim));
      CALL(cucomputemaxc(&p, &d_p, &d_wmod, &d_wd, order, dim, &wd, &d_wtemp));
      CALL(cucomputemaxcourant(&p, &d_p, &d_wmod, &d_wd, order, dim, &wd, &d_wtemp));
    }
    if (((p->courant) / (p->maxcourant)) > 1.0e-8) p->dt = (p->courant) / (p->maxcourant);
    if (n > 1) CALL(cugetdtvisc1(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2));
    if ((p->dtdiffvisc) > 1.0e-8 && (p->dt) > ((p->dtdiffvisc))) p->dt = (p->dtdiffvisc);

    /* the single step */
    ordero = 1;
    order = 0;
    for (int dir = 0; dir < NDIM; dir++) CALL(cucomputevels(&p, &d_p, &d_wmod, &d_wd, order, dir));
    for (int dir = 0; dir < NDIM; dir++) {
      for (int f = rho; f <= (mom1 + NDIM - 1); f++) {
        if (f == mom1 + dir) {
          CALL(cucomputept(&p, &d_p, &d_wmod, &d_wd, order, dir));
          CALL(cucomputepbg(&p, &d_p, &d_wmod, &d_wd, order, dir));
        }
        CALL(cucentdiff1(&p, &d_p, &d_state, &d_wmod, &d_wmod, &d_dwn1, &d_wd, order, ordero, p->dt, f, dir));
      }
      for (int f = energy; f <= (b1 + (NDIM - 1)); f++) {
        if (f == energy) {
          CALL(cucomputevels(&p, &d_p, &d_wmod, &d_wd, order, dir));
          CALL(cucomputepbg(&p, &d_p, &d_wmod, &d_wd, ordero, dir));
          CALL(cucomputept(&p, &d_p, &d_wmod, &d_wd, order, dir));
        }
        CALL(cucentdiff2(&p, &d_p, &d_state, &d_wmod, &d_wmod, &d_dwn1, &d_wd, order, ordero, p->dt, f, dir));
      }
    }
    CALL(cugrav(&p, &d_p, &d_state, &d_wmod, &d_wmod, &d_dwn1, &d_wd, order, ordero, p->dt));
    if (p->divbon == 1) CALL(cudivb(&p, &d_p, &d_w, &d_wmod, &d_dwn1, &d_wd, order, ordero, p->dt));
    if (p->hyperdifmom == 1) {
      const double dt = p->dt;
      p->maxviscoef = 0.0;
      CALL(cunushk1(&p, &d_p, &d_wmod, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2));
      for (int dim = 0; dim <= (NDIM - 1); dim++) { /* density */
        CALL(cucomputec(&p, &d_p, &d_wmod, &d_wd, order, dim));
        CALL(cucomputemaxc(&p, &d_p, &d_wmod, &d_wd, order, dim, &wd, &d_wtemp));
        cmax[dim] = p->cmax;
        CALL(cuhyperdifvisc1ir(&p, &d_p, &d_wmod, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, rho, dim));
        CALL(cuhyperdifvisc1r(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, rho, dim));
        CALL(cuhyperdifvisc1l(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, rho, dim));
        CALL(cuhyperdifrhosource1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, rho, dim, p->dt));
      }
      for (int dim = 0; dim <= (NDIM - 1); dim++) { /* energy */
        p->cmax = cmax[dim];
        CALL(cuhyperdifvisc1ir(&p, &d_p, &d_wmod, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, energy, dim));
        CALL(cuhyperdifvisc1r(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, energy, dim));
        CALL(cuhyperdifvisc1l(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, energy, dim));
        CALL(cuhyperdifesource1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, energy, dim, dt));
      }
      for (int dim = 0; dim <= (NDIM - 1); dim++) /* momentum */
        for (int f = 0; f <= (NDIM - 1); f++) {
          p->cmax = cmax[dim];
          CALL(cuhyperdifvisc1ir(&p, &d_p, &d_wmod, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, mom1 + f, dim));
          CALL(cuhyperdifvisc1r(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, mom1 + f, dim));
          CALL(cuhyperdifvisc1l(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, mom1 + f, dim));
          for (int ii1 = 0; ii1 <= 1; ii1++) {
            const int ii = ii1 == 0 ? dim : f, ii0 = ii1 == 0 ? f : dim;
            if (ii == dim)
              CALL(cuhyperdifmomsource1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, f, dim, ii, ii0,
                                        p->dt));
            else
              CALL(cuhyperdifmomsourcene1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, f, dim, ii,
                                          ii0, p->dt));
          }
        }
      for (int dim = 0; dim <= (NDIM - 1); dim++) /* magnetic field */
        for (int f = 0; f <= (NDIM - 1); f++) {
          if (f == dim) continue;
          p->cmax = cmax[dim];
          CALL(cuhyperdifvisc1ir(&p, &d_p, &d_wmod, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, b1 + f, dim));
          CALL(cuhyperdifvisc1r(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, b1 + f, dim));
          CALL(cuhyperdifvisc1l(&p, &d_p, &d_wmod, &wd, &d_wd, order, &d_wtemp, &d_wtemp1, &d_wtemp2, b1 + f, dim));
          for (int ii1 = 0; ii1 <= 1; ii1++) {
            const int jj = ii1 == 0 ? dim : f, mm = ii1 == 0 ? f : dim, ii0 = ii1 == 0 ? dim : f;
            const real sb = ii1 == 0 ? -1.0 : 1.0;
            if (mm == dim)
              CALL(cuhyperdifbsource1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, f, dim, jj, ii0, mm,
                                      sb, p->dt));
            else
              CALL(cuhyperdifbsourcene1(&p, &d_p, &d_wmod, &d_dwn1, &d_wd, order, ordero, &d_wtemp, f, dim, jj, ii0,
                                        mm, sb, p->dt));
          }
        }
    }
    CALL(cusource(&p, &d_p, &d_state, &d_w, &d_wmod, &d_dwn1, &d_wd, order, ordero, p->dt));
    for (int ii = 0; ii <= (b1 + (NDIM - 1)); ii++)
      for (int idir = 0; idir < NDIM; idir++)
        CALL(cuboundary(&p, &bp, &d_p, &d_bp, &d_state, &d_wmod, ordero, idir, ii));
  }
  CALL(cuupdate(&p, &w0, &wmod, &wtemp2, &state, &d_p, &d_w, &d_wmod, &d_wtemp2, &d_state, nt));
  CALL(cusync(&p));
  h.it = nt;
  if (smaug_vac_write_binary(argv[3], &h, pos, wmod + NVAR * N) != 0) {
    fprintf(stderr, "ref_loop: cannot write %s: %s\n", argv[3], smaug_vac_last_error());
    return 1;
  }
  printf("dt %.17g maxviscoef %.17g\n", p->dt, p->maxviscoef);
  CALL(cufinish(&p, &w0, &wnew, &state, &d_p, &d_bp, &d_w, &d_wnew, &d_wmod, &d_dwn1, &d_wd, &d_state, &d_wtemp,
                &d_wtemp1, &d_wtemp2));
  free(p);
  free(state);
  free(wmod);
  free(wd);
  free(pos);
  free(w);
  return 0;
}
