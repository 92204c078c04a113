/*
 * smaug_cukernels.h -- the reference's per-operator GPU entry points, for a
 * host loop written against them.
 *
 * The reference's host loop (dev/smaug/src/iosmaug.cpp:802-1166) drives its
 * step through ~35 `int cu*(struct params **p, ...)` functions declared in
 * dev/smaug/include/smaugcukernels.h:8-65, passing the run parameters
 * (struct params) and device pointers to its work arrays: wmod (the state
 * slots), wd (the derived fields), wtemp (temporaries).  This header declares
 * those functions with the same names, argument lists and struct layouts, and
 * libsmaug_cu2d.so / libsmaug_cu3d.so (smaug-all_b200/csrc/smaug_cucompat.cu,
 * one library per SMAUG_CU_NDIM, as the reference is built for one NDIM)
 * implement them.  A host loop of the reference's shape links against them
 * unchanged.
 *
 * Each function does what the reference's does, per operator, in FP64, with
 * the same outputs in the same arrays: the state slots of wmod, the derived
 * fields of wd (velocities, pressures, wave speeds, hyperviscosities), the
 * scalars of struct params (cmax, maxcourant, maxviscoef, dtdiffvisc).  The
 * kernels are built without FMA contraction and restate the reference's
 * arithmetic in its operation order, so a host loop driven through them
 * gives the reference's bits (the library's tests compare a loop of the
 * reference's shape with the CPU oracle bit for bit).  Stated differences:
 *   - cuinit takes the initial state from the host's wmod; the model's device
 *     initialiser (init_parallel and init_user) is not run;
 *   - one boundary type per direction: boundtype[0][dir][0] (the density's)
 *     selects the gradient zero rules and the ghost fill of every field;
 *   - the derived fields a function needs are recomputed from the state slot
 *     it is given (the reference's host loop computes them just before with
 *     cucomputevels / cucomputept / cucomputepbg from the same slot, so the
 *     values are the same); those functions still fill wd;
 *   - maxviscoef is the running maximum over all steps that the reference
 *     ends up with (its host loop zeroes p->maxviscoef before the
 *     hyperdiffusion block; the device-to-host params copy of the next
 *     cucomputec restores it): cucomputec and the hyperviscosity functions
 *     write that running maximum into p->maxviscoef;
 *   - cusource is the default model's (no source term); cunushk1 stores
 *     nothing, as the reference's shock viscosity (nushk1.cu:339-343).
 * Every function returns 0, or a negative SMAUG_ERR_* status (include/
 * smaug_b200.h) where the reference would have failed silently; the message
 * is in smaug_cu_last_error().  All work is synchronous, on the legacy
 * default stream, as in the reference.
 */
#ifndef SMAUG_CUKERNELS_H
#define SMAUG_CUKERNELS_H

#ifndef SMAUG_CU_NDIM
#define SMAUG_CU_NDIM 2
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* iotypes.h:1-45: FP64 reals; the sizes of the work arrays */
typedef double real;
#define NVECDIM SMAUG_CU_NDIM
#define NDIM SMAUG_CU_NDIM
#if SMAUG_CU_NDIM == 2
#define NVAR 10
#define NDERV 19
#elif SMAUG_CU_NDIM == 3
#define NVAR 13
#define NDERV 23
#else
#error "SMAUG_CU_NDIM must be 2 or 3"
#endif
#define NTEMP 8
#define NTEMP1 2
#define NTEMP2 1

/* iotypes.h:213-246: field ids of wmod slots, wd and the temporaries */
#if SMAUG_CU_NDIM == 2
typedef enum vars { rho, mom1, mom2, energy, b1, b2, energyb, rhob, b1b, b2b } CEV;
typedef enum dvars {
  vel1, vel2, flux, hdnur, hdnul, nushk1, nushk2, soundspeed, pressuret, pressurek, bdotv, divb, cfast, ptb, pkb,
  pos1, pos2, delx1, delx2
} DEV;
#else
typedef enum vars { rho, mom1, mom2, mom3, energy, b1, b2, b3, energyb, rhob, b1b, b2b, b3b } CEV;
typedef enum dvars {
  vel1, vel2, vel3, flux, hdnur, hdnul, nushk1, nushk2, nushk3, soundspeed, pressuret, pressurek, bdotv, divb,
  cfast, ptb, pkb, pos1, pos2, pos3, delx1, delx2, delx3
} DEV;
#endif
typedef enum tempvars { tmp1, tmp2, tmp3, tmp4, tmp5, tmp6, tmp7, tmp8 } TEV;

/* struct params, iotypes.h:86-179 (single-process layout) */
struct params {
  int n[NDIM];
  int ng[NDIM];
  int npgp[NDIM];
  int fullgridini;
  real hdmean, hdmax, pmax, pmin, pmean, emax, emin, emean;
  real xmax[NDIM];
  real xmin[NDIM];
  int nt;
  int it;
  real tmax;
  real qt;
  real boundu[NDIM][NVAR];
  real boundl[NDIM][NVAR];
  real cmax;
  real maxcourant;
  int steeringenabled;
  int finishsteering;
  real dt;
  real dx[NDIM];
  real gamma;
  real mu;
  real eta;
  real g[NDIM];
  int sodifon;
  int rkon;
  int moddton;
  int divbon;
  int divbfix;
  int cfgsavefrequency;
  int hyperdifmom;
  int mode;
  int readini;
  real courant;
  real maxviscoef;
  real dtdiffvisc;
  real chyp[NVAR];
  real chyp3;
  real test;
  int boundtype[NVAR][NDIM][2]; /* 0 periodic, 3 cont, 4 contcd4, 5 fixed, 6 symm, 7 asymm */
  int gpid[16];
  int npe;
  int noghost;
};

/* struct state, iotypes.h:182-194 */
struct state {
  int it;
  real t, dt, rho, m1, m2, m3, e, b1, b2, b3;
};

/* struct bparams, iobparams.h:1-32: the loaded values of fixed boundaries */
#define MSIZE1 128
#define MSIZE2 128
#define MSIZE3 128
struct bparams {
#if SMAUG_CU_NDIM == 3
  real fixed1[4 * MSIZE2 * MSIZE3 * NVAR];
  real fixed2[4 * MSIZE1 * MSIZE3 * NVAR];
  real fixed3[4 * MSIZE1 * MSIZE2 * NVAR];
#else
  real fixed1[4 * MSIZE2 * NVAR];
  real fixed2[4 * MSIZE1 * NVAR];
#endif
};

/* set-up and data movement (init.cu:816-1670, update.cu:162-235) */
int cuinit(struct params **p, struct bparams **bp, real **wmod, real **wnew, real **wd, struct state **state,
           struct params **d_p, struct bparams **d_bp, real **d_wnew, real **d_wmod, real **d_dwn1, real **d_wd,
           struct state **d_state, real **d_wtemp, real **d_wtemp1, real **d_wtemp2);
int initgrid(struct params **p, struct state **state, real **wd, struct params **d_p, real **d_dwn1, real **d_wd,
             struct state **d_state, real **d_wtemp, real **d_wtemp1, real **d_wtemp2);
int cuupdate(struct params **p, real **w, real **wmod, real **wtemp2, struct state **state, struct params **d_p,
             real **d_w, real **d_wmod, real **d_wtemp2, struct state **d_state, int step);
int cufinish(struct params **p, real **w, real **wnew, struct state **state, struct params **d_p,
             struct bparams **d_bp, real **d_w, real **d_wnew, real **d_wmod, real **d_dwn1, real **d_wd,
             struct state **d_state, real **d_wtemp, real **d_wtemp1, real **d_wtemp2);
int cusync(struct params **p);

/* ghost cells (boundary.cu, gradops.cu:833-1625) and the RK slot algebra (advance.cu) */
int cuboundary(struct params **p, struct bparams **bp, struct params **d_p, struct bparams **d_bp,
               struct state **d_s, real **d_wmod, int order, int idir, int field);
int cuadvance(struct params **p, struct params **d_p, real **d_wmod, real **d_w, int order);

/* derived fields and the dt block (computedervfields.cu, nushk1.cu) */
int cucomputedervfields(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order);
int cucomputevels(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir);
int cucomputemaxc(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir, real **wd,
                  real **d_wtemp);
int cucomputemaxcourant(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir,
                        real **wd, real **d_wtemp);
int cucomputec(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir);
int cucomputept(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir);
int cucomputepk(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir);
int cucomputepbg(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, int dir);
int cugetdtvisc1(struct params **p, struct params **d_p, real **d_wmod, real **wd, real **d_wd, int order,
                 real **d_wtemp, real **d_wtemp1, real **d_wtemp2);

/* fluxes and sources (centdiff1.cu, centdiff2.cu, divb.cu, usersource) */
int cucentdiff1(struct params **p, struct params **d_p, struct state **d_s, real **d_w, real **d_wmod,
                real **d_dwn1, real **d_wd, int order, int ordero, real dt, int field, int dir);
int cucentdiff2(struct params **p, struct params **d_p, struct state **d_s, real **d_w, real **d_wmod,
                real **d_dwn1, real **d_wd, int order, int ordero, real dt, int field, int dir);
int cugrav(struct params **p, struct params **d_p, struct state **d_s, real **d_w, real **d_wmod, real **d_dwn1,
           real **d_wd, int order, int ordero, real dt);
int cusource(struct params **p, struct params **d_p, struct state **d_s, real **d_w, real **d_wmod, real **d_dwn1,
             real **d_wd, int order, int ordero, real dt);
int cudivb(struct params **p, struct params **d_p, real **d_w, real **d_wmod, real **d_dwn1, real **d_wd, int order,
           int ordero, real dt);

/* hyperdiffusion (hyperdifvisc1r.cu, hyperdifvisc1l.cu, hyperdif*source*.cu, nushk1.cu) */
int cunushk1(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, real **d_wtemp,
             real **d_wtemp1, real **d_wtemp2);
int cuhyperdifvisc1ir(struct params **p, struct params **d_p, real **d_wmod, real **d_wd, int order, real **d_wtemp,
                      real **d_wtemp1, real **d_wtemp2, int field, int dim);
int cuhyperdifvisc1r(struct params **p, struct params **d_p, real **d_wmod, real **wd, real **d_wd, int order,
                     real **d_wtemp, real **d_wtemp1, real **d_wtemp2, int field, int dim);
int cuhyperdifvisc1l(struct params **p, struct params **d_p, real **d_wmod, real **wd, real **d_wd, int order,
                     real **d_wtemp, real **d_wtemp1, real **d_wtemp2, int field, int dim);
int cuhyperdifrhosource1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd,
                         int order, int ordero, real **d_wtemp, int field, int dim, real dt);
int cuhyperdifesource1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd, int order,
                       int ordero, real **d_wtemp, int field, int dim, real dt);
int cuhyperdifmomsource1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd,
                         int order, int ordero, real **d_wtemp, int field, int dim, int ii, int ii0, real dt);
int cuhyperdifmomsourcene1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd,
                           int order, int ordero, real **d_wtemp, int field, int dim, int ii, int ii0, real dt);
int cuhyperdifbsource1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd, int order,
                       int ordero, real **d_wtemp, int field, int dim, int jj, int ii0, int mm, real sb, real dt);
int cuhyperdifbsourcene1(struct params **p, struct params **d_p, real **d_wmod, real **d_dwn1, real **d_wd,
                         int order, int ordero, real **d_wtemp, int field, int dim, int jj, int ii0, int mm, real sb,
                         real dt);

/* The message of the last failed call (this library's addition). */
const char *smaug_cu_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
