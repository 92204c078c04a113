/*
 * smaug_oracle.h -- CPU restatement of the SMAUG/SAC ideal-MHD step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  It is never part of the product path.
 *
 * Layout (identical to the reference's wmod slot, iotypes.h:213-219):
 *   w[f * N + idx],  idx = (k * n1 + j) * n0 + i   (x fastest),
 *   N = n0 * n1 * n2 cells INCLUDING 2 ghost layers per side;
 *   2-D fields: rho m1 m2 e b1 b2 eb rhob b1b b2b            (NVAR = 10)
 *   3-D fields: rho m1 m2 m3 e b1 b2 b3 eb rhob b1b b2b b3b  (NVAR = 13)
 * Metric: delx[d][idx] = cell width along d at cell idx, the reference's
 * per-cell wd[delx1+d] as initgrid computes it (init.cu:1118-1670).
 */
#ifndef SMAUG_ORACLE_H
#define SMAUG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Momentum driver: the reference's user source term (addsourceterms2,
 * models/usersource.cu.spicule1:4-137, applied by cusource after the other
 * terms of a step, iosmaug.cpp:1153).  At every cell of the updated state:
 *   m_dir += h * vvz * (rho + rhob),  vvz = amp * F * tdep,
 *   F = f1 * f0 (2-D) or (f1 * f0) * f2 (3-D),
 *   f_d = exp(-(x_d - center_d)^2 / (width_d * width_d)), 1 where width_d = 0,
 *   x_d = xmin_d + i_d * dx_d,
 *   tdep = sin(2 pi t / period) (the model's commented time dependence), or 1
 *   when period = 0 (the model's choice).
 * The reference model applies it on the first iteration only (p->it == 1); a
 * run of one step compares like for like.
 */
typedef struct {
  int on;
  int dir;
  double amp, period;
  double center[3], width[3], xmin[3], dx[3];
} sm_oracle_driver;

typedef struct {
  int ndim;            /* 2 or 3 */
  int n[3];            /* cells per dim incl. ghosts (n[2] = 1 in 2-D) */
  double gamma;
  double chyp[13];     /* hyperdiffusion coefficient per field id */
  int btype[3];        /* per dim (iotypes.h:145): 0 periodic, 3 cont, 4 contcd4,
                          5 fixed, 6 symm, 7 asymm */
  double g[3];         /* gravity per dim */
  double courant;
  int hyperdif;        /* 1: hyperdiffusion sources on (p->hyperdifmom) */
  const double *delx[3];
  const sm_oracle_driver *drv;  /* NULL: no driver */
  int bmask[3];        /* per dim: evolved fields (bit f) that take asymm where btype is symm */
  const double *fixed; /* fixed (5) boundaries: the state as loaded (NVAR * N), or NULL */
  int divb;            /* 2-D: divergence-of-B source terms (p->divbon, p->divbfix) */
  double dxs[3];       /* p->dx: the uniform spacing the divB gradient divides by */
} sm_oracle_grid;

/* Per-run scalars carried between steps (p->dt, p->dtdiffvisc, p->maxviscoef). */
typedef struct {
  double dt;
  double dtdiffvisc;
  double maxviscoef;
  double maxcourant;
  double cmax[3];
  double t;            /* simulation time at the start of the next step */
} sm_oracle_state;

int sm_oracle_nvar(int ndim);

/* Fast magnetosonic speed per cell along dim (computec3, dervfields.cu:241-309). */
void sm_oracle_cfast(const sm_oracle_grid *g, const double *w, int dim, double *cf);

/* cmax per dim as cucomputemaxc finds it (max over all cells, from 0). */
void sm_oracle_cmax(const sm_oracle_grid *g, const double *w, double *cmax);

/*
 * dt selection of the reference host loop for moddton==1
 * (iosmaug.cpp:855-898 with cucomputemaxcourant and cugetdtvisc1).  step is
 * the loop index n; the viscous limit is evaluated for n > 1 only.
 */
double sm_oracle_select_dt(const sm_oracle_grid *g, const double *w, int step, sm_oracle_state *s);

/*
 * One stage: wout = wbase + h * L(win), then the ghost fill of wout.
 * L is the reference's single-step operator (iosmaug.cpp:904-1166).  With
 * wbase == win this is exactly one reference step.  cmax[d] are the hyperdiffusion
 * wave speeds of win.  Returns the largest hyperviscosity coefficient used.
 * wout must not alias win; it may alias wbase.
 */
double sm_oracle_stage(const sm_oracle_grid *g, const double *win, const double *wbase,
                       double *wout, double h, const double *cmax);
/* The same stage with the driver (if any) evaluated at time tin. */
double sm_oracle_stage_t(const sm_oracle_grid *g, const double *win, const double *wbase,
                         double *wout, double h, const double *cmax, double tin);

/* Ghost fill of the evolved fields, field by field and direction by direction
 * (iosmaug.cpp:1157-1166): periodic and contcd4 as models/boundary.cu.sedov3d,
 * cont, fixed, symm and asymm as the per-direction helpers of src/gradops.cu. */
void sm_oracle_boundary(const sm_oracle_grid *g, double *w);

/*
 * One full step.  rk4 = 0: the reference single step; rk4 = 1: SAC's
 * classical four-step Runge-Kutta (dev/sac/src/vac.t:447-462) around the
 * same operator.  dt_mode = 1 selects dt as the reference does, 0 keeps s->dt.
 * work must hold 4 * NVAR * N doubles.  step is the 1-based step index.
 * The driver's stage times are t, t + dt/2, t + dt/2, t + dt (RK4) or t;
 * s->t advances by dt.
 */
int sm_oracle_step(const sm_oracle_grid *g, double *w, int step, int rk4, int dt_mode,
                   sm_oracle_state *s, double *work);

#ifdef __cplusplus
}
#endif
#endif
