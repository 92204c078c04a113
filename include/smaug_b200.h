/*
 * smaug_b200.h -- C ABI of the B200 ideal-MHD step (SAC/SMAUG method).
 *
 * The reference drives its GPU step through ~35 per-operator entry points
 * declared in dev/smaug/include/smaugcukernels.h (cuinit, cucentdiff1,
 * cuhyperdifvisc1r, cuboundary, ...), called in sequence by the host loop
 * dev/smaug/src/iosmaug.cpp:802-1550.  This library exposes the same step at
 * the granularity a host loop needs, with plain pointers and sizes only:
 *
 *   smaug_create        replaces cuinit            (init.cu:816-1000)
 *   smaug_set_metric    replaces initgrid          (init.cu:1118-1670)
 *   smaug_set_state     replaces cuinit's H2D copy + the initial cuboundary
 *                       pass                       (iosmaug.cpp:786-794)
 *   smaug_step          replaces one loop iteration: cucomputedervfields,
 *                       the moddton dt block (cucomputec / cucomputemaxc /
 *                       cucomputemaxcourant / cugetdtvisc1), cucentdiff1/2,
 *                       cugrav, the hyperdiffusion chains (cuhyperdifvisc1r/l
 *                       + cuhyperdif*source*), cusource and cuboundary
 *                                                  (iosmaug.cpp:802-1166)
 *   smaug_get_state     replaces cuupdate          (update.cu:162-235)
 *   smaug_get_scalars   replaces reading p->dt, p->cmax, p->maxcourant,
 *                       p->maxviscoef, p->dtdiffvisc back from struct params
 *   smaug_destroy       replaces cufinish          (init.cu, never called by
 *                       the reference)
 *
 * Storage (same as the reference's wmod slot, iotypes.h:213-219): host state
 * buffers hold NVAR fields, field-major, x fastest, each of N cells
 * including two ghost layers per side:
 *   2-D: rho m1 m2 e b1 b2 eb rhob b1b b2b              NVAR = 10
 *   3-D: rho m1 m2 m3 e b1 b2 b3 eb rhob b1b b2b b3b    NVAR = 13
 *
 * Errors: every function returns SMAUG_OK (0) or a negative status and never
 * aborts (the reference's int-returning wrappers have no return value at
 * all); smaug_last_error() describes the last failure.  All work of one
 * context is ordered on one CUDA stream; one host thread per context.
 */
#ifndef SMAUG_B200_H
#define SMAUG_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SMAUG_OK = 0,
  SMAUG_ERR_ARG = -1,      /* invalid argument or size */
  SMAUG_ERR_CUDA = -2,     /* CUDA runtime error */
  SMAUG_ERR_STATE = -3,    /* call out of order (e.g. step before set_state) */
  SMAUG_ERR_NONFINITE = -4, /* dt or a reduction became NaN/Inf */
  SMAUG_ERR_FULL = -5       /* batch: no free slot or arena block for a simulation */
};

/*
 * Boundary types per direction (iotypes.h:145 boundtype codes).  The ghosts
 * are filled field by field, direction by direction (iosmaug.cpp:1157-1166):
 *   PERIODIC  wrap (models/boundary.cu.sedov3d)
 *   CONT      copies of the first/last inner cell (bc3_cont_dir, gradops.cu)
 *   CONTCD4   0 <- 4, 1 <- 3, n-1 <- n-5, n-2 <- n-4 (boundary.cu.sedov3d)
 *   FIXED     the values of the loaded state (bc3_setfixed_dir at it = -1,
 *             bc3_fixed_dir; iosmaug.cpp:645-654); as in the reference, a
 *             fixed direction also keeps the outermost ghost layer of every
 *             earlier direction at its loaded values
 *   SYMM      mirror (bc3_symm_dir; 2-D about the boundary face, 3-D about
 *             the first inner cell, as the reference's 2-D and 3-D branches)
 *   ASYMM     the mirror negated (bc3_asymm_dir)
 * The reference keeps a type per field; here a type per direction applies to
 * every evolved field, except that the fields in bmask[d] take ASYMM where
 * btype[d] is SYMM (a reflecting wall: the normal momentum and field flip).
 */
enum {
  SMAUG_BC_PERIODIC = 0,
  SMAUG_BC_CONT = 3,
  SMAUG_BC_CONTCD4 = 4,
  SMAUG_BC_FIXED = 5,
  SMAUG_BC_SYMM = 6,
  SMAUG_BC_ASYMM = 7
};

/*
 * Arithmetic of the step.  The reference computes everything in FP64 (real =
 * double, iotypes.h).  SMAUG_PREC_MIXED (no counterpart in the reference)
 * keeps the stage states and the stencil arithmetic in FP32 and FP64 where
 * accuracy needs it: background fields, total pressure and internal energy
 * (recovered by cancellation), the RK base state (an FP32 value plus an FP32
 * compensation), the RK combination and the dt reductions.  Needs rk4 = 1 and
 * exact = 0; host buffers stay FP64.
 */
enum { SMAUG_PREC_FP64 = 0, SMAUG_PREC_MIXED = 1 };

typedef struct smaug_ctx smaug_ctx;

typedef struct {
  int ndim;         /* 2 or 3 */
  int n[3];         /* cells per dim INCLUDING 2+2 ghost layers (n[2] = 1 in 2-D) */
  double gamma;     /* p->gamma */
  double courant;   /* p->courant */
  double chyp[13];  /* p->chyp, indexed by field id (layout above) */
  int btype[3];     /* per dim, SMAUG_BC_*; every evolved field, both sides (bmask below) */
  double g[3];      /* p->g */
  int hyperdif;     /* p->hyperdifmom: 1 = hyperdiffusion sources on */
  int rk4;          /* 1: classical four-stage RK (SAC fourstep); 0: single step (rkon=0) */
  int dt_mode;      /* 1: dt from the reference's moddton rule; 0: fixed dt = dt0 */
  double dt0;       /* initial dt (1e-8 when dt_mode = 1, iosmaug.cpp:327-330) */
  int exact;        /* 1: kernels built without FMA contraction (bit-reproducible) */
  int precision;    /* SMAUG_PREC_FP64 (default, 0) or SMAUG_PREC_MIXED */
  /*
   * Momentum driver (the reference's user source term, addsourceterms2 of
   * models/usersource.cu.spicule1:4-137, applied by cusource at
   * iosmaug.cpp:1153): after each stage's update, at every cell,
   *   m_dir += h * (drv_amp * F(x) * tdep(t)) * (rho + rhob)
   * with F the product over dims of exp(-(x_d - drv_center[d])^2 /
   * drv_width[d]^2) (1 along a dim whose width is 0), x_d = xmin[d] + i_d *
   * dx[d] (the reference's p->xmin, p->dx), and tdep = sin(2 pi t /
   * drv_period), or 1 when drv_period = 0 (the reference model's choice).
   * t is the stage's input time.  drv_on = 0 switches it off.
   */
  int drv_on;
  int drv_dir;            /* driven momentum component, 0 .. ndim-1 */
  double drv_amp;
  double drv_period;
  double drv_center[3];
  double drv_width[3];
  double xmin[3];         /* coordinate of cell 0 (a ghost) per dim */
  double dx[3];           /* grid spacing per dim */
  int bmask[3];           /* per dim: evolved fields (bit = field id) that take
                             SMAUG_BC_ASYMM where btype is SMAUG_BC_SYMM */
  /*
   * 1: the divergence-of-B source terms of cudivb (divb.cu:165-336, the
   * reference's divbon = divbfix = 1), after gravity: -divB (0, B, B.v, v)
   * with divB the 4th-order difference over the spacing dx[] above.  2-D
   * only (the reference's 3-D kernel reads an uninitialised bound).
   */
  int divb;
} smaug_params;

/* Number of fields for ndim (10 or 13). */
int smaug_nvar(int ndim);

int smaug_create(const smaug_params *prm, int device, smaug_ctx **out);
int smaug_destroy(smaug_ctx *ctx);

/*
 * Metric: ndim arrays of N doubles (cell widths along each dim at every cell,
 * the reference's wd[delx1..delx3] after initgrid), concatenated.
 */
int smaug_set_metric(smaug_ctx *ctx, const double *delx, size_t count);

/* Host state in/out: NVAR * N doubles (layout above).  Synchronous. */
int smaug_set_state(smaug_ctx *ctx, const double *w, size_t count);
int smaug_get_state(smaug_ctx *ctx, double *w, size_t count);

/* Device-resident variants: w points to NVAR * N doubles in device memory;
 * the copy is ordered on the context stream and not waited for. */
int smaug_set_state_device(smaug_ctx *ctx, const double *w_dev, size_t count);
int smaug_get_state_device(smaug_ctx *ctx, double *w_dev, size_t count);

/* Advance nsteps full steps (asynchronous on the context stream). */
int smaug_step(smaug_ctx *ctx, int nsteps);

/*
 * The same on the caller's CUDA stream (a cudaStream_t; NULL: the context
 * stream): the steps wait for all work queued on the context before, and
 * later context work waits for them, so the caller can order the steps
 * against its own kernels and copies without a host sync.  Like the
 * reference's per-step launch sequence (iosmaug.cpp:802-1166), but one call.
 */
int smaug_step_on(smaug_ctx *ctx, int nsteps, void *stream);

/*
 * One Runge-Kutta stage of the current step on the caller's stream (NULL:
 * the context stream): stages 1..4 in order with rk4 = 1 (stage 1 first
 * takes the step's dt, stage 4 finishes the step), stage 1 alone with
 * rk4 = 0.  Calling stages 1..4 is the same work, with the same results, as
 * smaug_step(ctx, 1); a host loop that interleaves its own work between the
 * stages uses this.  Out-of-order stages return SMAUG_ERR_STATE, as does
 * smaug_step while a step begun here is unfinished.  The granularity of the
 * reference's cuadvance stage slots (advance.cu:18-174) over the fused
 * operator.
 */
int smaug_stage(smaug_ctx *ctx, int stage, void *stream);

/*
 * The metric from cell positions (host only), replacing initgrid
 * (init.cu:1118-1670): pos holds ndim arrays of N doubles, the position
 * components of every cell including ghosts (the reference's wd[pos1..] as
 * set by init_parallel or read from a VAC file); dx the spacing per dim (it
 * replaces a zero difference).  delx receives ndim arrays of N doubles for
 * smaug_set_metric: the positions extrapolated linearly over two layers and a
 * pad on each side, then centrally differenced, as the reference does.
 * Errors: SMAUG_ERR_ARG with smaug_vac_last_error().
 */
int smaug_initgrid(int ndim, const int *n, const double *pos, const double *dx, double *delx);

/* Wait for all queued work; returns the first device-side error if any. */
int smaug_sync(smaug_ctx *ctx);

/*
 * out[0] dt of the last step, [1] maxcourant, [2] maxviscoef (running),
 * [3] dtdiffvisc, [4..6] cmax per dim of the current state,
 * [7] steps taken.  Synchronous.
 */
int smaug_get_scalars(smaug_ctx *ctx, double out[8]);

/*
 * Stage timing: when enabled, CUDA events bracket every stage kernel launch;
 * smaug_stage_times waits, returns the summed device time (ms) and the number
 * of timed launches since the last call, and resets.  (The reference's only
 * timing is the per-step wall clock printf, iosmaug.cpp:1515-1517.)
 */
int smaug_profile_stages(smaug_ctx *ctx, int enable);
int smaug_stage_times(smaug_ctx *ctx, double *ms_total, long long *count);

/*
 * smaug_step_noalloc -- no counterpart in the reference.
 *
 * One call advances a state by nsteps steps without allocating any device
 * memory, for callers that cannot call cudaMalloc: a framework whose caching
 * allocator owns the GPU's memory (a raw cudaMalloc would then fail or
 * fragment it), code that must not allocate once its set-up is done (a
 * real-time or serving loop with a fixed memory budget), or a host that only
 * holds device pointers handed to it by someone else.
 *
 * The caller passes everything by device pointer: the metric (ndim * N
 * doubles, as for smaug_set_metric), the input state and the output state
 * (NVAR * N doubles each, layout above; w_out may equal w_in).  The
 * Runge-Kutta stage buffers and the device-side scalars live in a file-scope
 * device array of SMAUG_NOALLOC_SCRATCH_BYTES that every GPU which loads the
 * library holds until the process exits.  Grids whose scratch would not fit
 * (3 * (2 + 2*ndim) * N doubles plus the metric lines, the scalars and a
 * 1-simulation descriptor for the stage kernel) are
 * rejected with SMAUG_ERR_ARG and a message in err.
 *
 * Each call starts afresh from w_in (dt from dt0 / the reference's dt rule,
 * counters cleared); the scratch keeps the previous call's contents, so calls
 * whose work overlaps on the GPU (different streams, other threads) race on
 * it and must be serialised by the caller.  The first call on a device looks
 * up the scratch address (cudaGetSymbolAddress).  Every call blocks: it
 * checks the metric on the device and waits for that check before it writes
 * anything (a bad metric returns SMAUG_ERR_ARG with w_out untouched, also
 * when w_out == w_in), copies small tables from host memory, and waits for
 * its stream before returning.  So it must not be called while its stream,
 * or (in global capture mode) any stream of the calling thread, is being
 * captured into a CUDA graph.  scalars_out (8 doubles, as smaug_get_scalars,
 * may be NULL) and err (may be NULL) are host buffers.  FP64 only: precision
 * must be SMAUG_PREC_FP64.
 */
#define SMAUG_NOALLOC_SCRATCH_BYTES (32u << 20)
int smaug_step_noalloc(const smaug_params *prm, const double *delx_dev, const double *w_in_dev,
                       double *w_out_dev, int nsteps, void *stream, double *scalars_out, char *err,
                       size_t errlen);

/*
 * Batches -- no counterpart in the reference (one SMAUG process runs one
 * simulation).  A batch holds many independent simulations of one ndim and
 * one precision, each of its own size and parameters, in one device arena
 * allocated at creation.  smaug_batch_step advances every simulation that
 * still has steps left by one RK4 step per step: one launch per RK stage for
 * all of them (a persistent kernel over a (simulation, tile) work list),
 * replayed from CUDA graphs.  Each simulation keeps its own dt (the
 * reference's rule, or fixed), maxima and status; its results are the same
 * as those of a context with the same smaug_params (the same kernel
 * arithmetic).  Simulations are added and removed between calls, on the
 * batch's stream; a finished simulation stops taking steps on the device.
 * All simulations use rk4 = 1 and exact = 0.
 */
typedef struct smaug_batch smaug_batch;

/* Arena bytes one simulation of these parameters takes (host only). */
int smaug_batch_footprint(const smaug_params *prm, size_t *bytes);

int smaug_batch_create(int ndim, int precision, int device, size_t arena_bytes, int max_sims,
                       smaug_batch **out);
int smaug_batch_destroy(smaug_batch *b);

/*
 * Admit a simulation: prm as for smaug_create (ndim and precision those of
 * the batch), delx as for smaug_set_metric, w as for smaug_set_state (host
 * buffers, copied before the call returns), nsteps = RK4 steps to take.
 * Returns SMAUG_ERR_FULL when no slot or no arena block is free, and
 * SMAUG_ERR_ARG for a metric that is not a tensor-product grid on the inner
 * cells or has a non-positive entry (checked on the device, in the slot's own
 * memory, which is released again).  The admission runs on a stream of its
 * own and waits only for its own copies and checks, not for the steps queued
 * on the batch; the next smaug_batch_step waits for it on the device.
 */
int smaug_batch_add(smaug_batch *b, const smaug_params *prm, const double *delx, const double *w,
                    long long nsteps, int *slot);
/* Remove a simulation.  Its slot and arena block become free for a new
 * admission once the steps and reads queued before the removal are done
 * (smaug_batch_add waits for them only when nothing else is free). */
int smaug_batch_remove(smaug_batch *b, int slot);

/* Enqueue nsteps batch steps (asynchronous). */
int smaug_batch_step(smaug_batch *b, int nsteps);

/* Steps left per slot (n >= max_sims entries; -1 for a free slot).  Waits. */
int smaug_batch_poll(smaug_batch *b, long long *steps_left, int n);

/* Wait; returns the first simulation error (its slot in *bad_slot, may be NULL). */
int smaug_batch_sync(smaug_batch *b, int *bad_slot);

/*
 * Polling and read-back that do not wait for later steps, for a serving loop
 * that keeps the next steps queued while it handles the last ones:
 *   smaug_batch_poll_begin   snapshot of the steps left per slot behind the
 *                            steps queued so far (*ticket names it; up to 4
 *                            snapshots wait at a time)
 *   smaug_batch_poll_end     wait for that snapshot only and return it (as
 *                            smaug_batch_poll; -1 for a free slot)
 *   smaug_batch_get_state_async
 *                            queue the read of a simulation that had finished
 *                            in the last snapshot waited for, on a read-back
 *                            stream that follows that snapshot (not the steps
 *                            queued after it); w is best pinned host memory
 *   smaug_batch_io_wait      wait for the queued reads
 */
int smaug_batch_poll_begin(smaug_batch *b, long long *ticket);
int smaug_batch_poll_end(smaug_batch *b, long long ticket, long long *steps_left, int n);
int smaug_batch_get_state_async(smaug_batch *b, int slot, double *w, size_t count);
int smaug_batch_io_wait(smaug_batch *b);

/* One simulation's state (NVAR * N doubles) and scalars (as smaug_get_scalars). */
int smaug_batch_get_state(smaug_batch *b, int slot, double *w, size_t count);
int smaug_batch_get_scalars(smaug_batch *b, int slot, double out[8]);

/*
 * Autotuner: times RK stage 1 of the current simulations with every tile
 * shape the stage kernel is built for (reps launches each) and keeps the
 * fastest.  ms_out (nms entries, may be NULL) receives the per-shape times;
 * -1 for a shape that cannot be resident on the device (not timed, never chosen).
 */
int smaug_batch_tune(smaug_batch *b, int reps, int *variant_out, double *ms_out, int nms);
int smaug_batch_set_variant(smaug_batch *b, int variant);

/* Stage timing, as smaug_profile_stages / smaug_stage_times (while it is on,
 * steps are launched directly instead of from CUDA graphs). */
int smaug_batch_profile_stages(smaug_batch *b, int enable);
int smaug_batch_stage_times(smaug_batch *b, double *ms_total, long long *count);

/* Free arena bytes, the largest free block, simulations held. */
int smaug_batch_info(smaug_batch *b, size_t *free_bytes, size_t *largest_free, int *sims);
void *smaug_batch_stream(smaug_batch *b);
long long smaug_batch_launch_count(smaug_batch *b);
const char *smaug_batch_last_error(smaug_batch *b);

/*
 * VAC configuration files: the reference's format for initial conditions and
 * snapshots (host only).  ascii .ini as readasciivacconfig reads it
 * (src/readwrite.c:982-1112); binary .out as writevacconfig writes it
 * (src/readwrite.c:160-368).  Positions are ndim arrays of N doubles (the
 * reference's wd[pos1..]), states nw arrays of N doubles (wmod slot layout),
 * x fastest, N = n[0] * .. * n[ndim-1].  The readers fill the header; with pos
 * and w both NULL they stop there (so a caller can size its buffers first).
 * Errors return SMAUG_ERR_ARG with smaug_vac_last_error() (per thread).
 */
typedef struct {
  char name[80];     /* first line / 79-byte name */
  int it;            /* iteration number (state.it) */
  double t;          /* simulation time (state.t) */
  int ndim, neqpar, nw;
  int n[3];          /* cells per dim (n[d] = 1 beyond ndim) */
  double eqpar[16];  /* gamma, eta, g_1 .. g_ndim, ... (neqpar of them) */
  char names[80];    /* variable names line */
} smaug_vac_header;

int smaug_vac_read_ascii(const char *path, smaug_vac_header *hdr, double *pos, size_t pos_count, double *w,
                         size_t w_count);
int smaug_vac_write_ascii(const char *path, const smaug_vac_header *hdr, const double *pos, const double *w);
int smaug_vac_read_binary(const char *path, smaug_vac_header *hdr, double *pos, size_t pos_count, double *w,
                          size_t w_count);
int smaug_vac_write_binary(const char *path, const smaug_vac_header *hdr, const double *pos, const double *w);
const char *smaug_vac_last_error(void);

/* The CUDA stream (cudaStream_t) all work of ctx is ordered on. */
void *smaug_stream(smaug_ctx *ctx);

/* Kernel launches issued so far by ctx (for launch accounting). */
long long smaug_launch_count(smaug_ctx *ctx);

const char *smaug_last_error(smaug_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
