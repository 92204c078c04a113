/*
 * smaug_run.c -- C host driver of the B200 ideal-MHD step.
 *
 * The host side of the reference, dev/smaug/src/iosmaug.cpp, in C over the
 * library's C ABI (include/smaug_b200.h): read a VAC ascii configuration
 * (readasciivacconfig, iosmaug.cpp:341-349), derive the metric from its
 * positions (initgrid, iosmaug.cpp:618-633), load the state (cuinit and the
 * initial cuboundary pass, iosmaug.cpp:520, 783-790), then the step loop
 * (iosmaug.cpp:799-1166): every save step a VAC snapshot of the state before
 * the step (writevacconfig, iosmaug.cpp:812-826), then one step -- the dt
 * block and the four Runge-Kutta stages, each stage one call on the host's
 * own CUDA stream -- and a final snapshot.
 *
 *   smaug_run CONFIG.ini STEPS OUTPREFIX [options]
 *     --single            the reference's single step (rkon = 0); default RK4
 *     --mixed             mixed precision (FP32 stage states and stencils)
 *     --exact             the FMA-free build (bit-reproducible)
 *     --fixed-dt DT       fixed dt; default the reference's dt rule (moddton)
 *     --courant C         Courant number (default 0.3)
 *     --btype B0,B1[,B2]  boundary type per dimension (default 0, periodic)
 *     --no-hyperdif       hyperdiffusion off (p->hyperdifmom = 0)
 *     --save-every K      snapshot every K steps (default: the final state only)
 *     --device D          CUDA device (default 0)
 *
 * Snapshots are VAC binary files OUTPREFIX_<step>.out (the reference's .out
 * layout: positions, then the NVAR fields of wmod) with it = the step count
 * and t = the simulation time.  The chyp constants are the Orszag-Tang model's
 * (models/iosmaugparams.h.ot:171-179): rho 0.045, e 0.02, momenta 0.4, B 0.02.
 * gamma and the gravity components come from the file's equation parameters
 * (gamma, eta, g_1 .. g_ndim), as readasciivacconfig reads them.
 * Exit status 0 on success; any library error is printed with its message.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>

#include "smaug_b200.h"

static void usage(void) {
  fprintf(stderr,
          "usage: smaug_run CONFIG.ini STEPS OUTPREFIX [--single] [--mixed] [--exact] [--fixed-dt DT]\n"
          "                 [--courant C] [--btype B0,B1[,B2]] [--no-hyperdif] [--save-every K] [--device D]\n");
}

#define TRY(call, what)                                                              \
  do {                                                                               \
    int rc_ = (call);                                                                \
    if (rc_ != SMAUG_OK) {                                                           \
      fprintf(stderr, "smaug_run: %s failed (%d): %s\n", what, rc_, err_of(ctx));    \
      goto fail;                                                                     \
    }                                                                                \
  } while (0)

/* the message of the failed call: the context's, else the file and grid
   helpers' (smaug_vac_last_error covers smaug_vac_* and smaug_initgrid) */
static const char *err_of(smaug_ctx *ctx) {
  const char *m = ctx ? smaug_last_error(ctx) : "";
  return (m && *m) ? m : smaug_vac_last_error();
}

static int write_snapshot(const char *prefix, const smaug_vac_header *h0, int it, double t, const double *pos,
                          const double *w) {
  char path[4096];
  smaug_vac_header h = *h0;
  h.it = it;
  h.t = t;
  snprintf(path, sizeof(path), "%s_%d.out", prefix, it);
  return smaug_vac_write_binary(path, &h, pos, w);
}

int main(int argc, char **argv) {
  if (argc >= 2 && !strcmp(argv[1], "--help")) {
    usage();
    return 0;
  }
  if (argc < 4) {
    usage();
    return 2;
  }
  const char *cfg = argv[1], *prefix = argv[3];
  const int nt = atoi(argv[2]);
  int rk4 = 1, mixed = 0, exact = 0, hyperdif = 1, save_every = 0, device = 0;
  int btype[3] = {0, 0, 0};
  double courant = 0.3, fixed_dt = 0.0;
  for (int i = 4; i < argc; ++i) {
    if (!strcmp(argv[i], "--single")) rk4 = 0;
    else if (!strcmp(argv[i], "--mixed")) mixed = 1;
    else if (!strcmp(argv[i], "--exact")) exact = 1;
    else if (!strcmp(argv[i], "--no-hyperdif")) hyperdif = 0;
    else if (!strcmp(argv[i], "--fixed-dt") && i + 1 < argc) fixed_dt = atof(argv[++i]);
    else if (!strcmp(argv[i], "--courant") && i + 1 < argc) courant = atof(argv[++i]);
    else if (!strcmp(argv[i], "--save-every") && i + 1 < argc) save_every = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--device") && i + 1 < argc) device = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--btype") && i + 1 < argc) {
      char *s = argv[++i];
      for (int d = 0; d < 3 && s && *s; ++d) {
        btype[d] = (int)strtol(s, &s, 10);
        if (*s == ',') ++s;
      }
    } else {
      usage();
      return 2;
    }
  }
  if (nt < 0) {
    usage();
    return 2;
  }

  smaug_ctx *ctx = NULL;
  double *pos = NULL, *w = NULL, *delx = NULL;
  cudaStream_t stream = NULL;
  int status = 1;

  /* readasciivacconfig: sizes first, then the positions and the state */
  smaug_vac_header h;
  TRY(smaug_vac_read_ascii(cfg, &h, NULL, 0, NULL, 0), "reading the configuration");
  const int D = h.ndim;
  if (D != 2 && D != 3) {
    fprintf(stderr, "smaug_run: ndim %d (2 or 3 needed)\n", D);
    return 1;
  }
  if (h.nw != smaug_nvar(D)) {
    fprintf(stderr, "smaug_run: the file holds %d fields, NVAR is %d for ndim %d\n", h.nw, smaug_nvar(D), D);
    return 1;
  }
  size_t N = 1;
  for (int d = 0; d < D; ++d) N *= (size_t)h.n[d];
  pos = (double *)malloc(sizeof(double) * D * N);
  w = (double *)malloc(sizeof(double) * h.nw * N);
  delx = (double *)malloc(sizeof(double) * D * N);
  if (!pos || !w || !delx) {
    fprintf(stderr, "smaug_run: out of host memory\n");
    goto fail;
  }
  TRY(smaug_vac_read_ascii(cfg, &h, pos, (size_t)D * N, w, (size_t)h.nw * N), "reading the configuration");

  /* struct params of the run (iosmaug.cpp:225-330) */
  smaug_params prm;
  memset(&prm, 0, sizeof(prm));
  prm.ndim = D;
  for (int d = 0; d < 3; ++d) prm.n[d] = d < D ? h.n[d] : 1;
  prm.gamma = h.neqpar > 0 ? h.eqpar[0] : 5.0 / 3.0;
  for (int d = 0; d < D; ++d) {
    prm.g[d] = h.neqpar > 2 + d ? h.eqpar[2 + d] : 0.0;
    prm.btype[d] = btype[d];
  }
  prm.courant = courant;
  prm.chyp[0] = 0.045;                                  /* rho */
  prm.chyp[1 + D] = 0.02;                               /* e */
  for (int k = 0; k < D; ++k) {
    prm.chyp[1 + k] = 0.4;                              /* momenta */
    prm.chyp[2 + D + k] = 0.02;                         /* B */
  }
  prm.hyperdif = hyperdif;
  prm.rk4 = rk4;
  prm.dt_mode = fixed_dt > 0.0 ? 0 : 1;
  prm.dt0 = fixed_dt;
  prm.exact = exact;
  prm.precision = mixed ? SMAUG_PREC_MIXED : SMAUG_PREC_FP64;
  /* grid spacing and origin from the positions (x_d at cells 0 and 1 along d) */
  for (int d = 0; d < D; ++d) {
    const size_t s = d == 0 ? 1 : d == 1 ? (size_t)h.n[0] : (size_t)h.n[0] * h.n[1];
    prm.xmin[d] = pos[(size_t)d * N];
    prm.dx[d] = pos[(size_t)d * N + s] - pos[(size_t)d * N];
  }

  /* initgrid: the metric from the positions */
  TRY(smaug_initgrid(D, prm.n, pos, prm.dx, delx), "smaug_initgrid");

  TRY(smaug_create(&prm, device, &ctx), "smaug_create");
  TRY(smaug_set_metric(ctx, delx, (size_t)D * N), "smaug_set_metric");
  TRY(smaug_set_state(ctx, w, (size_t)h.nw * N), "smaug_set_state");
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
    fprintf(stderr, "smaug_run: no CUDA stream\n");
    goto fail;
  }

  double t = 0.0, sc[8];
  const int stages = rk4 ? 4 : 1;
  for (int n = 1; n <= nt; ++n) {
    if (save_every > 0 && (n - 1) % save_every == 0) {
      TRY(smaug_get_state(ctx, w, (size_t)h.nw * N), "smaug_get_state");
      TRY(write_snapshot(prefix, &h, n - 1, t, pos, w), "writing a snapshot");
    }
    for (int k = 1; k <= stages; ++k) TRY(smaug_stage(ctx, k, stream), "smaug_stage");
    /* the step's dt (set on the device by the dt rule), for the snapshot
       time; the reference reads p->dt back every step as well */
    TRY(smaug_get_scalars(ctx, sc), "smaug_get_scalars");
    t += sc[0];
  }
  TRY(smaug_sync(ctx), "smaug_sync");
  TRY(smaug_get_state(ctx, w, (size_t)h.nw * N), "smaug_get_state");
  TRY(write_snapshot(prefix, &h, nt, t, pos, w), "writing the final snapshot");
  TRY(smaug_get_scalars(ctx, sc), "smaug_get_scalars");
  printf("smaug_run: %d steps, dt %.17g, maxviscoef %.17g, t %.17g\n", nt, sc[0], sc[2], t);
  status = 0;
fail:
  if (stream) cudaStreamDestroy(stream);
  if (ctx) smaug_destroy(ctx);
  free(pos);
  free(w);
  free(delx);
  return status;
}
