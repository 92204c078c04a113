// smaug_capi.cu -- host side of the C ABI declared in include/smaug_b200.h.
//
// One context = one simulation resident in HBM.  A step is a short fixed
// sequence of launches on the context's stream:
//   dt_kernel                 the reference's moddton dt block
//                             (iosmaug.cpp:855-898), from maxima that the
//                             previous stage already reduced on the device
//   stage kernel x 4 (or 1)   fused RK stages (fluxes + hyperdiffusion +
//                             ghost fill + wave-speed maxima)
//   finish_kernel             running maxviscoef, carry the maxima
// No host round trip happens inside a step (the reference copies struct
// params and often the whole derived-field array between host and device
// dozens of times per step).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/smaug_b200.h"
#include "smaug_device.cuh"
#include "smaug_batch.cuh"
#include "smaug_common.cuh"

using namespace smaug;

namespace {

// Everything one simulation's launches need: the context API and the
// no-allocation entry point both fill one of these.
struct Run : SimPlan {
  cudaStream_t stream = nullptr;
  double *W[4] = {nullptr, nullptr, nullptr, nullptr};  // state, then RK stages (or ping-pong)
  // mixed precision: FP32 base value, its FP32 compensation, two FP32 stage
  // states and the FP32 RK increment sum (W[0] then only stages loads/stores)
  float *F[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double *bg = nullptr;
  DevScalars *sc = nullptr;
  // the production RK4 path runs the batch stage kernel over a table of this
  // one simulation (so a simulation gives the same bits alone and in a batch)
  BatchInst *inst = nullptr;
  BatchInst h_inst{};
  int ntiles = 0;
  int grid = 0;  // persistent grid of the batch stage kernel (blocks), at most ntiles
  int cur = 0;
  long long launches = 0;
  // optional per-stage timing
  std::vector<cudaEvent_t> *ev = nullptr;
  size_t *ev_used = nullptr;
  // production RK4 path: CUDA graphs of kGraphSteps steps and of one step
  // (their kernel arguments hold the buffers and the physics; dropped when
  // those change)
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long long graph_launches = 0;  // kernel launches per step in the graphs
};

constexpr int kGraphSteps = 16;

void drop_graphs(Run &r) {
  for (auto &g : r.graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

__global__ void dt_kernel(DevScalars *sc, Phys p, int D) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    dt_update(sc, p, D);
    sc->go = 1;
  }
}

__global__ void finish_kernel(DevScalars *sc, int last) {
  if (threadIdx.x == 0 && blockIdx.x == 0) finish_update(sc, last);
}

__global__ void reset_scalars_kernel(DevScalars *sc, double dt0) {
  if (threadIdx.x == 0 && blockIdx.x == 0) reset_update(sc, dt0);
}

const char *plan(const smaug_params *prm, Run &r) { return plan_sim(prm, r); }

// Launch one stage kernel, bracketed by timing events when profiling is on.
template <typename F>
void timed_launch(Run &r, F launch) {
  cudaEvent_t e1 = nullptr;
  if (r.ev && r.ev_used) {
    while (r.ev->size() < *r.ev_used + 2) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) break;
      r.ev->push_back(e);
    }
    if (r.ev->size() >= *r.ev_used + 2) {
      cudaEventRecord((*r.ev)[*r.ev_used], r.stream);
      e1 = (*r.ev)[*r.ev_used + 1];
      *r.ev_used += 2;
    }
  }
  launch();
  if (e1) cudaEventRecord(e1, r.stream);
  r.launches++;
}

void launch_stage(Run &r, const StageArgs &a) {
  timed_launch(r, [&] {
    if (r.exact)
      smaug_exact::launch_stage(r.D, false, a, r.geo, r.phys, r.stream);
    else
      smaug_fast::launch_stage(r.D, r.mixed, a, r.geo, r.phys, r.stream);
  });
  if (!r.exact) r.launches++;  // the tiled build's ghost pass
}

// RK stage k (1..4) of the production path: the batch stage kernel, one
// block per tile of this simulation.
void launch_rk_stage(Run &r, int k) {
  timed_launch(r, [&] {
    smaug_batchk::launch_batch_stage(r.D, r.mixed, batch_default_variant(r.D, r.mixed), r.inst, nullptr, r.ntiles, k,
                                     r.grid, r.stream);
  });
  // its ghost pass: the ghost chunks of this simulation
  const int nch = (int)((ghost_cells(r.geo, r.D) + 255) / 256);
  smaug_batchk::launch_batch_ghost(r.D, r.mixed, r.inst, nullptr, nch, k, std::min(nch, 148 * 8), r.stream);
  r.launches++;
}

// Describe the simulation to the batch stage kernel (production RK4 path).
// Called whenever the metric, the backgrounds or the buffers change.
cudaError_t run_upload_inst(Run &r) {
  if (!r.rk4 || r.exact || !r.inst) return cudaSuccess;
  BatchInst &I = r.h_inst;
  I = BatchInst{};
  I.geo = r.geo;
  I.phys = r.phys;
  I.bg = r.bg;
  for (int k = 0; k < 4; ++k) I.W[k] = r.W[k];
  for (int k = 0; k < 5; ++k) I.F[k] = r.F[k];
  I.sc = r.sc;
  I.active = 1;
  int t[3];
  batch_tile_shape(r.D, batch_default_variant(r.D, r.mixed), t);
  r.ntiles = 1;
  for (int d = 0; d < 3; ++d) {
    I.tiles[d] = d < r.D ? (r.geo.n[d] - 4 + t[d] - 1) / t[d] : 1;
    r.ntiles *= I.tiles[d];
  }
  // a persistent grid, as a batch runs it: resident blocks on every SM, each
  // looping over tiles and keeping its maxima across them
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int occ = std::max(1, smaug_batchk::batch_stage_occupancy(r.D, r.mixed, batch_default_variant(r.D, r.mixed)));
  r.grid = std::min(r.ntiles, occ * sms);
  return cudaMemcpyAsync(r.inst, &I, sizeof(BatchInst), cudaMemcpyHostToDevice, r.stream);
}

// A state is in r.W[0] (evolved) and r.bg: fill ghosts, reset scalars,
// reduce the initial maxima (and, mixed, split it into value +
// compensation).  With fixed boundaries the maxima of the cells that keep
// their loaded values become the floor of every step's maxima, and every
// stage buffer gets those cells.  Asynchronous.
cudaError_t run_load(Run &r) {
  r.cur = 0;
  ghost_fill(r.W[0], r.NW, r.geo, r.D, r.stream);
  const double dt0 = r.phys.dt_mode == 1 ? (r.dt0 > 0 ? r.dt0 : 1.0e-8) : r.dt0;
  reset_scalars_kernel<<<1, 1, 0, r.stream>>>(r.sc, dt0);
  auto reduce = r.exact ? smaug_exact::launch_reduce : smaug_fast::launch_reduce;
  reduce(r.D, r.W[0], r.bg, r.geo, r.phys, &r.sc->red[0], r.stream, 0);
  r.launches += r.D + 2;
  if (r.geo.has_const) {
    reduce(r.D, r.W[0], r.bg, r.geo, r.phys, &r.sc->floor, r.stream, 1);
    r.launches++;
  }
  if (r.mixed) {
    split_kernel<<<148 * 8, 256, 0, r.stream>>>(r.W[0], r.F[0], r.F[1], (long long)r.NW * r.geo.N);
    r.launches++;
  }
  if (r.geo.has_const) {
    const size_t n = (size_t)r.NW * r.geo.N;
    for (int k = 1; k < 4; ++k)
      if (!r.mixed && r.W[k]) {
        const cudaError_t e = cudaMemcpyAsync(r.W[k], r.W[0], sizeof(double) * n, cudaMemcpyDeviceToDevice, r.stream);
        if (e != cudaSuccess) return e;
      }
    if (r.mixed)
      for (int k = 2; k < 4; ++k) {
        const cudaError_t e = cudaMemcpyAsync(r.F[k], r.F[0], sizeof(float) * n, cudaMemcpyDeviceToDevice, r.stream);
        if (e != cudaSuccess) return e;
      }
  }
  return cudaGetLastError();
}

// Mixed precision: bring the FP64 copy W[0] up to date with w32 + c32.
cudaError_t run_combine(Run &r) {
  if (!r.mixed) return cudaSuccess;
  combine_kernel<<<148 * 8, 256, 0, r.stream>>>(r.F[0], r.F[1], r.W[0], (long long)r.NW * r.geo.N);
  r.launches++;
  return cudaGetLastError();
}

// Stages per step: four for RK4, one for the single step.
inline int stages_per_step(const Run &r) { return r.rk4 ? 4 : 1; }

// Enqueue stage k (1..stages_per_step) of a step: stage 1 opens the step with
// the dt kernel, the last stage closes it with the finish kernel.
cudaError_t run_stage(Run &r, int k) {
  if (k == 1) {
    dt_kernel<<<1, 1, 0, r.stream>>>(r.sc, r.phys, r.D);
    r.launches++;
  }
  StageArgs a{};
  a.bg = r.bg;
  a.sc = r.sc;
  if (r.mixed || (r.rk4 && !r.exact)) {
    // production fourstep, FP64 or mixed (FP32 stage states: S1 = W + dt/2
    // L(W), S2 = W + dt/2 L(S1), S3 = W + dt L(S2), A = (S1 + 2 S2 + S3 -
    // 4 W)/3 accumulated stage by stage, W <- W + dt/6 L(S3) + A); the stage
    // roles are in batch_args (batch_kernels.inc)
    launch_rk_stage(r, k);
  } else if (!r.rk4) {
    double *w = r.W[r.cur], *o = r.W[1 - r.cur];
    a.in = w; a.base = w; a.out = o; a.acc = nullptr; a.kind = 0;
    a.red_in = 0; a.red_out = 1; a.hdiv = 1.0; a.tfrac = 0.0;
    launch_stage(r, a);
    r.cur = 1 - r.cur;
  } else {
    // SAC fourstep (vac.t:447-462): W1 = W + dt/2 L(W); W2 = W + dt/2 L(W1);
    // W3 = W + dt L(W2) and W1 <- (W1 + 2 W2 + W3 - 4 W)/3; W <- (W + dt/6 L(W3)) + W1
    double *W = r.W[0], *W1 = r.W[1], *W2 = r.W[2], *W3 = r.W[3];
    a.base = W;
    switch (k) {
      case 1: a.in = W;  a.out = W1; a.acc = nullptr; a.kind = 0; a.red_in = 0; a.red_out = 1; a.hdiv = 2.0; a.tfrac = 0.0; break;
      case 2: a.in = W1; a.out = W2; a.acc = nullptr; a.kind = 0; a.red_in = 1; a.red_out = 2; a.hdiv = 2.0; a.tfrac = 0.5; break;
      case 3: a.in = W2; a.out = W3; a.acc = W1; a.kind = 3; a.red_in = 2; a.red_out = 3; a.hdiv = 1.0; a.tfrac = 0.5; break;
      default: a.in = W3; a.out = W; a.acc = W1; a.kind = 4; a.red_in = 3; a.red_out = 4; a.hdiv = 6.0; a.tfrac = 1.0; break;
    }
    launch_stage(r, a);
  }
  if (k == stages_per_step(r)) {
    finish_kernel<<<1, 1, 0, r.stream>>>(r.sc, k);
    r.launches++;
  }
  return cudaGetLastError();
}

// Enqueue nsteps full steps.
cudaError_t run_steps(Run &r, int nsteps) {
  const int ns = stages_per_step(r);
  for (int it = 0; it < nsteps; ++it)
    for (int k = 1; k <= ns; ++k) {
      const cudaError_t e = run_stage(r, k);
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}

}  // namespace

struct smaug_ctx {
  smaug_params prm;
  int device = 0;
  Run run;
  double *dx1 = nullptr;     // concatenated 1-D metric
  double *drv = nullptr;     // driver factor lines
  double *dxlast = nullptr;  // full metric of the last dim
  bool have_metric = false, have_state = false;
  long long steps = 0;
  std::string err;
  bool profile = false;
  std::vector<cudaEvent_t> ev;
  size_t ev_used = 0;
  int next_stage = 1;          // smaug_stage: the stage the current step takes next
  cudaEvent_t join = nullptr;  // orders the context stream and a caller's stream
};

namespace {

int fail(smaug_ctx *c, int code, const std::string &m) {
  if (c) c->err = m;
  return code;
}

#define CK(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) return fail(ctx, SMAUG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

}  // namespace

extern "C" {

int smaug_nvar(int ndim) { return 4 + 3 * ndim; }

int smaug_create(const smaug_params *prm, int device, smaug_ctx **out) {
  if (!prm || !out) return SMAUG_ERR_ARG;
  *out = nullptr;
  smaug_ctx *ctx = new smaug_ctx();
  ctx->prm = *prm;
  ctx->device = device;
  *out = ctx;
  Run &r = ctx->run;
  if (const char *m = plan(prm, r)) return fail(ctx, SMAUG_ERR_ARG, m);
  r.ev = &ctx->ev;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking));
  const size_t fsz = sizeof(double) * (size_t)r.geo.N;
  for (int b = 0; b < (r.mixed ? 1 : 4); ++b) CK(cudaMalloc(&r.W[b], fsz * r.NW));
  if (r.mixed)
    for (auto &f : r.F) CK(cudaMalloc(&f, sizeof(float) * (size_t)r.geo.N * r.NW));
  CK(cudaMalloc(&r.bg, fsz * r.NB));
  CK(cudaMalloc(&ctx->dx1, 2 * sizeof(double) * (r.geo.n[0] + r.geo.n[1] + r.geo.n[2])));  // lines, reciprocals
  CK(cudaMalloc(&ctx->dxlast, fsz));
  CK(cudaMalloc(&r.sc, sizeof(DevScalars)));
  CK(cudaMalloc(&r.inst, sizeof(BatchInst)));
  {
    const size_t nl = (size_t)r.geo.n[0] + r.geo.n[1] + r.geo.n[2];
    std::vector<double> lines(nl);
    driver_lines(r, prm, lines.data());
    CK(cudaMalloc(&ctx->drv, sizeof(double) * nl));
    CK(cudaMemcpyAsync(ctx->drv, lines.data(), sizeof(double) * nl, cudaMemcpyHostToDevice, r.stream));
    CK(cudaStreamSynchronize(r.stream));
    size_t off = 0;
    for (int d = 0; d < 3; ++d) {
      r.geo.drvf[d] = ctx->drv + off;
      off += r.geo.n[d];
    }
  }
  CK(cudaMemsetAsync(r.sc, 0, sizeof(DevScalars), r.stream));
  CK(cudaEventCreateWithFlags(&ctx->join, cudaEventDisableTiming));
  CK(cudaStreamSynchronize(r.stream));
  return SMAUG_OK;
}

int smaug_destroy(smaug_ctx *ctx) {
  if (!ctx) return SMAUG_OK;
  Run &r = ctx->run;
  cudaSetDevice(ctx->device);
  if (r.stream) cudaStreamSynchronize(r.stream);
  for (auto &b : r.W) cudaFree(b);
  for (auto &f : r.F) cudaFree(f);
  cudaFree(r.bg);
  cudaFree(ctx->dx1);
  cudaFree(ctx->drv);
  cudaFree(ctx->dxlast);
  cudaFree(r.sc);
  cudaFree(r.inst);
  drop_graphs(r);
  for (auto e : ctx->ev) cudaEventDestroy(e);
  if (ctx->join) cudaEventDestroy(ctx->join);
  if (r.stream) cudaStreamDestroy(r.stream);
  delete ctx;
  return SMAUG_OK;
}

int smaug_set_metric(smaug_ctx *ctx, const double *delx, size_t count) {
  if (!ctx || !delx) return SMAUG_ERR_ARG;
  Run &r = ctx->run;
  if (!r.sc) return fail(ctx, SMAUG_ERR_STATE, "context not created");
  const int D = r.D;
  const long long N = r.geo.N;
  if (count != (size_t)D * (size_t)N) return fail(ctx, SMAUG_ERR_ARG, "metric must hold ndim * N doubles");
  CK(cudaSetDevice(ctx->device));
  // The stencils use delx at inner cells only, where the reference's metric
  // depends on that coordinate alone: keep one line per dim.
  const size_t nl = (size_t)r.geo.n[0] + r.geo.n[1] + r.geo.n[2];
  std::vector<double> d1(2 * nl);  // the lines, then their reciprocals
  double minsq[3];
  if (const char *m = metric_host(r, delx, d1.data(), minsq)) return fail(ctx, SMAUG_ERR_ARG, m);
  for (size_t i = 0; i < nl; ++i) d1[nl + i] = 1.0 / d1[i];
  CK(cudaMemcpyAsync(ctx->dx1, d1.data(), sizeof(double) * d1.size(), cudaMemcpyHostToDevice, r.stream));
  size_t off = 0;
  for (int d = 0; d < D; ++d) {
    r.geo.dx1[d] = ctx->dx1 + off;
    r.geo.rdx1[d] = ctx->dx1 + nl + off;
    off += r.geo.n[d];
  }
  CK(cudaMemcpyAsync(ctx->dxlast, delx + (size_t)(D - 1) * N, sizeof(double) * N, cudaMemcpyHostToDevice,
                     r.stream));
  r.geo.dxlast = ctx->dxlast;
  CK(cudaMemcpyAsync(r.sc->minsq, minsq, sizeof(minsq), cudaMemcpyHostToDevice, r.stream));
  CK(run_upload_inst(r));
  CK(cudaStreamSynchronize(r.stream));
  ctx->have_metric = true;
  return SMAUG_OK;
}

static int load_state(smaug_ctx *ctx, const double *w, size_t count, cudaMemcpyKind kind) {
  if (!ctx || !w) return SMAUG_ERR_ARG;
  Run &r = ctx->run;
  if (!ctx->have_metric) return fail(ctx, SMAUG_ERR_STATE, "smaug_set_metric must come first");
  const long long N = r.geo.N;
  if (count != (size_t)r.NVAR * (size_t)N) return fail(ctx, SMAUG_ERR_ARG, "state must hold NVAR * N doubles");
  CK(cudaSetDevice(ctx->device));
  const Phys before = r.phys;
  CK(cudaMemcpyAsync(r.W[0], w, sizeof(double) * N * r.NW, kind, r.stream));
  CK(cudaMemcpyAsync(r.bg, w + (size_t)N * r.NW, sizeof(double) * N * r.NB, kind, r.stream));
  // Are the energy background terms live?  Found on the device after the
  // copy; the load's initial maxima read the backgrounds either way (zeros
  // give the same values).
  r.phys.has_bgb = 1;
  CK(run_load(r));
  CK(cudaMemsetAsync(&r.sc->bg_live, 0, sizeof(int), r.stream));
  bg_scan_kernel<<<148 * 4, 256, 0, r.stream>>>(r.bg, N, r.D, r.sc);
  r.launches++;
  int live = 1;
  CK(cudaMemcpyAsync(&live, &r.sc->bg_live, sizeof(int), cudaMemcpyDeviceToHost, r.stream));
  CK(cudaStreamSynchronize(r.stream));
  r.phys.has_bgb = live;
  CK(run_upload_inst(r));
  CK(cudaStreamSynchronize(r.stream));
  ctx->have_state = true;
  // the graphs hold the physics by value (dt kernel): recapture if it changed
  if (memcmp(&before, &r.phys, sizeof(Phys)) != 0) drop_graphs(r);
  ctx->steps = 0;
  ctx->next_stage = 1;
  return SMAUG_OK;
}

int smaug_set_state(smaug_ctx *ctx, const double *w, size_t count) {
  return load_state(ctx, w, count, cudaMemcpyHostToDevice);
}
int smaug_set_state_device(smaug_ctx *ctx, const double *w, size_t count) {
  return load_state(ctx, w, count, cudaMemcpyDeviceToDevice);
}

static int store_state(smaug_ctx *ctx, double *w, size_t count, cudaMemcpyKind kind, bool sync) {
  if (!ctx || !w) return SMAUG_ERR_ARG;
  Run &r = ctx->run;
  if (!ctx->have_state) return fail(ctx, SMAUG_ERR_STATE, "no state loaded");
  const long long N = r.geo.N;
  if (count != (size_t)r.NVAR * (size_t)N) return fail(ctx, SMAUG_ERR_ARG, "state must hold NVAR * N doubles");
  CK(cudaSetDevice(ctx->device));
  CK(run_combine(r));
  CK(cudaMemcpyAsync(w, r.W[r.cur], sizeof(double) * N * r.NW, kind, r.stream));
  CK(cudaMemcpyAsync(w + (size_t)N * r.NW, r.bg, sizeof(double) * N * r.NB, kind, r.stream));
  if (sync) CK(cudaStreamSynchronize(r.stream));
  return SMAUG_OK;
}

int smaug_get_state(smaug_ctx *ctx, double *w, size_t count) {
  return store_state(ctx, w, count, cudaMemcpyDeviceToHost, true);
}
int smaug_get_state_device(smaug_ctx *ctx, double *w, size_t count) {
  return store_state(ctx, w, count, cudaMemcpyDeviceToDevice, false);
}

// The steps of the production RK4 path as graph replays: the launch sequence
// of a step is the same every step (the batch stage kernel over this
// simulation's one-entry table, its ghost pass, the dt and finish kernels).
cudaError_t ensure_graphs(Run &r) {
  const int len[2] = {kGraphSteps, 1};
  for (int k = 0; k < 2; ++k) {
    if (r.graph[k]) continue;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(r.stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    const long long l0 = r.launches;
    e = run_steps(r, len[k]);
    const cudaError_t e2 = cudaStreamEndCapture(r.stream, &g);
    r.graph_launches = (r.launches - l0) / len[k];
    r.launches = l0;
    if (e != cudaSuccess) return e;
    if (e2 != cudaSuccess) return e2;
    e = cudaGraphInstantiate(&r.graph[k], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t run_steps_graphed(Run &r, int nsteps) {
  const cudaError_t eg = ensure_graphs(r);
  if (eg != cudaSuccess) return eg;
  for (; nsteps >= kGraphSteps; nsteps -= kGraphSteps) {
    const cudaError_t e = cudaGraphLaunch(r.graph[0], r.stream);
    if (e != cudaSuccess) return e;
    r.launches += r.graph_launches * kGraphSteps;
  }
  for (; nsteps > 0; --nsteps) {
    const cudaError_t e = cudaGraphLaunch(r.graph[1], r.stream);
    if (e != cudaSuccess) return e;
    r.launches += r.graph_launches;
  }
  return cudaSuccess;
}

static int step_impl(smaug_ctx *ctx, int nsteps) {
  Run &r = ctx->run;
  r.ev_used = ctx->profile ? &ctx->ev_used : nullptr;
  if (r.rk4 && !r.exact && !ctx->profile)
    CK(run_steps_graphed(r, nsteps));
  else
    CK(run_steps(r, nsteps));
  ctx->steps += nsteps;
  return SMAUG_OK;
}

int smaug_step(smaug_ctx *ctx, int nsteps) {
  if (!ctx || nsteps < 0) return SMAUG_ERR_ARG;
  if (!ctx->have_state) return fail(ctx, SMAUG_ERR_STATE, "no state loaded");
  if (ctx->next_stage != 1) return fail(ctx, SMAUG_ERR_STATE, "a step begun by smaug_stage is not finished");
  CK(cudaSetDevice(ctx->device));
  return step_impl(ctx, nsteps);
}

// Run `body` with the context's launches on the caller's stream s: s first
// waits for everything queued on the context stream, and the context stream
// then waits for s, so work queued on either later stays in order.
extern "C++" {
template <typename F>
int on_stream(smaug_ctx *ctx, cudaStream_t s, F body) {
  Run &r = ctx->run;
  const cudaStream_t own = r.stream;
  if (!s || s == own) return body();
  CK(cudaEventRecord(ctx->join, own));
  CK(cudaStreamWaitEvent(s, ctx->join, 0));
  r.stream = s;
  const int rc = body();
  r.stream = own;
  CK(cudaEventRecord(ctx->join, s));
  CK(cudaStreamWaitEvent(own, ctx->join, 0));
  return rc;
}
}  // extern "C++"

int smaug_step_on(smaug_ctx *ctx, int nsteps, void *stream) {
  if (!ctx || nsteps < 0) return SMAUG_ERR_ARG;
  if (!ctx->have_state) return fail(ctx, SMAUG_ERR_STATE, "no state loaded");
  if (ctx->next_stage != 1) return fail(ctx, SMAUG_ERR_STATE, "a step begun by smaug_stage is not finished");
  CK(cudaSetDevice(ctx->device));
  // the graphs are captured on the context's own stream, never the caller's
  if (ctx->run.rk4 && !ctx->run.exact && !ctx->profile) CK(ensure_graphs(ctx->run));
  return on_stream(ctx, (cudaStream_t)stream, [&] { return step_impl(ctx, nsteps); });
}

int smaug_stage(smaug_ctx *ctx, int stage, void *stream) {
  if (!ctx) return SMAUG_ERR_ARG;
  if (!ctx->have_state) return fail(ctx, SMAUG_ERR_STATE, "no state loaded");
  Run &r = ctx->run;
  const int ns = stages_per_step(r);
  if (stage < 1 || stage > ns) return fail(ctx, SMAUG_ERR_ARG, "stage must be 1..4 (RK4) or 1 (single step)");
  if (stage != ctx->next_stage) return fail(ctx, SMAUG_ERR_STATE, "stages of a step must come in order 1, 2, ...");
  CK(cudaSetDevice(ctx->device));
  r.ev_used = ctx->profile ? &ctx->ev_used : nullptr;
  const int rc = on_stream(ctx, (cudaStream_t)stream, [&]() -> int {
    CK(run_stage(r, stage));
    return SMAUG_OK;
  });
  if (rc != SMAUG_OK) return rc;
  ctx->next_stage = stage == ns ? 1 : stage + 1;
  if (stage == ns) ctx->steps += 1;
  return SMAUG_OK;
}

int smaug_sync(smaug_ctx *ctx) {
  if (!ctx) return SMAUG_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->run.stream));
  int status = 0;
  CK(cudaMemcpy(&status, &ctx->run.sc->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (status != 0) return fail(ctx, status, "non-finite dt or wave speed on the device");
  return SMAUG_OK;
}

int smaug_get_scalars(smaug_ctx *ctx, double out[8]) {
  if (!ctx || !out) return SMAUG_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  DevScalars s;
  CK(cudaStreamSynchronize(ctx->run.stream));
  CK(cudaMemcpy(&s, ctx->run.sc, sizeof(DevScalars), cudaMemcpyDeviceToHost));
  out[0] = s.dt;
  out[1] = s.maxcourant;
  out[2] = s.maxviscoef;
  out[3] = s.dtdiffvisc;
  for (int d = 0; d < 3; ++d) out[4 + d] = d < ctx->run.D ? red_get(s.red[0], d) : 0.0;
  out[7] = (double)ctx->steps;
  return SMAUG_OK;
}

int smaug_profile_stages(smaug_ctx *ctx, int enable) {
  if (!ctx) return SMAUG_ERR_ARG;
  ctx->profile = enable != 0;
  ctx->ev_used = 0;
  return SMAUG_OK;
}

int smaug_stage_times(smaug_ctx *ctx, double *ms_total, long long *count) {
  if (!ctx || !ms_total || !count) return SMAUG_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->run.stream));
  double t = 0.0;
  for (size_t i = 0; i + 1 < ctx->ev_used; i += 2) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev[i], ctx->ev[i + 1]));
    t += ms;
  }
  *ms_total = t;
  *count = (long long)(ctx->ev_used / 2);
  ctx->ev_used = 0;
  return SMAUG_OK;
}

// ---------------------------------------------------------------------------
// smaug_step_noalloc: the RK step for callers that cannot allocate device
// memory.  Its scratch (the three Runge-Kutta stage buffers, the device-side
// scalars and the 1-D metric lines) lives in this file-scope device array,
// which every GPU that loads the library holds until the process exits.
// Host code must not use g_noalloc_scratch as an address: it is a host-side
// stand-in for the symbol; the device address comes from
// cudaGetSymbolAddress, once per device, in noalloc_scratch().
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[SMAUG_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices] = {nullptr};

void set_err(char *err, size_t errlen, const char *msg) {
  if (err && errlen) {
    std::strncpy(err, msg, errlen - 1);
    err[errlen - 1] = '\0';
  }
}

// Device address of the scratch array on the current device (looked up on
// the first call per device).
cudaError_t noalloc_scratch(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}
}  // namespace

int smaug_step_noalloc(const smaug_params *prm, const double *delx_dev, const double *w_in_dev, double *w_out_dev,
                       int nsteps, void *stream, double *scalars_out, char *err, size_t errlen) {
  if (!prm || !delx_dev || !w_in_dev || !w_out_dev || nsteps < 0) {
    set_err(err, errlen, "null argument or negative step count");
    return SMAUG_ERR_ARG;
  }
  Run r;
  if (const char *m = plan(prm, r)) {
    set_err(err, errlen, m);
    return SMAUG_ERR_ARG;
  }
  if (r.mixed) {
    set_err(err, errlen, "smaug_step_noalloc runs the FP64 path only (precision = 0)");
    return SMAUG_ERR_ARG;
  }
  const long long N = r.geo.N;
  const size_t head = (sizeof(DevScalars) + 255) / 256 * 256 + (sizeof(BatchInst) + 255) / 256 * 256;
  const size_t lines = ((size_t)(r.geo.n[0] + r.geo.n[1] + r.geo.n[2]) * sizeof(double) + 255) / 256 * 256;
  const size_t field = ((size_t)r.NW * (size_t)N * sizeof(double) + 255) / 256 * 256;
  const size_t need = head + 3 * lines + 3 * field;  // metric lines and reciprocals, driver lines, RK buffers
  if (need > (size_t)SMAUG_NOALLOC_SCRATCH_BYTES) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "grid needs %zu bytes of scratch, above the %u-byte maximum of smaug_step_noalloc",
                  need, (unsigned)SMAUG_NOALLOC_SCRATCH_BYTES);
    set_err(err, errlen, msg);
    return SMAUG_ERR_ARG;
  }
  void *base = nullptr;
  cudaError_t e = noalloc_scratch(&base);
  if (e != cudaSuccess) {
    set_err(err, errlen, cudaGetErrorString(e));
    return SMAUG_ERR_CUDA;
  }
  unsigned char *s = (unsigned char *)base;
  r.stream = (cudaStream_t)stream;
  r.sc = (DevScalars *)s;
  r.inst = (BatchInst *)(s + (sizeof(DevScalars) + 255) / 256 * 256);
  double *dx1 = (double *)(s + head);
  r.W[0] = w_out_dev;
  r.bg = w_out_dev + (size_t)r.NW * N;
  double *drv = (double *)(s + head + 2 * lines);
  for (int k = 0; k < 3; ++k) r.W[1 + k] = (double *)(s + head + 3 * lines + k * field);
  const size_t nl = (size_t)r.geo.n[0] + r.geo.n[1] + r.geo.n[2];  // metric_kernel writes the reciprocals after the lines
  size_t off = 0;
  for (int d = 0; d < r.D; ++d) {
    r.geo.dx1[d] = dx1 + off;
    r.geo.rdx1[d] = dx1 + nl + off;
    off += r.geo.n[d];
  }
  r.geo.dxlast = delx_dev + (size_t)(r.D - 1) * N;
  off = 0;
  for (int d = 0; d < 3; ++d) {
    r.geo.drvf[d] = drv + off;
    off += r.geo.n[d];
  }
  r.phys.has_bgb = 1;
  std::vector<double> drv_host((size_t)r.geo.n[0] + r.geo.n[1] + r.geo.n[2]);
  driver_lines(r, prm, drv_host.data());
#define NA(call)                                \
  do {                                          \
    cudaError_t e_ = (call);                    \
    if (e_ != cudaSuccess) {                    \
      set_err(err, errlen, cudaGetErrorString(e_)); \
      return SMAUG_ERR_CUDA;                    \
    }                                           \
  } while (0)
  // every call starts from cleared scalars: the array keeps the last call's data
  NA(cudaMemsetAsync(r.sc, 0, sizeof(DevScalars), r.stream));
  // The metric is checked before anything of the caller's is written, so a
  // bad metric leaves w_out (which may be w_in) as it was.  The check's
  // status is read back here; the load below clears it again (minsq stays).
  minsq_init_kernel<<<1, 1, 0, r.stream>>>(r.sc);
  metric_kernel<<<148 * 4, 256, 0, r.stream>>>(delx_dev, r.geo, r.D, dx1, r.sc);
  NA(cudaGetLastError());
  int metric_status = 0;
  NA(cudaMemcpyAsync(&metric_status, &r.sc->status, sizeof(int), cudaMemcpyDeviceToHost, r.stream));
  NA(cudaStreamSynchronize(r.stream));
  if (metric_status != 0) {
    set_err(err, errlen, "metric is not positive or not a tensor-product grid on the inner cells");
    return SMAUG_ERR_ARG;
  }
  if (w_out_dev != w_in_dev)
    NA(cudaMemcpyAsync(w_out_dev, w_in_dev, sizeof(double) * (size_t)r.NVAR * N, cudaMemcpyDeviceToDevice, r.stream));
  NA(cudaMemcpyAsync(drv, drv_host.data(), sizeof(double) * drv_host.size(), cudaMemcpyHostToDevice, r.stream));
  NA(run_load(r));  // ghost fill of w_out, scalars reset (minsq kept), initial maxima
  NA(run_upload_inst(r));
  NA(run_steps(r, nsteps));
  if (r.cur != 0)  // single-step mode with an odd step count: result in W[1]
    NA(cudaMemcpyAsync(w_out_dev, r.W[1], sizeof(double) * (size_t)r.NW * N, cudaMemcpyDeviceToDevice, r.stream));
  DevScalars hs;
  NA(cudaMemcpyAsync(&hs, r.sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, r.stream));
  NA(cudaStreamSynchronize(r.stream));
#undef NA
  if (scalars_out) {
    scalars_out[0] = hs.dt;
    scalars_out[1] = hs.maxcourant;
    scalars_out[2] = hs.maxviscoef;
    scalars_out[3] = hs.dtdiffvisc;
    for (int d = 0; d < 3; ++d) scalars_out[4 + d] = d < r.D ? red_get(hs.red[0], d) : 0.0;
    scalars_out[7] = (double)nsteps;
  }
  if (hs.status != 0) {
    set_err(err, errlen, "non-finite dt or wave speed on the device");
    return hs.status;
  }
  set_err(err, errlen, "");
  return SMAUG_OK;
}

void *smaug_stream(smaug_ctx *ctx) { return ctx ? (void *)ctx->run.stream : nullptr; }
long long smaug_launch_count(smaug_ctx *ctx) { return ctx ? ctx->run.launches : 0; }
const char *smaug_last_error(smaug_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

}  // extern "C"
