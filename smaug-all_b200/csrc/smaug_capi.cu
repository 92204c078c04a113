// smaug_capi.cu -- host side of the C ABI declared in include/smaug_b200.h.
//
// One context = one simulation resident in HBM.  A step is a short fixed
// sequence of launches on the context's stream:
//   dt_kernel                 the reference's moddton dt block
//                             (iosmaug.cpp:855-898), from maxima that the
//                             previous stage already reduced on the device
//   stage_kernel x 4 (or 1)   fused RK stages (fluxes + hyperdiffusion +
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

namespace smaug_exact {
void launch_stage(int D, const smaug::StageArgs &a, const smaug::Geo &g, const smaug::Phys &p, cudaStream_t st);
void launch_reduce(int D, const double *w, const double *bg, const smaug::Geo &g, const smaug::Phys &p,
                   smaug::Reduce *r, cudaStream_t st);
}  // namespace smaug_exact
namespace smaug_fast {
void launch_stage(int D, const smaug::StageArgs &a, const smaug::Geo &g, const smaug::Phys &p, cudaStream_t st);
void launch_reduce(int D, const double *w, const double *bg, const smaug::Geo &g, const smaug::Phys &p,
                   smaug::Reduce *r, cudaStream_t st);
}  // namespace smaug_fast

using namespace smaug;

struct smaug_ctx {
  smaug_params prm;
  int device = 0;
  int D = 0, NW = 0, NB = 0, NVAR = 0;
  Geo geo{};
  Phys phys{};
  cudaStream_t stream = nullptr;
  double *W[4] = {nullptr, nullptr, nullptr, nullptr};  // state, RK stages / ping-pong
  double *bg = nullptr;
  double *dx1 = nullptr;     // concatenated 1-D metric
  double *dxlast = nullptr;  // full metric of the last dim
  DevScalars *sc = nullptr;
  bool have_metric = false, have_state = false;
  int cur = 0;  // which W buffer holds the state (single-step ping-pong)
  long long launches = 0;
  long long steps = 0;
  std::string err;
  // optional per-stage timing (the reference's tcal accumulator, iosmaug.cpp:1515-1517)
  bool profile = false;
  std::vector<cudaEvent_t> ev;  // pairs around stage launches
  size_t ev_used = 0;
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

// ndimp of the reference's reductions (computedervfields.cu:1940-1950).
long long ref_ndimp(long long dimp) {
  double fn, fractn, in;
  fn = log((double)dimp) / log(2.0);
  fractn = modf(fn, &in);
  if (fractn > 0) {
    fn += 1;
    return (long long)(int)pow(2, fn);
  }
  return dimp;
}

// Ghost fill of the evolved fields from their interior sources (periodic /
// contcd4), used once when a state is loaded (iosmaug.cpp:786-794).
__global__ void ghost_fill_kernel(double *w, int nw, Geo g, int D) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < g.N; j += (long long)gridDim.x * blockDim.x) {
    long long r = j;
    int c[3] = {0, 0, 0};
    c[0] = (int)(r % g.n[0]);
    r /= g.n[0];
    c[1] = (int)(r % g.n[1]);
    c[2] = (int)(r / g.n[1]);
    int s[3] = {c[0], c[1], c[2]};
    bool ghost = false;
    for (int d = 0; d < D; ++d) {
      const int n = g.n[d], x = c[d];
      if (x >= 2 && x <= n - 3) continue;
      ghost = true;
      if (g.btype[d] == 0)
        s[d] = x < 2 ? x + (n - 4) : x - (n - 4);
      else
        s[d] = x == 0 ? 4 : x == 1 ? 3 : x == n - 1 ? n - 5 : n - 4;
    }
    if (!ghost) continue;
    const long long src = s[0] + (long long)s[1] * g.st[1] + (long long)s[2] * g.st[2];
    for (int f = 0; f < nw; ++f) w[(long long)f * g.N + j] = w[(long long)f * g.N + src];
  }
}

// The moddton dt block of the reference loop (iosmaug.cpp:855-898):
// dt = courant / maxcourant, then for n > 1 the viscous limit of cugetdtvisc1
// (nushk1.cu:658-790) as that routine actually evaluates it: its buffer holds
// maxviscoef/delx^2 on the first K cells and the courant values c_f/delx of
// the last dimension on the rest.
__global__ void dt_kernel(DevScalars *sc, Phys p, int D) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  sc->step += 1;
  const int n = sc->step;
  if (p.dt_mode == 1) {
    const double maxc = red_get(sc->red[0], 3);
    sc->maxcourant = maxc;
    if (((p.courant) / (maxc)) > 1.0e-8) sc->dt = (p.courant) / (maxc);
    if (n > 1) {
      const double cpred = red_get(sc->red[0], 4);
      double dtd = 0.0000000001;
      for (int dir = 0; dir < D; ++dir) {
        double m = cpred;
        double v = ((sc->maxviscoef) + 0.0) / (p.minsq[dir]);
        if (v > m) m = v;
        if (m > dtd) dtd = m;
        dtd = 0.25 / dtd;
      }
      sc->dtdiffvisc = dtd;
    }
    if ((sc->dtdiffvisc) > 1.0e-8 && (sc->dt) > ((sc->dtdiffvisc))) sc->dt = sc->dtdiffvisc;
  }
  if (!isfinite(sc->dt) || sc->dt <= 0.0) sc->status = SMAUG_ERR_NONFINITE;
  for (int s = 1; s < 5; ++s)
    for (int k = 0; k < 8; ++k) sc->red[s].v[k] = 0ull;
}

// End of step: running maximum of the hyperviscosity (the reference's reset
// is undone by cucomputec's params copy, computedervfields.cu:2298-2328) and
// carry the maxima of the new state to slot 0.
__global__ void finish_kernel(DevScalars *sc, int last) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double nu = 0.0;
  for (int s = 1; s <= last; ++s) nu = fmax(nu, red_get(sc->red[s], 5));
  if (nu > sc->maxviscoef) sc->maxviscoef = nu;
  sc->red[0] = sc->red[last];
  for (int k = 0; k < 6; ++k) {
    double v = red_get(sc->red[0], k);
    if (!isfinite(v)) sc->status = SMAUG_ERR_NONFINITE;
  }
}

void launch_stage(smaug_ctx *c, const StageArgs &a) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c->profile) {
    while (c->ev.size() < c->ev_used + 2) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) break;
      c->ev.push_back(e);
    }
    if (c->ev.size() >= c->ev_used + 2) {
      e0 = c->ev[c->ev_used];
      e1 = c->ev[c->ev_used + 1];
      c->ev_used += 2;
      cudaEventRecord(e0, c->stream);
    }
  }
  if (c->prm.exact)
    smaug_exact::launch_stage(c->D, a, c->geo, c->phys, c->stream);
  else
    smaug_fast::launch_stage(c->D, a, c->geo, c->phys, c->stream);
  if (e1) cudaEventRecord(e1, c->stream);
  c->launches++;
}

}  // namespace

extern "C" {

int smaug_nvar(int ndim) { return 4 + 3 * ndim; }

int smaug_create(const smaug_params *prm, int device, smaug_ctx **out) {
  if (!prm || !out) return SMAUG_ERR_ARG;
  *out = nullptr;
  smaug_ctx *ctx = new smaug_ctx();
  ctx->prm = *prm;
  ctx->device = device;
  const int D = prm->ndim;
  if (D != 2 && D != 3) {
    int r = fail(ctx, SMAUG_ERR_ARG, "ndim must be 2 or 3");
    *out = ctx;
    return r;
  }
  ctx->D = D;
  ctx->NW = 2 + 2 * D;
  ctx->NVAR = 4 + 3 * D;
  ctx->NB = ctx->NVAR - ctx->NW;
  long long N = 1;
  for (int d = 0; d < 3; ++d) {
    int n = d < D ? prm->n[d] : 1;
    if (d < D && (n < 10 || n > (1 << 20))) {
      int r = fail(ctx, SMAUG_ERR_ARG, "each dimension needs 10..2^20 cells including ghosts");
      *out = ctx;
      return r;
    }
    if (d < D && prm->btype[d] != SMAUG_BC_PERIODIC && prm->btype[d] != SMAUG_BC_CONTCD4) {
      int r = fail(ctx, SMAUG_ERR_ARG, "boundary type must be periodic (0) or contcd4 (4)");
      *out = ctx;
      return r;
    }
    ctx->geo.n[d] = n;
    ctx->geo.btype[d] = d < D ? prm->btype[d] : 0;
    N *= n;
  }
  ctx->geo.st[0] = 1;
  ctx->geo.st[1] = ctx->geo.n[0];
  ctx->geo.st[2] = (long long)ctx->geo.n[0] * ctx->geo.n[1];
  ctx->geo.N = N;
  const long long ndimp = ref_ndimp(N);
  ctx->geo.K = ((ndimp + 511) / 512) * 64;
  Phys &p = ctx->phys;
  p.gamma = prm->gamma;
  p.courant = prm->courant;
  for (int f = 0; f < 13; ++f) p.chyp[f] = prm->chyp[f];
  p.has_grav = 0;
  for (int d = 0; d < 3; ++d) {
    p.g[d] = d < D ? prm->g[d] : 0.0;
    if (p.g[d] != 0.0) p.has_grav = 1;
  }
  p.hyperdif = prm->hyperdif;
  p.dt_mode = prm->dt_mode;
  *out = ctx;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  const size_t fsz = sizeof(double) * (size_t)N;
  const int nbuf = 4;
  for (int b = 0; b < nbuf; ++b) CK(cudaMalloc(&ctx->W[b], fsz * ctx->NW));
  CK(cudaMalloc(&ctx->bg, fsz * ctx->NB));
  CK(cudaMalloc(&ctx->dx1, sizeof(double) * (ctx->geo.n[0] + ctx->geo.n[1] + ctx->geo.n[2])));
  CK(cudaMalloc(&ctx->dxlast, fsz));
  CK(cudaMalloc(&ctx->sc, sizeof(DevScalars)));
  CK(cudaMemsetAsync(ctx->sc, 0, sizeof(DevScalars), ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SMAUG_OK;
}

int smaug_destroy(smaug_ctx *ctx) {
  if (!ctx) return SMAUG_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto &b : ctx->W) cudaFree(b);
  cudaFree(ctx->bg);
  cudaFree(ctx->dx1);
  cudaFree(ctx->dxlast);
  cudaFree(ctx->sc);
  for (auto e : ctx->ev) cudaEventDestroy(e);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return SMAUG_OK;
}

int smaug_set_metric(smaug_ctx *ctx, const double *delx, size_t count) {
  if (!ctx || !delx) return SMAUG_ERR_ARG;
  const int D = ctx->D;
  const long long N = ctx->geo.N;
  if (count != (size_t)D * (size_t)N) return fail(ctx, SMAUG_ERR_ARG, "metric must hold ndim * N doubles");
  CK(cudaSetDevice(ctx->device));
  // 1-D metric per dim from an inner line; the stencils use delx at inner
  // cells only, where the reference's metric depends on that coordinate alone.
  std::vector<double> d1(ctx->geo.n[0] + ctx->geo.n[1] + ctx->geo.n[2]);
  size_t off = 0;
  for (int d = 0; d < D; ++d) {
    const double *m = delx + (size_t)d * N;
    const int n = ctx->geo.n[d];
    for (int x = 0; x < n; ++x) {
      int c[3] = {2, 2, D == 3 ? 2 : 0};
      c[d] = x;
      d1[off + x] = m[c[0] + c[1] * ctx->geo.st[1] + c[2] * ctx->geo.st[2]];
    }
    // verify on all inner cells
    for (long long j = 0; j < N; ++j) {
      long long r = j;
      int c[3];
      c[0] = (int)(r % ctx->geo.n[0]);
      r /= ctx->geo.n[0];
      c[1] = (int)(r % ctx->geo.n[1]);
      c[2] = (int)(r / ctx->geo.n[1]);
      bool inner = true;
      for (int e = 0; e < D; ++e)
        if (c[e] < 2 || c[e] > ctx->geo.n[e] - 3) inner = false;
      if (inner && m[j] != d1[off + c[d]])
        return fail(ctx, SMAUG_ERR_ARG, "metric is not a tensor-product grid on the inner cells");
      if (!(m[j] > 0.0)) return fail(ctx, SMAUG_ERR_ARG, "metric entries must be positive");
    }
    off += n;
  }
  CK(cudaMemcpyAsync(ctx->dx1, d1.data(), sizeof(double) * d1.size(), cudaMemcpyHostToDevice, ctx->stream));
  off = 0;
  for (int d = 0; d < D; ++d) {
    ctx->geo.dx1[d] = ctx->dx1 + off;
    off += ctx->geo.n[d];
  }
  CK(cudaMemcpyAsync(ctx->dxlast, delx + (size_t)(D - 1) * N, sizeof(double) * N, cudaMemcpyHostToDevice,
                     ctx->stream));
  ctx->geo.dxlast = ctx->dxlast;
  // min over the first K cells of delx^2 (zeropadmaxdtvisc's cells)
  for (int d = 0; d < D; ++d) {
    double mn = INFINITY;
    const double *m = delx + (size_t)d * N;
    for (long long j = 0; j < ctx->geo.K && j < N; ++j) {
      double v = (m[j]) * (m[j]);
      if (v < mn) mn = v;
    }
    ctx->phys.minsq[d] = mn;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->have_metric = true;
  return SMAUG_OK;
}

static int load_state(smaug_ctx *ctx, const double *w, size_t count, cudaMemcpyKind kind) {
  if (!ctx || !w) return SMAUG_ERR_ARG;
  if (!ctx->have_metric) return fail(ctx, SMAUG_ERR_STATE, "smaug_set_metric must come first");
  const long long N = ctx->geo.N;
  if (count != (size_t)ctx->NVAR * (size_t)N) return fail(ctx, SMAUG_ERR_ARG, "state must hold NVAR * N doubles");
  CK(cudaSetDevice(ctx->device));
  ctx->cur = 0;
  CK(cudaMemcpyAsync(ctx->W[0], w, sizeof(double) * N * ctx->NW, kind, ctx->stream));
  CK(cudaMemcpyAsync(ctx->bg, w + (size_t)N * ctx->NW, sizeof(double) * N * ctx->NB, kind, ctx->stream));
  // host-side scan of the backgrounds: are the energy background terms live?
  if (kind == cudaMemcpyHostToDevice) {
    int has = 0;
    const double *b = w + (size_t)N * ctx->NW;
    for (long long j = 0; j < N && !has; ++j) {
      if (b[j] != 0.0) has = 1;  // eb
      for (int k = 0; k < ctx->D; ++k)
        if (b[(size_t)(2 + k) * N + j] != 0.0) has = 1;
    }
    ctx->phys.has_bgb = has;
  } else {
    ctx->phys.has_bgb = 1;
  }
  ghost_fill_kernel<<<148 * 8, 256, 0, ctx->stream>>>(ctx->W[0], ctx->NW, ctx->geo, ctx->D);
  DevScalars init{};
  init.dt = ctx->prm.dt_mode == 1 ? 1.0e-8 : ctx->prm.dt0;
  if (ctx->prm.dt_mode == 1 && ctx->prm.dt0 > 0) init.dt = ctx->prm.dt0;
  CK(cudaMemcpyAsync(ctx->sc, &init, sizeof(DevScalars), cudaMemcpyHostToDevice, ctx->stream));
  if (ctx->prm.exact)
    smaug_exact::launch_reduce(ctx->D, ctx->W[0], ctx->bg, ctx->geo, ctx->phys, &ctx->sc->red[0], ctx->stream);
  else
    smaug_fast::launch_reduce(ctx->D, ctx->W[0], ctx->bg, ctx->geo, ctx->phys, &ctx->sc->red[0], ctx->stream);
  ctx->launches += 2;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->have_state = true;
  ctx->steps = 0;
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
  if (!ctx->have_state) return fail(ctx, SMAUG_ERR_STATE, "no state loaded");
  const long long N = ctx->geo.N;
  if (count != (size_t)ctx->NVAR * (size_t)N) return fail(ctx, SMAUG_ERR_ARG, "state must hold NVAR * N doubles");
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(w, ctx->W[ctx->cur], sizeof(double) * N * ctx->NW, kind, ctx->stream));
  CK(cudaMemcpyAsync(w + (size_t)N * ctx->NW, ctx->bg, sizeof(double) * N * ctx->NB, kind, ctx->stream));
  if (sync) CK(cudaStreamSynchronize(ctx->stream));
  return SMAUG_OK;
}

int smaug_get_state(smaug_ctx *ctx, double *w, size_t count) {
  return store_state(ctx, w, count, cudaMemcpyDeviceToHost, true);
}
int smaug_get_state_device(smaug_ctx *ctx, double *w, size_t count) {
  return store_state(ctx, w, count, cudaMemcpyDeviceToDevice, false);
}

int smaug_step(smaug_ctx *ctx, int nsteps) {
  if (!ctx || nsteps < 0) return SMAUG_ERR_ARG;
  if (!ctx->have_state) return fail(ctx, SMAUG_ERR_STATE, "no state loaded");
  CK(cudaSetDevice(ctx->device));
  for (int it = 0; it < nsteps; ++it) {
    dt_kernel<<<1, 1, 0, ctx->stream>>>(ctx->sc, ctx->phys, ctx->D);
    ctx->launches++;
    StageArgs a{};
    a.bg = ctx->bg;
    a.sc = ctx->sc;
    if (!ctx->prm.rk4) {
      double *w = ctx->W[ctx->cur], *o = ctx->W[1 - ctx->cur];
      a.in = w; a.base = w; a.out = o; a.acc = nullptr; a.kind = 0;
      a.red_in = 0; a.red_out = 1; a.hdiv = 1.0;
      launch_stage(ctx, a);
      finish_kernel<<<1, 1, 0, ctx->stream>>>(ctx->sc, 1);
      ctx->cur = 1 - ctx->cur;
    } else {
      // SAC fourstep (vac.t:447-462): W1 = W + dt/2 L(W); W2 = W + dt/2 L(W1);
      // W3 = W + dt L(W2) and W1 <- (W1 + 2 W2 + W3 - 4 W)/3; W <- (W + dt/6 L(W3)) + W1
      double *W = ctx->W[0], *W1 = ctx->W[1], *W2 = ctx->W[2], *W3 = ctx->W[3];
      a.base = W;
      a.in = W;  a.out = W1; a.acc = nullptr; a.kind = 0; a.red_in = 0; a.red_out = 1; a.hdiv = 2.0;
      launch_stage(ctx, a);
      a.in = W1; a.out = W2; a.red_in = 1; a.red_out = 2; a.hdiv = 2.0;
      launch_stage(ctx, a);
      a.in = W2; a.out = W3; a.acc = W1; a.kind = 3; a.red_in = 2; a.red_out = 3; a.hdiv = 1.0;
      launch_stage(ctx, a);
      a.in = W3; a.out = W;  a.acc = W1; a.kind = 4; a.red_in = 3; a.red_out = 4; a.hdiv = 6.0;
      launch_stage(ctx, a);
      finish_kernel<<<1, 1, 0, ctx->stream>>>(ctx->sc, 4);
    }
    ctx->launches++;
    CK(cudaGetLastError());
    ctx->steps++;
  }
  return SMAUG_OK;
}

int smaug_sync(smaug_ctx *ctx) {
  if (!ctx) return SMAUG_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  int status = 0;
  CK(cudaMemcpy(&status, &ctx->sc->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (status != 0) return fail(ctx, status, "non-finite dt or wave speed on the device");
  return SMAUG_OK;
}

int smaug_get_scalars(smaug_ctx *ctx, double out[8]) {
  if (!ctx || !out) return SMAUG_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  DevScalars s;
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(&s, ctx->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost));
  out[0] = s.dt;
  out[1] = s.maxcourant;
  out[2] = s.maxviscoef;
  out[3] = s.dtdiffvisc;
  for (int d = 0; d < 3; ++d) out[4 + d] = d < ctx->D ? red_get(s.red[0], d) : 0.0;
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
  CK(cudaStreamSynchronize(ctx->stream));
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

void *smaug_stream(smaug_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
long long smaug_launch_count(smaug_ctx *ctx) { return ctx ? ctx->launches : 0; }
const char *smaug_last_error(smaug_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

}  // extern "C"
