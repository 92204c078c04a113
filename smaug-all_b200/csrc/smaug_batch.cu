// smaug_batch.cu -- host side of the batch C ABI (smaug_batch_* in
// include/smaug_b200.h).
//
// A batch holds many independent simulations of one ndim and one precision,
// of any sizes, in one device arena.  A batch step is six launches for all
// of them together:
//   batch_dt_kernel        per simulation: the reference's dt rule, and
//                          whether it takes this step (steps left, status)
//   batch stage kernel x4  one persistent launch per RK stage over the work
//                          list of (simulation, tile) items
//   batch_finish_kernel    per simulation: running maxima, status
// and a chunk of steps is replayed from a CUDA graph.  Simulations are added
// and removed between steps (admission by arena footprint); finished ones
// stop taking steps on the device without a host round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/smaug_b200.h"
#include "smaug_batch.cuh"
#include "smaug_common.cuh"

namespace {

constexpr int kGraphSteps = 16;  // steps per replay of the long graph
// launches per step: dt, four stages each followed by its ghost pass, finish
constexpr int kLaunchesPerStep = 10;

__global__ void batch_dt_kernel(BatchInst *tab, long long *left, int *status, int n, int D) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  BatchInst &I = tab[i];
  if (!I.active) return;
  DevScalars *sc = I.sc;
  if (left[i] > 0 && sc->status == 0) {
    dt_update(sc, I.phys, D);
    sc->go = 1;
    left[i] -= 1;
  } else {
    sc->go = 0;
  }
  status[i] = sc->status;
}

__global__ void batch_finish_kernel(BatchInst *tab, int *status, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  BatchInst &I = tab[i];
  if (!I.active || !I.sc->go) return;
  finish_update(I.sc, 4);
  status[i] = I.sc->status;
}

// Every simulation in the batch takes stage 1 (autotuning only: stage 1
// writes scratch buffers that the next real step rewrites).
__global__ void batch_go_kernel(BatchInst *tab, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && tab[i].active) tab[i].sc->go = 1;
}

__global__ void one_reset_kernel(DevScalars *sc, double dt0) {
  if (threadIdx.x == 0 && blockIdx.x == 0) reset_update(sc, dt0);
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Arena bytes one simulation takes (the order below is the carve order).
size_t sim_footprint(const SimPlan &p) {
  const size_t N = (size_t)p.geo.N;
  size_t b = align256(sizeof(DevScalars));
  const size_t nl = (size_t)(p.geo.n[0] + p.geo.n[1] + p.geo.n[2]);
  b += align256(2 * sizeof(double) * nl);  // metric lines and their reciprocals
  b += align256(sizeof(double) * nl);      // driver lines
  b += align256(sizeof(double) * N);                  // dxlast
  b += align256(sizeof(double) * (size_t)p.NB * N);   // backgrounds
  b += align256(sizeof(double) * (size_t)p.NW * N);   // W[0]
  if (p.mixed)
    b += 5 * align256(sizeof(float) * (size_t)p.NW * N);
  else
    b += 3 * align256(sizeof(double) * (size_t)p.NW * N);
  return b;
}

struct Slot {
  bool used = false;
  bool pending = false;  // removed, but queued work may still read its slot and block
  size_t off = 0, bytes = 0;
  SimPlan plan;
  long long steps_total = 0;
};

// A removed simulation's arena block and slot, released once the work queued
// before the removal (on the step stream and the read-back stream) is done.
struct Pending {
  size_t off = 0, bytes = 0;
  int slot = -1;
  cudaEvent_t ev_main = nullptr, ev_io = nullptr;
};

constexpr int kSnaps = 4;  // poll snapshots in flight

// Per slot: the steps it has left and its status (set at admission, on the
// upload stream, by a kernel: its arguments are copied at launch).
__global__ void set_slot_kernel(long long *left, int *status, int slot, long long nsteps) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    left[slot] = nsteps;
    status[slot] = 0;
  }
}

}  // namespace

struct smaug_batch {
  int D = 0, device = 0;
  bool mixed = false;
  int max_inst = 0;
  cudaStream_t stream = nullptr, cap = nullptr;
  char *arena = nullptr;
  size_t arena_bytes = 0;
  std::map<size_t, size_t> free_;  // offset -> size
  BatchInst *d_tab = nullptr;
  long long *d_left = nullptr;
  int *d_status = nullptr;
  std::vector<BatchInst> h_tab;
  std::vector<Slot> slots;
  WorkItem *d_work = nullptr;
  WorkItem *d_gwork = nullptr;  // ghost chunks (256 ghost cells of one simulation each)
  size_t gwork_cap = 0;
  int ngwork = 0, ggrid = 0;
  size_t work_cap = 0;
  int nwork = 0, grid = 0, variant = 0, sms = 148;
  bool dirty = true;
  cudaGraphExec_t g1 = nullptr, gk = nullptr;
  long long launches = 0;
  // stage timing: steps are then launched directly, each stage kernel
  // bracketed by events
  bool profile = false;
  std::vector<cudaEvent_t> ev;
  size_t ev_used = 0;
  std::string err;
  // Admissions run on `up`, asynchronous state reads on `io`, so that neither
  // waits for the steps queued on `stream`; the step stream waits for the
  // admissions before its next launch (up_done).
  cudaStream_t up = nullptr, io = nullptr;
  cudaEvent_t up_done = nullptr;
  bool up_dirty = false;
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> ev_pool;
  // poll snapshots: steps left per slot, copied into pinned memory behind the
  // steps queued so far (ticket t uses ring entry t % kSnaps)
  long long *snap_h[kSnaps] = {};
  cudaEvent_t snap_ev[kSnaps] = {};
  long long snap_ticket[kSnaps] = {-1, -1, -1, -1};
  long long next_ticket = 0;
  int last_snap = -1;  // ring entry of the last snapshot waited for (asynchronous reads follow it)
  // pinned staging of the work lists and the table (two sets, used in turn)
  BatchInst *st_tab[2] = {};
  WorkItem *st_work[2] = {}, *st_gwork[2] = {};
  size_t st_work_cap[2] = {}, st_gwork_cap[2] = {};
  cudaEvent_t st_ev[2] = {};
  int st_cur = 0;
};

namespace {

int bfail(smaug_batch *b, int code, const std::string &m) {
  if (b) b->err = m;
  return code;
}

#define BK(call)                                                                                         \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) return bfail(b, SMAUG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

bool arena_alloc(smaug_batch *b, size_t bytes, size_t *off) {
  for (auto it = b->free_.begin(); it != b->free_.end(); ++it) {
    if (it->second >= bytes) {
      *off = it->first;
      const size_t rest = it->second - bytes, o = it->first + bytes;
      b->free_.erase(it);
      if (rest) b->free_[o] = rest;
      return true;
    }
  }
  return false;
}

void arena_free(smaug_batch *b, size_t off, size_t bytes) {
  auto it = b->free_.emplace(off, bytes).first;
  auto nx = std::next(it);
  if (nx != b->free_.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    b->free_.erase(nx);
  }
  if (it != b->free_.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      b->free_.erase(it);
    }
  }
}

void drop_graphs(smaug_batch *b) {
  if (b->g1) cudaGraphExecDestroy(b->g1);
  if (b->gk) cudaGraphExecDestroy(b->gk);
  b->g1 = b->gk = nullptr;
}

// Tiles per dim of a simulation for the batch's tile shape.
void set_tiles(const smaug_batch *b, BatchInst &I) {
  int t[3];
  batch_tile_shape(b->D, b->variant, t);
  for (int d = 0; d < 3; ++d) I.tiles[d] = d < b->D ? (I.geo.n[d] - 4 + t[d] - 1) / t[d] : 1;
}

// Rebuild the work list and the persistent grid for the current simulations
// and tile shape.
// Grow pinned staging buffer k of `what` (its copies from two rebuilds ago
// are done: the caller waited for st_ev[k]).
int stage_grow(smaug_batch *b, WorkItem **buf, size_t *cap, size_t need) {
  if (need <= *cap) return SMAUG_OK;
  if (*buf) cudaFreeHost(*buf);
  *buf = nullptr;
  *cap = std::max(need, (size_t)1024) * 2;
  BK(cudaMallocHost((void **)buf, sizeof(WorkItem) * *cap));
  return SMAUG_OK;
}

// Rebuild the work list and the persistent grid for the current simulations
// and tile shape.  The table and the lists go to the device from pinned
// staging buffers (two sets, used in turn), so nothing here waits for the
// steps already queued, except when a device list must grow.
int rebuild(smaug_batch *b) {
  std::vector<WorkItem> w, gw;
  for (int i = 0; i < b->max_inst; ++i) {
    if (!b->slots[i].used) continue;
    set_tiles(b, b->h_tab[i]);
    const int *tl = b->h_tab[i].tiles;
    for (int z = 0; z < tl[2]; ++z)
      for (int y = 0; y < tl[1]; ++y)
        for (int x = 0; x < tl[0]; ++x) w.push_back({i, x, y, z});
    const long long ng = ghost_cells(b->h_tab[i].geo, b->D);
    for (long long t = 0; t < (ng + 255) / 256; ++t) gw.push_back({i, (int)t, 0, 0});
  }
  if (gw.size() > b->gwork_cap || w.size() > b->work_cap) {  // queued steps read the device lists
    BK(cudaStreamSynchronize(b->stream));
    if (gw.size() > b->gwork_cap) {
      if (b->d_gwork) cudaFree(b->d_gwork);
      b->gwork_cap = std::max(gw.size(), (size_t)1024) * 2;
      BK(cudaMalloc(&b->d_gwork, sizeof(WorkItem) * b->gwork_cap));
    }
    if (w.size() > b->work_cap) {
      if (b->d_work) cudaFree(b->d_work);
      b->work_cap = std::max(w.size(), (size_t)1024) * 2;
      BK(cudaMalloc(&b->d_work, sizeof(WorkItem) * b->work_cap));
    }
  }
  const int k = b->st_cur;
  b->st_cur ^= 1;
  BK(cudaEventSynchronize(b->st_ev[k]));  // the copies out of set k, two rebuilds ago
  int rc = stage_grow(b, &b->st_gwork[k], &b->st_gwork_cap[k], gw.size());
  if (rc != SMAUG_OK) return rc;
  rc = stage_grow(b, &b->st_work[k], &b->st_work_cap[k], w.size());
  if (rc != SMAUG_OK) return rc;
  std::memcpy(b->st_tab[k], b->h_tab.data(), sizeof(BatchInst) * b->max_inst);
  if (!gw.empty()) std::memcpy(b->st_gwork[k], gw.data(), sizeof(WorkItem) * gw.size());
  if (!w.empty()) std::memcpy(b->st_work[k], w.data(), sizeof(WorkItem) * w.size());
  if (!gw.empty())
    BK(cudaMemcpyAsync(b->d_gwork, b->st_gwork[k], sizeof(WorkItem) * gw.size(), cudaMemcpyHostToDevice, b->stream));
  BK(cudaMemcpyAsync(b->d_tab, b->st_tab[k], sizeof(BatchInst) * b->max_inst, cudaMemcpyHostToDevice, b->stream));
  if (!w.empty())
    BK(cudaMemcpyAsync(b->d_work, b->st_work[k], sizeof(WorkItem) * w.size(), cudaMemcpyHostToDevice, b->stream));
  BK(cudaEventRecord(b->st_ev[k], b->stream));
  b->ngwork = (int)gw.size();
  b->ggrid = std::min(b->ngwork, 148 * 8);
  b->nwork = (int)w.size();
  const int occ = std::max(1, smaug_batchk::batch_stage_occupancy(b->D, b->mixed, b->variant));
  b->grid = std::min(b->nwork, occ * b->sms);
  drop_graphs(b);
  b->dirty = false;
  return SMAUG_OK;
}

// The step stream waits for the admissions queued on the upload stream.
int join_uploads(smaug_batch *b) {
  if (!b->up_dirty) return SMAUG_OK;
  BK(cudaEventRecord(b->up_done, b->up));
  BK(cudaStreamWaitEvent(b->stream, b->up_done, 0));
  b->up_dirty = false;
  return SMAUG_OK;
}

cudaEvent_t pool_event(smaug_batch *b) {
  if (!b->ev_pool.empty()) {
    cudaEvent_t e = b->ev_pool.back();
    b->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
  return e;
}

// Release the blocks and slots of removed simulations whose queued work is
// done (wait: also those whose work is still queued, waiting for it).
int reclaim(smaug_batch *b, bool wait) {
  for (size_t i = 0; i < b->pending.size();) {
    Pending &q = b->pending[i];
    if (wait) {
      BK(cudaEventSynchronize(q.ev_main));
      BK(cudaEventSynchronize(q.ev_io));
    } else if (cudaEventQuery(q.ev_main) != cudaSuccess || cudaEventQuery(q.ev_io) != cudaSuccess) {
      ++i;
      continue;
    }
    arena_free(b, q.off, q.bytes);
    b->slots[q.slot].pending = false;
    b->ev_pool.push_back(q.ev_main);
    b->ev_pool.push_back(q.ev_io);
    b->pending.erase(b->pending.begin() + i);
  }
  cudaGetLastError();  // a not-ready query leaves no error behind
  return SMAUG_OK;
}

void enqueue_step(smaug_batch *b, cudaStream_t s, bool timed = false) {
  const int nb = (b->max_inst + 127) / 128;
  batch_dt_kernel<<<nb, 128, 0, s>>>(b->d_tab, b->d_left, b->d_status, b->max_inst, b->D);
  for (int k = 1; k <= 4; ++k) {
    cudaEvent_t e1 = nullptr;
    if (timed) {
      while (b->ev.size() < b->ev_used + 2) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) break;
        b->ev.push_back(e);
      }
      if (b->ev.size() >= b->ev_used + 2) {
        cudaEventRecord(b->ev[b->ev_used], s);
        e1 = b->ev[b->ev_used + 1];
        b->ev_used += 2;
      }
    }
    smaug_batchk::launch_batch_stage(b->D, b->mixed, b->variant, b->d_tab, b->d_work, b->nwork, k, b->grid, s);
    if (e1) cudaEventRecord(e1, s);
    smaug_batchk::launch_batch_ghost(b->D, b->mixed, b->d_tab, b->d_gwork, b->ngwork, k, b->ggrid, s);
  }
  batch_finish_kernel<<<nb, 128, 0, s>>>(b->d_tab, b->d_status, b->max_inst);
}

int capture(smaug_batch *b, int steps, cudaGraphExec_t *out) {
  cudaGraph_t g = nullptr;
  BK(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < steps; ++i) enqueue_step(b, b->cap);
  BK(cudaStreamEndCapture(b->cap, &g));
  cudaError_t e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  BK(e);
  return SMAUG_OK;
}

}  // namespace

extern "C" {

int smaug_batch_footprint(const smaug_params *prm, size_t *bytes) {
  if (!prm || !bytes) return SMAUG_ERR_ARG;
  SimPlan p;
  if (plan_sim(prm, p)) return SMAUG_ERR_ARG;
  *bytes = sim_footprint(p);
  return SMAUG_OK;
}

int smaug_batch_create(int ndim, int precision, int device, size_t arena_bytes, int max_sims, smaug_batch **out) {
  if (!out) return SMAUG_ERR_ARG;
  *out = nullptr;
  smaug_batch *b = new smaug_batch();
  *out = b;
  if (ndim != 2 && ndim != 3) return bfail(b, SMAUG_ERR_ARG, "ndim must be 2 or 3");
  if (precision != SMAUG_PREC_FP64 && precision != SMAUG_PREC_MIXED)
    return bfail(b, SMAUG_ERR_ARG, "precision must be SMAUG_PREC_FP64 or SMAUG_PREC_MIXED");
  if (max_sims < 1 || max_sims > (1 << 16)) return bfail(b, SMAUG_ERR_ARG, "max_sims must be 1..65536");
  if (arena_bytes < 4096) return bfail(b, SMAUG_ERR_ARG, "arena too small");
  b->D = ndim;
  b->mixed = precision == SMAUG_PREC_MIXED;
  b->variant = batch_default_variant(ndim, b->mixed);
  b->device = device;
  b->max_inst = max_sims;
  b->arena_bytes = arena_bytes & ~(size_t)255;
  b->h_tab.assign(max_sims, BatchInst{});
  b->slots.assign(max_sims, Slot{});
  BK(cudaSetDevice(device));
  int sms = 0;
  BK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  b->sms = sms > 0 ? sms : 148;
  BK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  BK(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  BK(cudaStreamCreateWithFlags(&b->up, cudaStreamNonBlocking));
  BK(cudaStreamCreateWithFlags(&b->io, cudaStreamNonBlocking));
  BK(cudaEventCreateWithFlags(&b->up_done, cudaEventDisableTiming));
  for (int k = 0; k < kSnaps; ++k) {
    BK(cudaMallocHost((void **)&b->snap_h[k], sizeof(long long) * max_sims));
    BK(cudaEventCreateWithFlags(&b->snap_ev[k], cudaEventDisableTiming));
  }
  for (int k = 0; k < 2; ++k) {
    BK(cudaMallocHost((void **)&b->st_tab[k], sizeof(BatchInst) * max_sims));
    BK(cudaEventCreateWithFlags(&b->st_ev[k], cudaEventDisableTiming));
  }
  BK(cudaMalloc(&b->arena, b->arena_bytes));
  b->free_[0] = b->arena_bytes;
  BK(cudaMalloc(&b->d_tab, sizeof(BatchInst) * max_sims));
  BK(cudaMalloc(&b->d_left, sizeof(long long) * max_sims));
  BK(cudaMalloc(&b->d_status, sizeof(int) * max_sims));
  BK(cudaMemsetAsync(b->d_tab, 0, sizeof(BatchInst) * max_sims, b->stream));
  BK(cudaMemsetAsync(b->d_left, 0, sizeof(long long) * max_sims, b->stream));
  BK(cudaMemsetAsync(b->d_status, 0, sizeof(int) * max_sims, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  return SMAUG_OK;
}

int smaug_batch_destroy(smaug_batch *b) {
  if (!b) return SMAUG_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->up) cudaStreamSynchronize(b->up);
  if (b->io) cudaStreamSynchronize(b->io);
  drop_graphs(b);
  for (auto e : b->ev) cudaEventDestroy(e);
  cudaFree(b->arena);
  cudaFree(b->d_tab);
  cudaFree(b->d_left);
  cudaFree(b->d_status);
  cudaFree(b->d_work);
  cudaFree(b->d_gwork);
  for (auto &q : b->pending) {
    if (q.ev_main) cudaEventDestroy(q.ev_main);
    if (q.ev_io) cudaEventDestroy(q.ev_io);
  }
  for (auto e : b->ev_pool) cudaEventDestroy(e);
  for (int k = 0; k < kSnaps; ++k) {
    if (b->snap_h[k]) cudaFreeHost(b->snap_h[k]);
    if (b->snap_ev[k]) cudaEventDestroy(b->snap_ev[k]);
  }
  for (int k = 0; k < 2; ++k) {
    if (b->st_tab[k]) cudaFreeHost(b->st_tab[k]);
    if (b->st_work[k]) cudaFreeHost(b->st_work[k]);
    if (b->st_gwork[k]) cudaFreeHost(b->st_gwork[k]);
    if (b->st_ev[k]) cudaEventDestroy(b->st_ev[k]);
  }
  if (b->up_done) cudaEventDestroy(b->up_done);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (b->cap) cudaStreamDestroy(b->cap);
  if (b->up) cudaStreamDestroy(b->up);
  if (b->io) cudaStreamDestroy(b->io);
  delete b;
  return SMAUG_OK;
}

int smaug_batch_add(smaug_batch *b, const smaug_params *prm, const double *delx, const double *w, long long nsteps,
                    int *slot_out) {
  if (!b || !prm || !delx || !w || !slot_out || nsteps < 0) return SMAUG_ERR_ARG;
  *slot_out = -1;
  SimPlan p;
  if (const char *m = plan_sim(prm, p)) return bfail(b, SMAUG_ERR_ARG, m);
  if (p.D != b->D) return bfail(b, SMAUG_ERR_ARG, "simulation ndim differs from the batch's");
  if (p.mixed != b->mixed) return bfail(b, SMAUG_ERR_ARG, "simulation precision differs from the batch's");
  if (!p.rk4 || p.exact) return bfail(b, SMAUG_ERR_ARG, "batch simulations use rk4 = 1 and exact = 0");
  const long long N = p.geo.N;
  // one line per dim here; the metric itself is checked on the device below
  const size_t nl = (size_t)p.geo.n[0] + p.geo.n[1] + p.geo.n[2];
  std::vector<double> d1(2 * nl);  // the lines, then their reciprocals
  metric_lines_host(p, delx, d1.data());
  for (size_t i = 0; i < nl; ++i) d1[nl + i] = 1.0 / d1[i];
  BK(cudaSetDevice(b->device));
  // a slot and a block: first from what is free now, then, if removed
  // simulations still wait for their queued work, after waiting for it
  const size_t fp = sim_footprint(p);
  int slot = -1;
  size_t off = 0;
  for (int attempt = 0; attempt < 2 && slot < 0; ++attempt) {
    const int rc = reclaim(b, attempt == 1);
    if (rc != SMAUG_OK) return rc;
    int cand = -1;
    for (int i = 0; i < b->max_inst; ++i)
      if (!b->slots[i].used && !b->slots[i].pending) {
        cand = i;
        break;
      }
    if (cand >= 0 && arena_alloc(b, fp, &off)) slot = cand;
    if (b->pending.empty()) break;
  }
  if (slot < 0) return bfail(b, SMAUG_ERR_FULL, "no free simulation slot or arena block of the simulation's footprint");
  // every return below that does not admit the simulation releases its block
  // (stream order keeps a later admission's uploads behind any copy queued here)
  struct BlockGuard {
    smaug_batch *b;
    size_t off, bytes;
    bool keep = false;
    ~BlockGuard() {
      if (!keep) arena_free(b, off, bytes);
    }
  } guard{b, off, fp};
  // carve
  char *q = b->arena + off;
  auto take = [&](size_t bytes) {
    char *r = q;
    q += align256(bytes);
    return r;
  };
  DevScalars *sc = (DevScalars *)take(sizeof(DevScalars));
  double *dx1 = (double *)take(sizeof(double) * d1.size());
  double *drv = (double *)take(sizeof(double) * nl);
  std::vector<double> drv_host(nl);
  driver_lines(p, prm, drv_host.data());
  double *dxlast = (double *)take(sizeof(double) * N);
  double *bg = (double *)take(sizeof(double) * p.NB * N);
  BatchInst I{};
  I.W[0] = (double *)take(sizeof(double) * p.NW * N);
  if (p.mixed)
    for (auto &f : I.F) f = (float *)take(sizeof(float) * p.NW * N);
  else
    for (int k = 1; k < 4; ++k) I.W[k] = (double *)take(sizeof(double) * p.NW * N);
  const double *bh = w + (size_t)N * p.NW;
  // Whether the energy background terms are live is found on the device
  // (bg_scan_kernel) and set after the load; the load's initial maxima read
  // the backgrounds either way (zeros give the same values).
  p.phys.has_bgb = 1;
  size_t o1 = 0;
  for (int d = 0; d < p.D; ++d) {
    p.geo.dx1[d] = dx1 + o1;
    p.geo.rdx1[d] = dx1 + nl + o1;
    o1 += p.geo.n[d];
  }
  p.geo.dxlast = dxlast;
  o1 = 0;
  for (int d = 0; d < 3; ++d) {
    p.geo.drvf[d] = drv + o1;
    o1 += p.geo.n[d];
  }
  I.geo = p.geo;
  I.phys = p.phys;
  I.bg = bg;
  I.sc = sc;
  I.active = 1;
  // the admission's own stream: it neither waits for the queued steps nor
  // touches their memory (the slot and the block are not referenced by any of
  // them); the step stream waits for it before its next launch
  cudaStream_t s = b->up;
  // The full metric goes to a stage buffer that nothing uses before the
  // first step (mixed F[2]: NW >= 2 D floats per cell; FP64 W[1]) for its
  // check; the last dim's array stays as dxlast.
  double *mscratch = p.mixed ? (double *)(void *)I.F[2] : I.W[1];
  BK(cudaMemsetAsync(sc, 0, sizeof(DevScalars), s));
  BK(cudaMemcpyAsync(dx1, d1.data(), sizeof(double) * d1.size(), cudaMemcpyHostToDevice, s));
  BK(cudaMemcpyAsync(drv, drv_host.data(), sizeof(double) * drv_host.size(), cudaMemcpyHostToDevice, s));
  BK(cudaMemcpyAsync(mscratch, delx, sizeof(double) * p.D * N, cudaMemcpyHostToDevice, s));
  BK(cudaMemcpyAsync(dxlast, mscratch + (size_t)(p.D - 1) * N, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  BK(cudaMemcpyAsync(I.W[0], w, sizeof(double) * p.NW * N, cudaMemcpyHostToDevice, s));
  BK(cudaMemcpyAsync(bg, bh, sizeof(double) * p.NB * N, cudaMemcpyHostToDevice, s));
  ghost_fill(I.W[0], p.NW, p.geo, p.D, s);
  const double dt0 = p.phys.dt_mode == 1 ? (p.dt0 > 0 ? p.dt0 : 1.0e-8) : p.dt0;
  one_reset_kernel<<<1, 1, 0, s>>>(sc, dt0);  // status 0
  minsq_init_kernel<<<1, 1, 0, s>>>(sc);
  metric_kernel<<<b->sms * 4, 256, 0, s>>>(mscratch, p.geo, p.D, nullptr, sc);
  bg_scan_kernel<<<b->sms * 4, 256, 0, s>>>(bg, N, p.D, sc);
  smaug_fast::launch_reduce(p.D, I.W[0], bg, p.geo, p.phys, &sc->red[0], s, 0);
  if (p.geo.has_const) smaug_fast::launch_reduce(p.D, I.W[0], bg, p.geo, p.phys, &sc->floor, s, 1);
  if (p.mixed) split_kernel<<<148 * 8, 256, 0, s>>>(I.W[0], I.F[0], I.F[1], (long long)p.NW * N);
  b->launches += p.D + 5 + (p.mixed ? 1 : 0) + (p.geo.has_const ? 1 : 0);
  BK(cudaGetLastError());
  if (p.geo.has_const) {  // fixed boundaries: every stage buffer holds the loaded ghosts
    const size_t n = (size_t)p.NW * N;
    if (p.mixed) {
      for (int k = 2; k < 4; ++k)
        BK(cudaMemcpyAsync(I.F[k], I.F[0], sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
    } else {
      for (int k = 1; k < 4; ++k)
        BK(cudaMemcpyAsync(I.W[k], I.W[0], sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }
  }
  int chk[2] = {0, 0};  // metric status, live background
  BK(cudaMemcpyAsync(&chk[0], &sc->status, sizeof(int), cudaMemcpyDeviceToHost, s));
  BK(cudaMemcpyAsync(&chk[1], &sc->bg_live, sizeof(int), cudaMemcpyDeviceToHost, s));
  BK(cudaStreamSynchronize(s));  // the sources above are host temporaries
  if (chk[0] != 0) {
    return bfail(b, SMAUG_ERR_ARG, "metric is not a tensor-product grid on the inner cells, or has a non-positive entry");
  }
  p.phys.has_bgb = chk[1];
  I.phys = p.phys;
  set_slot_kernel<<<1, 1, 0, s>>>(b->d_left, b->d_status, slot, nsteps);
  BK(cudaGetLastError());
  b->up_dirty = true;
  guard.keep = true;
  Slot &S = b->slots[slot];
  S.used = true;
  S.off = off;
  S.bytes = fp;
  S.plan = p;
  S.steps_total = nsteps;
  b->h_tab[slot] = I;
  b->dirty = true;
  *slot_out = slot;
  return SMAUG_OK;
}

int smaug_batch_remove(smaug_batch *b, int slot) {
  if (!b || slot < 0 || slot >= b->max_inst || !b->slots[slot].used) return SMAUG_ERR_ARG;
  BK(cudaSetDevice(b->device));
  // Steps queued before now, and state reads queued on the read-back stream,
  // may still read the slot's table entry, its steps-left counter and its
  // block: both are released once that work is done (reclaim, at the next
  // admission).  Later steps no longer include the simulation.
  Pending q;
  q.off = b->slots[slot].off;
  q.bytes = b->slots[slot].bytes;
  q.slot = slot;
  q.ev_main = pool_event(b);
  q.ev_io = pool_event(b);
  if (!q.ev_main || !q.ev_io) return bfail(b, SMAUG_ERR_CUDA, "no CUDA event for a removal");
  BK(cudaEventRecord(q.ev_main, b->stream));
  BK(cudaEventRecord(q.ev_io, b->io));
  b->pending.push_back(q);
  b->h_tab[slot] = BatchInst{};
  b->slots[slot] = Slot{};
  b->slots[slot].pending = true;
  b->dirty = true;
  return SMAUG_OK;
}

int smaug_batch_step(smaug_batch *b, int nsteps) {
  if (!b || nsteps < 0) return SMAUG_ERR_ARG;
  BK(cudaSetDevice(b->device));
  {
    const int rc = join_uploads(b);
    if (rc != SMAUG_OK) return rc;
  }
  if (b->dirty) {
    int rc = rebuild(b);
    if (rc != SMAUG_OK) return rc;
  }
  if (b->nwork == 0) return SMAUG_OK;
  if (b->profile) {
    for (int i = 0; i < nsteps; ++i) enqueue_step(b, b->stream, true);
    b->launches += (long long)kLaunchesPerStep * nsteps;
    BK(cudaGetLastError());
    return SMAUG_OK;
  }
  if (nsteps >= kGraphSteps && !b->gk) {
    int rc = capture(b, kGraphSteps, &b->gk);
    if (rc != SMAUG_OK) return rc;
  }
  if (nsteps % kGraphSteps && !b->g1) {
    int rc = capture(b, 1, &b->g1);
    if (rc != SMAUG_OK) return rc;
  }
  for (int i = 0; i + kGraphSteps <= nsteps; i += kGraphSteps) {
    BK(cudaGraphLaunch(b->gk, b->stream));
    b->launches += (long long)kLaunchesPerStep * kGraphSteps;
  }
  for (int i = 0; i < nsteps % kGraphSteps; ++i) {
    BK(cudaGraphLaunch(b->g1, b->stream));
    b->launches += kLaunchesPerStep;
  }
  return SMAUG_OK;
}

int smaug_batch_poll(smaug_batch *b, long long *steps_left, int n) {
  if (!b || !steps_left || n < b->max_inst) return SMAUG_ERR_ARG;
  BK(cudaSetDevice(b->device));
  {
    const int rc_ = join_uploads(b);
    if (rc_ != SMAUG_OK) return rc_;
  }
  BK(cudaMemcpyAsync(steps_left, b->d_left, sizeof(long long) * b->max_inst, cudaMemcpyDeviceToHost, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  for (int i = 0; i < b->max_inst; ++i)
    if (!b->slots[i].used) steps_left[i] = -1;
  return SMAUG_OK;
}

int smaug_batch_poll_begin(smaug_batch *b, long long *ticket) {
  if (!b || !ticket) return SMAUG_ERR_ARG;
  BK(cudaSetDevice(b->device));
  {
    const int rc_ = join_uploads(b);
    if (rc_ != SMAUG_OK) return rc_;
  }
  const long long t = b->next_ticket;
  const int k = (int)(t % kSnaps);
  if (b->snap_ticket[k] >= 0) return bfail(b, SMAUG_ERR_STATE, "more than 4 poll snapshots waiting: end one first");
  BK(cudaMemcpyAsync(b->snap_h[k], b->d_left, sizeof(long long) * b->max_inst, cudaMemcpyDeviceToHost, b->stream));
  BK(cudaEventRecord(b->snap_ev[k], b->stream));
  b->snap_ticket[k] = t;
  b->next_ticket = t + 1;
  *ticket = t;
  return SMAUG_OK;
}

int smaug_batch_poll_end(smaug_batch *b, long long ticket, long long *steps_left, int n) {
  if (!b || !steps_left || n < b->max_inst || ticket < 0) return SMAUG_ERR_ARG;
  const int k = (int)(ticket % kSnaps);
  if (b->snap_ticket[k] != ticket) return bfail(b, SMAUG_ERR_STATE, "no such poll snapshot waiting");
  BK(cudaSetDevice(b->device));
  BK(cudaEventSynchronize(b->snap_ev[k]));
  std::memcpy(steps_left, b->snap_h[k], sizeof(long long) * b->max_inst);
  for (int i = 0; i < b->max_inst; ++i)
    if (!b->slots[i].used) steps_left[i] = -1;
  b->snap_ticket[k] = -1;
  b->last_snap = k;
  return SMAUG_OK;
}

int smaug_batch_get_state_async(smaug_batch *b, int slot, double *w, size_t count) {
  if (!b || !w || slot < 0 || slot >= b->max_inst || !b->slots[slot].used) return SMAUG_ERR_ARG;
  if (b->last_snap < 0) return bfail(b, SMAUG_ERR_STATE, "smaug_batch_get_state_async follows smaug_batch_poll_end");
  const SimPlan &p = b->slots[slot].plan;
  const BatchInst &I = b->h_tab[slot];
  const long long N = p.geo.N;
  if (count != (size_t)p.NVAR * (size_t)N) return bfail(b, SMAUG_ERR_ARG, "state must hold NVAR * N doubles");
  BK(cudaSetDevice(b->device));
  // after the steps the last waited-for snapshot followed; the steps queued
  // since do not write a simulation that had finished by then
  BK(cudaStreamWaitEvent(b->io, b->snap_ev[b->last_snap], 0));
  if (p.mixed) {
    combine_kernel<<<148 * 4, 256, 0, b->io>>>(I.F[0], I.F[1], I.W[0], (long long)p.NW * N);
    b->launches++;
    BK(cudaGetLastError());
  }
  BK(cudaMemcpyAsync(w, I.W[0], sizeof(double) * p.NW * N, cudaMemcpyDeviceToHost, b->io));
  BK(cudaMemcpyAsync(w + (size_t)p.NW * N, I.bg, sizeof(double) * p.NB * N, cudaMemcpyDeviceToHost, b->io));
  return SMAUG_OK;
}

int smaug_batch_io_wait(smaug_batch *b) {
  if (!b) return SMAUG_ERR_ARG;
  BK(cudaSetDevice(b->device));
  BK(cudaStreamSynchronize(b->io));
  return SMAUG_OK;
}

int smaug_batch_sync(smaug_batch *b, int *bad_slot) {
  if (!b) return SMAUG_ERR_ARG;
  if (bad_slot) *bad_slot = -1;
  BK(cudaSetDevice(b->device));
  {
    const int rc_ = join_uploads(b);
    if (rc_ != SMAUG_OK) return rc_;
  }
  std::vector<int> st(b->max_inst);
  BK(cudaMemcpyAsync(st.data(), b->d_status, sizeof(int) * b->max_inst, cudaMemcpyDeviceToHost, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  for (int i = 0; i < b->max_inst; ++i)
    if (b->slots[i].used && st[i] != 0) {
      if (bad_slot) *bad_slot = i;
      return bfail(b, st[i], "simulation " + std::to_string(i) + ": non-finite dt or wave speed");
    }
  return SMAUG_OK;
}

int smaug_batch_get_state(smaug_batch *b, int slot, double *w, size_t count) {
  if (!b || !w || slot < 0 || slot >= b->max_inst || !b->slots[slot].used) return SMAUG_ERR_ARG;
  const SimPlan &p = b->slots[slot].plan;
  const BatchInst &I = b->h_tab[slot];
  const long long N = p.geo.N;
  if (count != (size_t)p.NVAR * (size_t)N) return bfail(b, SMAUG_ERR_ARG, "state must hold NVAR * N doubles");
  BK(cudaSetDevice(b->device));
  {
    const int rc_ = join_uploads(b);
    if (rc_ != SMAUG_OK) return rc_;
  }
  if (p.mixed) {
    combine_kernel<<<148 * 8, 256, 0, b->stream>>>(I.F[0], I.F[1], I.W[0], (long long)p.NW * N);
    b->launches++;
    BK(cudaGetLastError());
  }
  BK(cudaMemcpyAsync(w, I.W[0], sizeof(double) * p.NW * N, cudaMemcpyDeviceToHost, b->stream));
  BK(cudaMemcpyAsync(w + (size_t)p.NW * N, I.bg, sizeof(double) * p.NB * N, cudaMemcpyDeviceToHost, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  return SMAUG_OK;
}

int smaug_batch_get_scalars(smaug_batch *b, int slot, double out[8]) {
  if (!b || !out || slot < 0 || slot >= b->max_inst || !b->slots[slot].used) return SMAUG_ERR_ARG;
  BK(cudaSetDevice(b->device));
  {
    const int rc_ = join_uploads(b);
    if (rc_ != SMAUG_OK) return rc_;
  }
  DevScalars s;
  long long left = 0;
  BK(cudaMemcpyAsync(&s, b->h_tab[slot].sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, b->stream));
  BK(cudaMemcpyAsync(&left, b->d_left + slot, sizeof(long long), cudaMemcpyDeviceToHost, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  out[0] = s.dt;
  out[1] = s.maxcourant;
  out[2] = s.maxviscoef;
  out[3] = s.dtdiffvisc;
  for (int d = 0; d < 3; ++d) out[4 + d] = d < b->D ? red_get(s.red[0], d) : 0.0;
  out[7] = (double)(b->slots[slot].steps_total - left);
  return SMAUG_OK;
}

int smaug_batch_tune(smaug_batch *b, int reps, int *variant_out, double *ms_out, int nms) {
  if (!b || reps < 1) return SMAUG_ERR_ARG;
  BK(cudaSetDevice(b->device));
  {
    const int rc_ = join_uploads(b);
    if (rc_ != SMAUG_OK) return rc_;
  }
  const int nv = b->D == 2 ? kBatchVariants2 : kBatchVariants3;
  cudaEvent_t e0, e1;
  BK(cudaEventCreate(&e0));
  BK(cudaEventCreate(&e1));
  int best = b->variant;
  float best_ms = 1e30f;
  for (int v = 0; v < nv; ++v) {
    // a shape that cannot be resident on this device (its shared memory or
    // registers) is not timed: ms -1
    if (smaug_batchk::batch_stage_occupancy(b->D, b->mixed, v) <= 0) {
      (void)cudaGetLastError();
      if (ms_out && v < nms) ms_out[v] = -1.0;
      continue;
    }
    b->variant = v;
    int rc = rebuild(b);
    if (rc != SMAUG_OK) return rc;
    if (b->nwork == 0) break;
    batch_go_kernel<<<(b->max_inst + 127) / 128, 128, 0, b->stream>>>(b->d_tab, b->max_inst);
    smaug_batchk::launch_batch_stage(b->D, b->mixed, v, b->d_tab, b->d_work, b->nwork, 1, b->grid, b->stream);
    BK(cudaEventRecord(e0, b->stream));
    for (int r = 0; r < reps; ++r)
      smaug_batchk::launch_batch_stage(b->D, b->mixed, v, b->d_tab, b->d_work, b->nwork, 1, b->grid, b->stream);
    BK(cudaEventRecord(e1, b->stream));
    BK(cudaEventSynchronize(e1));
    // a launch that the device refused (a configuration error, reported
    // synchronously) has timed nothing
    if (cudaGetLastError() != cudaSuccess) {
      if (ms_out && v < nms) ms_out[v] = -1.0;
      continue;
    }
    float ms = 0.f;
    BK(cudaEventElapsedTime(&ms, e0, e1));
    ms /= reps;
    b->launches += reps + 2;
    if (ms_out && v < nms) ms_out[v] = ms;
    if (ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->variant = best;
  b->dirty = true;
  if (variant_out) *variant_out = best;
  return SMAUG_OK;
}

int smaug_batch_set_variant(smaug_batch *b, int variant) {
  if (!b) return SMAUG_ERR_ARG;
  const int nv = b->D == 2 ? kBatchVariants2 : kBatchVariants3;
  if (variant < 0 || variant >= nv) return bfail(b, SMAUG_ERR_ARG, "no such tile variant");
  BK(cudaSetDevice(b->device));
  if (smaug_batchk::batch_stage_occupancy(b->D, b->mixed, variant) <= 0) {
    (void)cudaGetLastError();
    return bfail(b, SMAUG_ERR_ARG, "tile variant cannot be resident on this device");
  }
  b->variant = variant;
  b->dirty = true;
  return SMAUG_OK;
}

int smaug_batch_info(smaug_batch *b, size_t *free_bytes, size_t *largest_free, int *sims) {
  if (!b) return SMAUG_ERR_ARG;
  size_t tot = 0, big = 0;
  for (auto &f : b->free_) {
    tot += f.second;
    big = std::max(big, f.second);
  }
  int n = 0;
  for (auto &s : b->slots) n += s.used;
  if (free_bytes) *free_bytes = tot;
  if (largest_free) *largest_free = big;
  if (sims) *sims = n;
  return SMAUG_OK;
}

int smaug_batch_profile_stages(smaug_batch *b, int enable) {
  if (!b) return SMAUG_ERR_ARG;
  b->profile = enable != 0;
  b->ev_used = 0;
  return SMAUG_OK;
}

int smaug_batch_stage_times(smaug_batch *b, double *ms_total, long long *count) {
  if (!b || !ms_total || !count) return SMAUG_ERR_ARG;
  BK(cudaSetDevice(b->device));
  BK(cudaStreamSynchronize(b->stream));
  double t = 0.0;
  for (size_t i = 0; i + 1 < b->ev_used; i += 2) {
    float ms = 0.f;
    BK(cudaEventElapsedTime(&ms, b->ev[i], b->ev[i + 1]));
    t += ms;
  }
  *ms_total = t;
  *count = (long long)(b->ev_used / 2);
  b->ev_used = 0;
  return SMAUG_OK;
}

void *smaug_batch_stream(smaug_batch *b) { return b ? (void *)b->stream : nullptr; }
long long smaug_batch_launch_count(smaug_batch *b) { return b ? b->launches : 0; }
const char *smaug_batch_last_error(smaug_batch *b) { return b ? b->err.c_str() : "null batch"; }

}  // extern "C"
