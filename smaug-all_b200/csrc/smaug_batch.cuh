// smaug_batch.cuh -- device-side description of a batch: many independent
// simulations (same ndim and precision, any sizes) advanced together, one
// launch per RK stage for all of them.
#pragma once
#include "smaug_device.cuh"

namespace smaug {

// One simulation of a batch, resident in the batch's device table.
struct BatchInst {
  Geo geo;
  Phys phys;
  const double *bg;  // NB background fields
  double *W[4];      // FP64 path: state and the three RK stage buffers; mixed: W[0] only (load/store)
  float *F[5];       // mixed path: w32, c32, two FP32 stage states, FP32 RK sum
  DevScalars *sc;
  int tiles[3];      // tiles per dimension for the batch's current tile shape
  int active;        // slot holds a simulation
};

// Work list entry: simulation slot and tile index within it.
struct WorkItem {
  int inst;
  int tile;    // stage items: the tile's x index; ghost items: the chunk
  int by, bz;  // stage items: the tile's y and z indices
};

// Tile shapes and occupancy targets (resident blocks per SM the register
// allocation is made for) the stage kernel is built for; the autotuner picks
// one.  Variant 0 is the single-simulation default.
constexpr int kBatchVariants2 = 11;
constexpr int kBatchVariants3 = 10;
struct BatchVariant {
  int t[3];
  int min_blocks;
};
__host__ __device__ inline BatchVariant batch_variant(int D, int v) {
  if (D == 2) {
    switch (v) {
      case 1: return {{32, 8, 1}, 2};
      case 2: return {{8, 32, 1}, 2};
      case 3: return {{32, 16, 1}, 1};
      case 4: return {{16, 16, 1}, 3};
      case 5: return {{32, 8, 1}, 3};
      case 6: return {{16, 16, 1}, 4};
      case 7: return {{32, 8, 1}, 4};
      case 8: return {{16, 16, 1}, 5};
      case 9: return {{16, 8, 1}, 8};
      case 10: return {{32, 16, 1}, 2};
      default: return {{16, 16, 1}, 2};
    }
  }
  switch (v) {
    case 1: return {{16, 8, 2}, 2};
    case 2: return {{32, 4, 2}, 2};
    case 3: return {{8, 8, 4}, 3};
    case 4: return {{16, 8, 2}, 3};
    case 5: return {{8, 8, 4}, 4};
    case 6: return {{8, 8, 8}, 2};
    case 7: return {{16, 8, 4}, 2};
    case 8: return {{8, 8, 8}, 1};
    case 9: return {{16, 8, 4}, 1};
    default: return {{8, 8, 4}, 2};
  }
}

// Default variant of a single simulation and of an untuned batch (the
// serving loop's), per ndim and precision: the fastest of the variants in
// B200 sweeps of RK stage 1 on 96 Orszag-Tang simulations 128^2..768^2, on
// 48 driven atmosphere slices (the served mix) and on one 128^3 blast wave.  A batch
// and a single-simulation context on the same variant give the same bits.
__host__ __device__ inline int batch_default_variant(int D, bool mixed) {
  if (D == 2) return mixed ? 6 : 0;
  return mixed ? 6 : 9;
}

__host__ __device__ inline void batch_tile_shape(int D, int v, int *t) {
  const BatchVariant b = batch_variant(D, v);
  t[0] = b.t[0];
  t[1] = b.t[1];
  t[2] = b.t[2];
}

}  // namespace smaug

namespace smaug_batchk {
// per (ndim, stencil type) translation units (batch_k{2,3}{f,d}.cu)
void launch_batch_stage_2f(int, const smaug::BatchInst *, const smaug::WorkItem *, int, int, int, cudaStream_t);
void launch_batch_stage_2d(int, const smaug::BatchInst *, const smaug::WorkItem *, int, int, int, cudaStream_t);
void launch_batch_stage_3f(int, const smaug::BatchInst *, const smaug::WorkItem *, int, int, int, cudaStream_t);
void launch_batch_stage_3d(int, const smaug::BatchInst *, const smaug::WorkItem *, int, int, int, cudaStream_t);
void launch_batch_ghost_2f(const smaug::BatchInst *, const smaug::WorkItem *, int, int, int, cudaStream_t);
void launch_batch_ghost_2d(const smaug::BatchInst *, const smaug::WorkItem *, int, int, int, cudaStream_t);
void launch_batch_ghost_3f(const smaug::BatchInst *, const smaug::WorkItem *, int, int, int, cudaStream_t);
void launch_batch_ghost_3d(const smaug::BatchInst *, const smaug::WorkItem *, int, int, int, cudaStream_t);
int batch_stage_occupancy_2f(int);
int batch_stage_occupancy_2d(int);
int batch_stage_occupancy_3f(int);
int batch_stage_occupancy_3d(int);

// Launch one RK stage (1..4) for every work item whose simulation takes the
// current step (work == nullptr: items are the tiles of simulation 0).
// grid: persistent block count.
inline void launch_batch_stage(int D, bool mixed, int variant, const smaug::BatchInst *tab,
                               const smaug::WorkItem *work, int nwork, int stage, int grid, cudaStream_t st) {
  if (D == 2)
    (mixed ? launch_batch_stage_2f : launch_batch_stage_2d)(variant, tab, work, nwork, stage, grid, st);
  else
    (mixed ? launch_batch_stage_3f : launch_batch_stage_3d)(variant, tab, work, nwork, stage, grid, st);
}
// The ghost pass of RK stage `stage` (gwork == nullptr: the n chunks of
// simulation 0).
inline void launch_batch_ghost(int D, bool mixed, const smaug::BatchInst *tab, const smaug::WorkItem *gwork, int n,
                               int stage, int grid, cudaStream_t st) {
  if (D == 2)
    (mixed ? launch_batch_ghost_2f : launch_batch_ghost_2d)(tab, gwork, n, stage, grid, st);
  else
    (mixed ? launch_batch_ghost_3f : launch_batch_ghost_3d)(tab, gwork, n, stage, grid, st);
}
// Blocks per SM the stage kernel of (D, mixed, variant) can keep resident.
inline int batch_stage_occupancy(int D, bool mixed, int variant) {
  if (D == 2) return mixed ? batch_stage_occupancy_2f(variant) : batch_stage_occupancy_2d(variant);
  return mixed ? batch_stage_occupancy_3f(variant) : batch_stage_occupancy_3d(variant);
}
}  // namespace smaug_batchk
