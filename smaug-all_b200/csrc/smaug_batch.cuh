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
  int tile;
};

// Tile shapes the batch kernels are built for (the autotuner picks one).
constexpr int kBatchVariants2 = 4;  // 2-D: 16x16, 32x8, 8x32, 32x16
constexpr int kBatchVariants3 = 3;  // 3-D: 8x8x4, 16x8x2, 32x4x2
__host__ __device__ inline void batch_tile_shape(int D, int v, int *t) {
  t[2] = 1;
  if (D == 2) {
    switch (v) {
      case 1: t[0] = 32; t[1] = 8; break;
      case 2: t[0] = 8; t[1] = 32; break;
      case 3: t[0] = 32; t[1] = 16; break;
      default: t[0] = 16; t[1] = 16; break;
    }
  } else {
    switch (v) {
      case 1: t[0] = 16; t[1] = 8; t[2] = 2; break;
      case 2: t[0] = 32; t[1] = 4; t[2] = 2; break;
      default: t[0] = 8; t[1] = 8; t[2] = 4; break;
    }
  }
}

}  // namespace smaug

namespace smaug_batchk {
// Launch one RK stage (1..4) for every work item whose simulation takes the
// current step (work == nullptr: items are the tiles of simulation 0).
// grid: persistent block count.
void launch_batch_stage(int D, bool mixed, int variant, const smaug::BatchInst *tab, const smaug::WorkItem *work,
                        int nwork, int stage, int grid, cudaStream_t st);
// Blocks per SM the stage kernel of (D, mixed, variant) can keep resident.
int batch_stage_occupancy(int D, bool mixed, int variant);
}  // namespace smaug_batchk
