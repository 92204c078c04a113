// batch_kernels.cu -- the production RK4 stage kernel: one persistent launch
// per RK stage walks a work list of (simulation, tile) items over every
// simulation of a batch (a single-simulation context is a table of one
// simulation and no list: item w is its tile w).  Each item runs the same tile body as the
// single-simulation kernel (smaug_tile.cuh), so a simulation's results do not
// depend on what else is in the batch or on the tile shape: the arithmetic of
// a cell is the same, and the maxima are order-independent.
// Built with FMA contraction and FP32 subnormal flushing, like stage_fast.cu.
#define SMAUG_NS smaug_batchk
#define SMAUG_TILED 1
#include <cuda_runtime.h>

#include "smaug_batch.cuh"
#include "smaug_stage.cuh"
#include "smaug_tile.cuh"

namespace smaug_batchk {
using namespace smaug;

// The stage's buffers for one simulation: mixed RK stage k reads F[in] and
// writes F[out] (stage 4 writes the base w32/c32); FP64 stage k reads W[k-1]
// and writes W[k mod 4], with W[1] as the accumulator of stages 3 and 4.
__device__ __forceinline__ StageArgs batch_args(const BatchInst &I, int stage, bool mixed) {
  StageArgs a{};
  a.bg = I.bg;
  a.sc = I.sc;
  a.red_in = stage - 1;
  a.red_out = stage;
  a.hdiv = stage == 3 ? 1.0 : stage == 4 ? 6.0 : 2.0;
  a.tfrac = stage == 1 ? 0.0 : stage == 4 ? 1.0 : 0.5;
  if (mixed) {
    a.w32 = I.F[0];
    a.c32 = I.F[1];
    a.acc32 = I.F[4];
    a.in32 = stage == 1 ? I.F[0] : stage == 3 ? I.F[3] : I.F[2];
    a.out32 = stage == 2 ? I.F[3] : stage == 4 ? nullptr : I.F[2];
    a.kind = stage;
  } else {
    a.base = I.W[0];
    a.in = I.W[stage - 1];
    a.out = I.W[stage & 3];
    a.acc = stage >= 3 ? I.W[1] : nullptr;
    a.kind = stage >= 3 ? stage : 0;
  }
  return a;
}

template <int D, typename T, typename S>
__global__ void __launch_bounds__(S::NT, 512 / S::NT)
    batch_stage_kernel(const BatchInst *__restrict__ tab, const WorkItem *__restrict__ work, int nwork, int stage) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ Geo sg;
  __shared__ Phys sp;
  __shared__ int go;
  constexpr bool MIXED = sizeof(T) == sizeof(float);
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const WorkItem it = work ? work[w] : WorkItem{0, w};  // no list: tile w of simulation 0
    const BatchInst &I = tab[it.inst];
    if (threadIdx.x == 0) {
      go = I.active && I.sc->go;
      sg = I.geo;
      sp = I.phys;
    }
    __syncthreads();
    if (go) {
      const StageArgs a = batch_args(I, stage, MIXED);
      const int tx = I.tiles[0], ty = I.tiles[1];
      const int bx = it.tile % tx, by = (it.tile / tx) % ty, bz = it.tile / (tx * ty);
      // private copies: the compiler keeps the fields it uses in registers
      // instead of reloading them from shared memory after every store to the
      // tile buffers
      const Geo g = sg;
      const Phys p = sp;
      tile_body<D, T, S>(a, g, p, bx, by, bz, reinterpret_cast<T *>(smraw));
    }
    __syncthreads();  // sg / sp / go / the tile's shared memory are reused by the next item
  }
}

template <int D, typename T, typename S>
struct BatchLaunch {
  static constexpr int smem = tile_smem_elems<D, S>() * (int)sizeof(T);
  static void set_attr() {
    static bool init[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !init[dev]) {
      cudaFuncSetAttribute(batch_stage_kernel<D, T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (dev >= 0 && dev < 64) init[dev] = true;
    }
  }
  static void run(const BatchInst *tab, const WorkItem *work, int nwork, int stage, int grid, cudaStream_t st) {
    set_attr();
    batch_stage_kernel<D, T, S><<<grid, S::NT, smem, st>>>(tab, work, nwork, stage);
  }
  static int occupancy() {
    set_attr();
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_stage_kernel<D, T, S>, S::NT, smem);
    return n;
  }
};

template <int D, typename T, typename F>
static auto with_shape(int v, F f) {
  if (D == 2) {
    switch (v) {
      case 1: return f(BatchLaunch<D, T, Tile<32, 8, 1>>{});
      case 2: return f(BatchLaunch<D, T, Tile<8, 32, 1>>{});
      case 3: return f(BatchLaunch<D, T, Tile<32, 16, 1>>{});
      default: return f(BatchLaunch<D, T, Tile<16, 16, 1>>{});
    }
  } else {
    switch (v) {
      case 1: return f(BatchLaunch<D, T, Tile<16, 8, 2>>{});
      case 2: return f(BatchLaunch<D, T, Tile<32, 4, 2>>{});
      default: return f(BatchLaunch<D, T, Tile<8, 8, 4>>{});
    }
  }
}

template <typename F>
static auto dispatch(int D, bool mixed, int v, F f) {
  if (D == 2) return mixed ? with_shape<2, float>(v, f) : with_shape<2, double>(v, f);
  return mixed ? with_shape<3, float>(v, f) : with_shape<3, double>(v, f);
}

void launch_batch_stage(int D, bool mixed, int variant, const BatchInst *tab, const WorkItem *work, int nwork,
                        int stage, int grid, cudaStream_t st) {
  if (nwork <= 0 || grid <= 0) return;
  dispatch(D, mixed, variant, [&](auto L) {
    decltype(L)::run(tab, work, nwork, stage, grid, st);
    return 0;
  });
}

int batch_stage_occupancy(int D, bool mixed, int variant) {
  return dispatch(D, mixed, variant, [&](auto L) { return decltype(L)::occupancy(); });
}

}  // namespace smaug_batchk
