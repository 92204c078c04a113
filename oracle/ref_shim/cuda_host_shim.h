/*
 * cuda_host_shim.h -- test infrastructure, NOT product code.
 *
 * Lets the SMAUG reference's own CUDA C sources (dev/smaug/src/*.cu) compile
 * and run on the host, so that the reference itself can serve as the parity
 * pin for the oracle and the GPU path.  Every reference kernel on the hot path
 * is "one thread per cell, each thread writes only its own cell" (see e.g.
 * dev/smaug/src/centdiff1.cu:261-553), so running the launch grid serially,
 * block by block and thread by thread, reproduces the launch exactly.  The
 * shared-memory max reductions are the exception; build_ref.py replaces their
 * launches by shim_blockmax() below, which returns the same block maxima.
 *
 * This header is force-included (g++ -include) into every translation unit of
 * the host build made by oracle/ref_shim/build_ref.py.  It maps the CUDA
 * keywords and the handful of runtime calls the reference uses onto plain C.
 */
#ifndef SMAUG_CUDA_HOST_SHIM_H
#define SMAUG_CUDA_HOST_SHIM_H

#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <math.h>

#define __global__
#define __device__
#define __host__
#define __shared__ static
#define __forceinline__ inline

struct shim_uint3 {
  unsigned int x, y, z;
};
struct dim3 {
  unsigned int x, y, z;
  dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};

/* The launch loop sets these before each emulated thread runs. */
extern shim_uint3 blockIdx, threadIdx, blockDim, gridDim;

static inline void __syncthreads(void) {}

typedef int cudaError_t;
enum { cudaSuccess = 0 };
enum cudaMemcpyKind {
  cudaMemcpyHostToHost = 0,
  cudaMemcpyHostToDevice = 1,
  cudaMemcpyDeviceToHost = 2,
  cudaMemcpyDeviceToDevice = 3
};
struct cudaDeviceProp {
  char name[256];
  int major, minor;
};

/* Device memory is host memory; calloc so a fresh buffer reads as zeros. */
static inline cudaError_t cudaMalloc(void **p, size_t n) {
  *p = calloc(n ? n : 1, 1);
  return *p ? cudaSuccess : 2;
}
static inline cudaError_t cudaFree(void *p) {
  free(p);
  return cudaSuccess;
}
static inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, int kind) {
  (void)kind;
  if (n && d != s) memmove(d, s, n);
  return cudaSuccess;
}
static inline cudaError_t cudaThreadSynchronize(void) { return cudaSuccess; }
static inline cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
static inline cudaError_t cudaGetLastError(void) { return cudaSuccess; }
static inline const char *cudaGetErrorString(cudaError_t e) {
  (void)e;
  return "no error (host shim)";
}
static inline cudaError_t cudaSetDevice(int d) {
  (void)d;
  return cudaSuccess;
}
static inline cudaError_t cudaGetDeviceCount(int *n) {
  *n = 1;
  return cudaSuccess;
}
static inline cudaError_t cudaGetDeviceProperties(cudaDeviceProp *p, int d) {
  (void)d;
  strcpy(p->name, "host-shim");
  p->major = 1;
  p->minor = 0;
  return cudaSuccess;
}

/* Serial emulation of kernel<<<nb, nt>>>(args). */
#define SHIM_LAUNCH(NB, NT, CALL)                                              \
  do {                                                                         \
    unsigned int shim_nb_ = (unsigned int)(NB), shim_nt_ = (unsigned int)(NT); \
    gridDim.x = shim_nb_; gridDim.y = 1; gridDim.z = 1;                        \
    blockDim.x = shim_nt_; blockDim.y = 1; blockDim.z = 1;                     \
    for (unsigned int shim_b_ = 0; shim_b_ < shim_nb_; ++shim_b_)              \
      for (unsigned int shim_t_ = 0; shim_t_ < shim_nt_; ++shim_t_) {          \
        blockIdx.x = shim_b_; blockIdx.y = 0; blockIdx.z = 0;                  \
        threadIdx.x = shim_t_; threadIdx.y = 0; threadIdx.z = 0;               \
        CALL;                                                                  \
      }                                                                        \
  } while (0)

/*
 * Replacement for the four interleaved shared-memory max reductions
 * (computedervfields.cu:1054-1086, hyperdifvisc1r.cu:227-257,
 *  hyperdifvisc1l.cu:234-264, nushk1.cu:76-106).  Each block b of NT threads
 * reduces temp[b*NT .. b*NT+NT) restricted to indices < ndimp, starting from
 * 0.0, and stores the maximum in out[b]; when write_temp is set the block
 * maximum is also written to temp[b] (what the nushk1.cu variant does).  Max
 * is exact, so the serial order gives the same result as the tree.
 */
static inline void shim_blockmax(int nb, int nt, double *out, double *temp, int ndimp,
                                 int write_temp) {
  for (int b = 0; b < nb; ++b) {
    double m = 0.0;
    for (int t = 0; t < nt; ++t) {
      long idx = (long)b * nt + t;
      double v = (idx < ndimp) ? temp[idx] : 0.0;
      if (v > m) m = v;
    }
    out[b] = m;
  }
  if (write_temp)
    for (int b = 0; b < nb; ++b) temp[b] = out[b];
}

#endif
