// Stage kernels of the batch for ndim 3, float stencils (batch_kernels.inc).
#define BATCH_D 3
#define BATCH_T float
#define BATCH_SUFFIX f
#include "batch_kernels.inc"
