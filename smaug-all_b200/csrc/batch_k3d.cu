// Stage kernels of the batch for ndim 3, double stencils (batch_kernels.inc).
#define BATCH_D 3
#define BATCH_T double
#define BATCH_SUFFIX d
#include "batch_kernels.inc"
