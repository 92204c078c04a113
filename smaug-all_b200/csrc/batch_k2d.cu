// Stage kernels of the batch for ndim 2, double stencils (batch_kernels.inc).
#define BATCH_D 2
#define BATCH_T double
#define BATCH_SUFFIX d
#include "batch_kernels.inc"
