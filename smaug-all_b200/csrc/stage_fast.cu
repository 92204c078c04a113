// Production stage kernels: the shared-memory tiled kernel, built with FMA
// contraction.
#define SMAUG_NS smaug_fast
#define SMAUG_TILED 1
#include "stage_variant.inc"
