// Stage kernels built with FMA contraction (the production FP64 variant).
#define SMAUG_NS smaug_fast
#include "stage_variant.inc"
