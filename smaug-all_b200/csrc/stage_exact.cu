// Stage kernels built with -fmad=false: every multiply and add rounds
// separately, as in the oracle and the reference host build, so results are
// bit-reproducible against them.
#define SMAUG_NS smaug_exact
#include "stage_variant.inc"
