// Register-resident passes for lines of 384 samples: 32 lanes x 12 samples,
// radix stages 4,4,4,2,3.
#include "fast.cuh"

using FwixPlan384 = fwix::fast::Plan<384, 12, fwix::fast::Radices<4,4,4,2,3>>;
FWIX_FAST_INSTANTIATE(FwixPlan384, 384)
