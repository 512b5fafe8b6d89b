// Register-resident passes for lines of 640 samples: 32 lanes x 20 samples,
// radix stages 4,4,4,2,5.
#include "fast.cuh"

using FwixPlan640 = fwix::fast::Plan<640, 20, fwix::fast::Radices<4,4,4,2,5>>;
FWIX_FAST_INSTANTIATE(FwixPlan640, 640)
