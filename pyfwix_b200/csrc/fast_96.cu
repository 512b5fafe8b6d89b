// Register-resident passes for lines of 96 samples: 8 lanes x 12 samples,
// radix stages 4,4,2,3.
#include "fast.cuh"

using FwixPlan96 = fwix::fast::Plan<96, 12, fwix::fast::Radices<4,4,2,3>>;
FWIX_FAST_INSTANTIATE(FwixPlan96, 96)
