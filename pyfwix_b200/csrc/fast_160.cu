// Register-resident passes for lines of 160 samples: 8 lanes x 20 samples,
// radix stages 4,4,2,5.
#include "fast.cuh"

using FwixPlan160 = fwix::fast::Plan<160, 20, fwix::fast::Radices<4,4,2,5>>;
FWIX_FAST_INSTANTIATE(FwixPlan160, 160)
