// Register-resident passes for lines of 256 samples: 32 lanes x 8 samples,
// radix stages 8,8,4.
#include "fast.cuh"

using FwixPlan256 = fwix::fast::Plan<256, 8, fwix::fast::Radices<8,8,4>>;
FWIX_FAST_INSTANTIATE(FwixPlan256, 256)
