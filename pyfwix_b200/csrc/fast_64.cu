// Register-resident passes for lines of 64 samples: 8 lanes x 8 samples,
// radix stages 8,8.
#include "fast.cuh"

using FwixPlan64 = fwix::fast::Plan<64, 8, fwix::fast::Radices<8,8>>;
FWIX_FAST_INSTANTIATE(FwixPlan64, 64)
