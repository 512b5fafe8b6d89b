// Register-resident passes for lines of 512 samples: 32 lanes x 16 samples,
// radix stages 8,8,8.
#include "fast.cuh"

using FwixPlan512 = fwix::fast::Plan<512, 16, fwix::fast::Radices<8,8,8>>;
FWIX_FAST_INSTANTIATE(FwixPlan512, 512)
