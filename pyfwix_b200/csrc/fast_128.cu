// Register-resident passes for lines of 128 samples: 16 lanes x 8 samples,
// radix stages 8,4,4.
#include "fast.cuh"

using FwixPlan128 = fwix::fast::Plan<128, 8, fwix::fast::Radices<8,4,4>>;
FWIX_FAST_INSTANTIATE(FwixPlan128, 128)
