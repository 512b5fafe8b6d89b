// Register-resident passes for lines of 192 samples: 16 lanes x 12 samples,
// radix stages 4,4,4,3.
#include "fast.cuh"

using FwixPlan192 = fwix::fast::Plan<192, 12, fwix::fast::Radices<4,4,4,3>>;
FWIX_FAST_INSTANTIATE(FwixPlan192, 192)
