// Register-resident passes for lines of 320 samples: 16 lanes x 20 samples,
// radix stages 4,4,4,5.
#include "fast.cuh"

using FwixPlan320 = fwix::fast::Plan<320, 20, fwix::fast::Radices<4,4,4,5>>;
FWIX_FAST_INSTANTIATE(FwixPlan320, 320)
