// Register-resident passes for lines of 192 samples: 16 lanes x 12 samples,
// radix stages 4,4,4,3.
// The exchange placements (XSw) are the ones with the fewest shared-memory
// bank conflicts for this plan's strides, per exchange.
#include "fast.cuh"

using FwixPlan192 = fwix::fast::Plan<192, 12, fwix::fast::Radices<4,4,4,3>, 0,
                                        fwix::fast::XSw<fwix::fast::xs(2, 1, 15), fwix::fast::xs(2, 1, 15), -1, 0, 0, -1>>;
FWIX_FAST_INSTANTIATE(FwixPlan192, 192)
