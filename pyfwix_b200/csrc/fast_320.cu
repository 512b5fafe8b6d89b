// Register-resident passes for lines of 320 samples: 16 lanes x 20 samples,
// radix stages 4,4,4,5.
// The exchange placements (XSw) are the ones with the fewest shared-memory
// bank conflicts for this plan's strides, per exchange.
#include "fast.cuh"

using FwixPlan320 = fwix::fast::Plan<320, 20, fwix::fast::Radices<4,4,4,5>, 0,
                                        fwix::fast::XSw<fwix::fast::xs(2, 1, 15), fwix::fast::xs(2, 1, 15), -1, 0, 0, fwix::fast::xs(4, 7, 7)>>;
FWIX_FAST_INSTANTIATE(FwixPlan320, 320)
