// Register-resident passes for lines of 640 samples: 32 lanes x 20 samples,
// radix stages 4,4,4,2,5.
// The exchange placements (XSw) are the ones with the fewest shared-memory
// bank conflicts for this plan's strides, per exchange.
#include "fast.cuh"

using FwixPlan640 = fwix::fast::Plan<640, 20, fwix::fast::Radices<4,4,4,2,5>, 0,
                                        fwix::fast::XSw<fwix::fast::xs(2, 1, 15), fwix::fast::xs(2, 1, 15), -1, -1, 0, 0, fwix::fast::xs(5, 7, 15), fwix::fast::xs(4, 15, 15)>>;
FWIX_FAST_INSTANTIATE(FwixPlan640, 640)
