// Register-resident passes for lines of 96 samples: 8 lanes x 12 samples,
// radix stages 4,4,2,3.
// The exchange placements (XSw) are the ones with the fewest shared-memory
// bank conflicts for this plan's strides, per exchange.
#include "fast.cuh"

using FwixPlan96 = fwix::fast::Plan<96, 12, fwix::fast::Radices<4,4,2,3>, 0,
                                        fwix::fast::XSw<-1, fwix::fast::xs(2, 1, 7), -1, 0, fwix::fast::xs(1, 1, 7), fwix::fast::xs(3, 5, 7)>>;
FWIX_FAST_INSTANTIATE(FwixPlan96, 96)
