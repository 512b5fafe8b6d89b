// Register-resident passes for lines of 160 samples: 8 lanes x 20 samples,
// radix stages 4,4,2,5.
// The exchange placements (XSw) are the ones with the fewest shared-memory
// bank conflicts for this plan's strides, per exchange.
#include "fast.cuh"

using FwixPlan160 = fwix::fast::Plan<160, 20, fwix::fast::Radices<4,4,2,5>, 0,
                                        fwix::fast::XSw<-1, fwix::fast::xs(2, 1, 7), -1, 0, fwix::fast::xs(3, 5, 7), fwix::fast::xs(5, 7, 15)>>;
FWIX_FAST_INSTANTIATE(FwixPlan160, 160)
