// Register-resident passes for lines of 384 samples: 32 lanes x 12 samples,
// radix stages 4,4,4,2,3.
// The exchange placements (XSw) are the ones with the fewest shared-memory
// bank conflicts for this plan's strides, per exchange.
#include "fast.cuh"

using FwixPlan384 = fwix::fast::Plan<384, 12, fwix::fast::Radices<4,4,4,2,3>, 0,
                                        fwix::fast::XSw<fwix::fast::xs(2, 1, 15), fwix::fast::xs(2, 1, 15), -1, -1, 0, 0, fwix::fast::xs(3, 1, 7), -1>>;
FWIX_FAST_INSTANTIATE(FwixPlan384, 384)
