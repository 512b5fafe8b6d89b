// Register-resident passes for lines of 128 samples: 16 lanes x 8 samples,
// radix stages 8,4,4.
// The exchange placements (XSw) are the ones with the fewest shared-memory
// bank conflicts for this plan's strides, per exchange (pyfwix_b200/tune_fft.py).
#include "fast.cuh"

using FwixPlan128 = fwix::fast::Plan<128, 8, fwix::fast::Radices<8,4,4>, 0,
                                        fwix::fast::XSw<-1, fwix::fast::xs(2, 1, 15), fwix::fast::xs(2, 1, 15), fwix::fast::xs(2, 1, 15)>>;
FWIX_FAST_INSTANTIATE(FwixPlan128, 128)
