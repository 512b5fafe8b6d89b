// Register-resident passes for lines of 320 samples: 16 lanes x 20 samples,
// radix stages 20, 4, 4 (the radix-20 butterfly is a prime-factor 4 x 5
// transform, so the first stage needs no twiddles and the line is exchanged
// through shared memory once less than with radix-4 stages throughout).
// The exchange placements (XSw) are the ones with the fewest shared-memory
// bank conflicts for this plan's strides, per exchange (pyfwix_b200/tune_fft.py).
#include "fast.cuh"

using FwixPlan320 = fwix::fast::Plan<320, 20, fwix::fast::Radices<20, 4, 4>, 0,
    fwix::fast::XSw<fwix::fast::xs(2, 1, 15), fwix::fast::xs(4, 7, 7), fwix::fast::xs(2, 1, 15), fwix::fast::xs(2, 1, 15)>>;
FWIX_FAST_INSTANTIATE(FwixPlan320, 320)
