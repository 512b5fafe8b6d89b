// Register-resident passes for lines of 384 samples: 32 lanes x 12 samples,
// radix stages 12, 4, 4, 2 (the radix-12 butterfly is a prime-factor 4 x 3
// transform, so the first stage needs no twiddles and the line is exchanged
// through shared memory once less than with radix-4 stages throughout).
// The exchange placements (XSw) are the ones with the fewest shared-memory
// bank conflicts for this plan's strides, per exchange (pyfwix_b200/tune_fft.py).
#include "fast.cuh"

using FwixPlan384 = fwix::fast::Plan<384, 12, fwix::fast::Radices<12, 4, 4, 2>, 0,
    fwix::fast::XSw<fwix::fast::xs(2, 1, 15), -1, -1, fwix::fast::xs(1, 1, 15), -1, fwix::fast::xs(2, 1, 15)>>;
FWIX_FAST_INSTANTIATE(FwixPlan384, 384)
