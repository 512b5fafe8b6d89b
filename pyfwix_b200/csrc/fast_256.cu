// Register-resident passes for lines of 256 samples: 16 lanes x 16 samples,
// radix stages 16,16 (one shared-memory exchange per transform).  Rows place
// sample p at p + (p >> 4) (their lines have room for it); the columns, whose
// tile lines have no spare room, use the XOR placements (XSw) that
// pyfwix_b200/tune_fft.py picks, conflict-free as well.
#include "fast.cuh"

using FwixRowPlan256 = fwix::fast::Plan<256, 16, fwix::fast::Radices<16, 16>, 1>;
using FwixColPlan256 = fwix::fast::Plan<256, 16, fwix::fast::Radices<16, 16>, 0, fwix::fast::XSw<fwix::fast::xs(4, 1, 15), fwix::fast::xs(4, 1, 15)>>;
FWIX_FAST_INSTANTIATE2(FwixRowPlan256, FwixColPlan256, 256)
