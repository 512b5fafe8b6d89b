// Register-resident passes for lines of 256 samples.  Rows: 16 lanes x 16
// samples, radix stages 16,16 (one shared-memory exchange per transform).
// Columns: 32 lanes x 8 samples, radix stages 8,8,4 (fewer registers per lane,
// which the column passes need for their per-term spectra); their exchange
// placements (XSw) are the ones pyfwix_b200/tune_fft.py picks.
#include "fast.cuh"

using FwixRowPlan256 = fwix::fast::Plan<256, 16, fwix::fast::Radices<16, 16>, 1>;
using FwixColPlan256 = fwix::fast::Plan<256, 8, fwix::fast::Radices<8, 8, 4>, 0, fwix::fast::XSw<-1, -1, fwix::fast::xs(2, 1, 15), -1>>;
FWIX_FAST_INSTANTIATE2(FwixRowPlan256, FwixColPlan256, 256)
