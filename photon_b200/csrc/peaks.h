// Bandwidth probes for the roofline denominators that the measured-peaks file does not cover.
#pragma once

#include <cstddef>

namespace ptw {

// Read bandwidth of an L2-resident buffer of `bytes` bytes (loads that bypass L1), read `reps`
// times per launch; best of five launches after a warm-up. Throws Error.
double measure_l2_read_gbs(int device, size_t bytes, int reps);

}  // namespace ptw
