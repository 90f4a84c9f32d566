// Gather-rate calibration of the device (calibrate.cu).
#pragma once

#include "common.cuh"

namespace knb {

// Random 4-byte gathers per second over the whole GPU: source 0 from a
// device array of `words` FP32 values, 1 from each SM's own shared memory,
// 2, 4 or 8 from the shared memory of a cluster of that many CTAs. Throws
// knb::Error for other sources or array sizes outside [1024, 2^31].
double measure_gather_rate(int source, uint64_t words, cudaStream_t s);

}  // namespace knb
