// Synthetic R-MAT graphs and lognormal strengths on the device.
#pragma once

#include "graph.cuh"

namespace knb {

struct RmatEdges {
  uint32_t n = 0;
  uint64_t m = 0;
  DevBuf<uint32_t> src, tgt;
  DevBuf<float> w32;  // lognormal strengths, when requested
};

RmatEdges generate_rmat(int scale, uint64_t edge_factor, double a, double b, double c,
                        uint64_t seed, bool clean, bool symmetrize, bool lognormal, uint64_t wseed,
                        cudaStream_t s);

}  // namespace knb
