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

// Host G(n, m) (crates/engine/src/generate.rs:255-290) with node offset.
void gnm_edges(uint64_t n, uint64_t m, bool directed, bool loops, uint64_t seed, uint64_t rep,
               int64_t offset, int64_t* src, int64_t* tgt);
void gnm_batch(uint64_t count, const int64_t* n, const int64_t* m, bool directed, bool loops,
               uint64_t seed, int64_t* src, int64_t* tgt, int threads);
void power_law_sizes(uint64_t count, double alpha, double lo, double hi, uint64_t seed,
                     int64_t* out);

}  // namespace knb
