// Katz and Bonacich power centrality on the device: the attenuated series
// x = b + t A x (reference: crates/engine/src/metrics/spectral.rs:300-672).
#pragma once

#include <vector>

#include "graph.cuh"

namespace knb {

struct SeriesParams {
  int mode = 2;        // 1 out, 2 in, 3 all
  bool weighted = false;
  int loops = 1;       // 0 twice, 1 once, 2 ignore
  double tol = 1e-12;
  int64_t max_iter = 10000;
};

struct SeriesResult {
  int64_t iterations = 0;  // sweeps of the series
  int64_t collatz = 0;     // power-iteration steps of the attenuation check
  double radius = 0;       // the spectral-radius bound the check returned
  bool dense = false;      // Bonacich: solved by dense elimination
  double seconds = 0;
  int kernel_launches = 0;
};

// Katz centrality x = alpha A x + beta (spectral.rs:365-407); beta holds 1
// or n values. Writes n scores to host `out`. Throws knb::Error.
void katz(GraphHandleImpl& g, double alpha, const std::vector<double>& beta, bool normalized,
          const SeriesParams& p, double* out, SeriesResult* r, cudaStream_t s);

// Bonacich power centrality (spectral.rs:596-655): (I - exponent A)^-1 A 1,
// scaled so the squares sum to n, or (rescale) so the scores sum to 1.
void bonacich_power(GraphHandleImpl& g, double exponent, bool rescale, const SeriesParams& p,
                    double* out, SeriesResult* r, cudaStream_t s);

}  // namespace knb
