// PageRank on the device: options, results and the solver entry points.
#pragma once

#include "graph.cuh"

namespace knb {

enum Precision : int32_t {
  PREC_FP64 = 0,   // every sweep in FP64 (arc values FP64 unless exact in FP32)
  PREC_MIXED = 1,  // FP32 sweeps, then FP64-accurate sweeps on the same trajectory
  PREC_FP32 = 2,   // FP32 sweeps only (no FP64 refinement; diagnostics)
};

struct PagerankParams {
  double damping = 0.85;
  bool directed = true;
  bool weighted = false;
  const double* personalization = nullptr;  // host, n values, or null (uniform)
  bool pers_on_device = false;              // personalization is a device pointer
  int dangling = 0;                         // 0 personalized, 1 uniform
  int loops = 0;                            // 0 twice, 1 once, 2 ignore
  double tol = 1e-12;
  int64_t max_iter = 10000;
  int precision = PREC_FP64;
  int ipt = 0;                  // merge-path items per thread (0: tuned)
  int variant = 0;              // sweep kernel: 1 CTA tiles, 2 warp tiles (0: tuned)
  double switch_factor = 8192;  // mixed: leave FP32 once change <= tol * factor
  double switch_floor = 2e-6;   //        ... or once change <= this floor
  bool fp64_values = false;     // FP64 sweeps read FP64 values even if FP32 is exact
  bool relabel = true;          // sweep on the operator renumbered by column count
};

struct PagerankInfo {
  int64_t iterations = 0;       // sweeps in total (the trajectory length)
  int64_t iterations_fp32 = 0;  // of which FP32
  double change = 0;            // L1 change of the last sweep
  double seconds = 0;           // device time of the solve (events)
  int32_t converged = 0;
  int32_t kernel_launches = 0;  // kernels launched by the solve
  int32_t sweep_kernel = 0;     // the FP32-phase (or FP64) sweep kernel, tuning key 4 codes
  int32_t long_row = 0;         // sliced sweeps: the long-row threshold
  int32_t hot_columns = 0;      // FP32 values of the most gathered columns kept in L1
};

// Process-wide tuning knobs (set through net_set_tuning); 0 leaves a
// parameter to the library's choice.
struct Tuning {
  int ipt = 0;            // merge-path items per thread: 4, 8 or 16
  int relabel = 1;        // 1: sweep on the operator renumbered by column count
  int variant = 0;        // sweep kernel: 1 CTA tiles, 2-5 warp tiles (see pagerank.cu)
  int carveout = -1;      // preferred shared-memory carveout percent (-1: what the resident CTAs need)
  int64_t hot_nodes = -1; // hot-node sweeps: cap on the nodes kept in shared memory (-1: none)
  int persistent = 1;     // warp-tile sweeps: 1 launches only the CTAs that fit at once
  int refine = 1;         // mixed: 1 anchor + refinement sweeps, 0 plain FP64 sweeps
  int long_row = 0;       // sliced sweeps: rows of at least this many arcs are long (0: 255)
  int64_t smem_hot = -1;  // sliced sweeps with a shared-memory tier: FP32 values kept there (-1: 32768)
  int autotune = 1;       // 1: pick the sweep kernel per operator by timing candidates (large operators)
  int bulk_ctas = 0;      // bulk-staged sliced sweeps: CTAs per SM the carveout is sized for (0: 4)
  int64_t bulk_skip_chunk = -1;  // test of the bounded waits: a chunk of the first warp never copied
  int64_t small_edges = 1 << 18;  // FP64 solves (host teleport vector, if any) on at most
                                  // this many edges run as one packed-graph launch (0: never)
  double switch_factor = 8192;
  double switch_floor = 2e-6;
};
Tuning& tuning();

// Runs PageRank on handle `g`; writes n FP64 scores to `out` (host pointer
// unless out_on_device). Throws knb::Error on failure (non-convergence too).
void pagerank(GraphHandleImpl& g, const PagerankParams& prm, double* out, bool out_on_device,
              PagerankInfo* info, cudaStream_t s);
// The same on a given pull operator (rows = arcs into a node).
void pagerank_op(Operator& op, const PagerankParams& prm, double* out, bool out_on_device,
                 PagerankInfo* info, cudaStream_t s);
// Which rows PageRank pulls along (1 in-CSR, 2 directions ignored, 0 the
// undirected CSR) and the diagonal factor of a self-loop in them.
int pagerank_rows(const GraphHandleImpl& g, bool directed);
// Checks a device personalization vector of n values (finite, nonnegative,
// positive sum) and rescales it to sum 1 in place, as the reference's
// `probabilities` (crates/engine/src/metrics/spectral.rs:284-305).
void normalize_personalization_device(double* p, uint32_t n, cudaStream_t s);
double pagerank_loop_factor(int which, int loops);

// Device time of the dominant kernel (the merge-path sweep) of the last solve
// on this thread: launches and total milliseconds, measured with events.
struct SweepTiming {
  int64_t launches = 0;
  double ms = 0;
  double bytes_per_launch = 0;  // algorithmic bytes of one sweep
};
// phase 0: FP32 sweeps, 1: FP64 sweeps (the anchor sweep in mixed solves
// with refinement), 2: refinement sweeps
SweepTiming last_sweep_timing(int phase);
void set_sweep_timing(bool on);

}  // namespace knb
