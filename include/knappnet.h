/*
 * C interface of the knappnet B200 library: the reference engine's
 * spectral-centrality entry points (graph build, degree, PageRank,
 * eigenvector centrality and the measures built on the same products),
 * computed on an NVIDIA B200 (sm_100a), plus additive extensions. The
 * reference entry points keep the signatures and codes of
 * crates/capi/include/netcapi.h, so a program built against that header
 * links against this library unchanged.
 *
 * How every function behaves:
 * - A function with an `err` buffer returns 0 when it succeeds. On failure
 *   it returns a non-zero status and leaves a message in `err`, cut to
 *   `err_len` bytes and NUL-terminated. Count accessors answer -1 when
 *   given a NULL handle.
 * - Nodes are numbered from 0. The caller owns every output buffer; a
 *   per-node result needs room for n doubles.
 * - The caller owns a handle until it passes it to net_graph_free (NULL is
 *   ignored there). A handle never changes after it is built, so threads
 *   may share it.
 * - Codes: mode 1 follows arcs out of a node, 2 into it, 3 both ways;
 *   loops 0 counts an undirected self-loop twice (as igraph), 1 once (as
 *   NetworkX), 2 not at all; dangling 0 sends the mass of nodes without
 *   out-arcs along the personalization vector, 1 spreads it uniformly;
 *   scale 0 makes the largest score 1, 1 gives unit Euclidean length. A
 *   tolerance or iteration cap that is not positive means the default
 *   (1e-12, 10000). `threads` is accepted and ignored: no result depends
 *   on it.
 * - A graph is stored in the memory of the CUDA device that is current
 *   when it is built. Functions named `_device` take device pointers.
 */
#ifndef KNAPPNET_H
#define KNAPPNET_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define NET_API __attribute__((visibility("default")))
#else
#define NET_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct GraphHandle GraphHandle;

/* ---- Reference entry points ------------------------------------------- */

/* Makes a handle for a graph of n nodes and m edges src[k] -> tgt[k], with
 * one weight per edge or none (weights NULL). With directed == 0 every edge
 * is stored both ways. Replaces netcapi.h:46-48 (crates/capi/src/lib.rs:139-164). */
NET_API int32_t net_graph_new(int64_t n, const int64_t *src, const int64_t *tgt,
                      const double *weights, int64_t m, int32_t directed,
                      GraphHandle **out, char *err, size_t err_len);

/* Frees a handle and the device memory behind it; NULL does nothing.
 * Replaces netcapi.h:51 (lib.rs:171-175). */
NET_API void net_graph_free(GraphHandle *h);

/* n of the handle; -1 when h is NULL. Replaces netcapi.h:54 (lib.rs:182-184). */
NET_API int64_t net_graph_node_count(const GraphHandle *h);

/* m as given to net_graph_new, repeated edges and self-loops included; -1
 * when h is NULL. Replaces netcapi.h:57. */
NET_API int64_t net_graph_edge_count(const GraphHandle *h);

/* Per-node count of the arcs that mode selects, or the sum of their
 * weights when weighted != 0; n doubles to out. Replaces
 * netcapi.h:383-384 (lib.rs:192-212). */
NET_API int32_t net_degree(const GraphHandle *h, int32_t mode, int32_t loops,
                   int32_t weighted, double *out, char *err, size_t err_len);

/* Stationary distribution of the damped random walk: n scores adding up
 * to 1 go to out. The teleport vector is uniform when personalization is
 * NULL, else n values that must not be negative (rescaled to sum 1). With
 * directed == 0 each arc is walked both ways.
 * Replaces netcapi.h:463-467 (crates/capi/src/spectral.rs:59-97). */
NET_API int32_t net_pagerank(const GraphHandle *h, double damping, int32_t directed,
                     int32_t weighted, const double *personalization,
                     int32_t dangling, int32_t loops, double tol,
                     int64_t max_iter, int32_t threads, double *out,
                     char *err, size_t err_len);

/* Katz scores: the solution x of x = alpha A' x + beta, with beta one value
 * shared by all nodes or one per node. The call fails when alpha reaches
 * 1 / lambda_max, where the series no longer converges; normalized != 0
 * rescales x to Euclidean length 1. Replaces netcapi.h:472-476
 * (crates/capi/src/spectral.rs:107-140). */
NET_API int32_t net_katz(const GraphHandle *h, double alpha, const double *beta,
                         int64_t beta_len, int32_t mode, int32_t weighted, int32_t loops,
                         int32_t normalized, double tol, int64_t max_iter, int32_t threads,
                         double *out, char *err, size_t err_len);

/* Bonacich's power centrality c = (I - exponent A)^-1 A 1, rescaled to a sum
 * of squares n, or to a sum of 1 when rescale != 0. When the series would
 * not converge (|exponent| lambda_max >= 1) the system is solved densely,
 * for at most 5,000 nodes; a singular system fails the call.
 * Replaces netcapi.h:481-486 (crates/capi/src/spectral.rs:149-179). */
NET_API int32_t net_bonacich_power(const GraphHandle *h, double exponent, int32_t mode,
                                   int32_t weighted, int32_t loops, int32_t rescale,
                                   double tol, int64_t max_iter, int32_t threads,
                                   double *out, char *err, size_t err_len);

/* Kleinberg's hubs and authorities: n hub scores and n authority scores.
 * *value gets the leading eigenvalue of A^T A and *unique is 1 when the top
 * singular value has multiplicity one; scale 0 makes the largest score 1,
 * 1 the sum 1, 2 the Euclidean length 1. Replaces netcapi.h:489-493
 * (crates/capi/src/spectral.rs:189-230). */
NET_API int32_t net_hits(const GraphHandle *h, int32_t weighted, int32_t loops, int32_t scale,
                         double tol, int64_t max_iter, int32_t threads, double *hubs,
                         double *authorities, double *value, int32_t *unique, char *err,
                         size_t err_len);

/* The leading eigenvector of the adjacency matrix in the direction mode
 * picks, as n scores; *eigenvalue gets its eigenvalue and *connected is 1
 * when the graph is connected (strongly, for directed graphs).
 * Replaces netcapi.h:455-459 (crates/capi/src/topography.rs:208-249). */
NET_API int32_t net_eigenvector(const GraphHandle *h, int32_t mode, int32_t weighted,
                        int32_t scale, int32_t loops, double tol,
                        int64_t max_iter, int32_t threads, double *out,
                        double *eigenvalue, int32_t *connected, char *err,
                        size_t err_len);

/* The graph as sna and UCINET read it, an adjacency matrix: one edge per
 * pair of nodes, carrying the largest weight of its parallel edges (keep 0)
 * or the smallest (keep 1), and no self-loops; undirected != 0 also merges
 * the two directions of a directed graph. The new handle lists its edges in
 * (from, to) order; free it with net_graph_free.
 * Replaces netcapi.h:59-65 (crates/capi/src/topography.rs:42-56). */
NET_API int32_t net_graph_simplify(const GraphHandle *h, int32_t undirected, int32_t keep,
                                   GraphHandle **out, char *err, size_t err_len);

/* Eigenvector centrality of a two-mode network: the leading singular
 * vectors of the binary incidence matrix, each mode scaled to Euclidean
 * length 1 (NaN for every node when there are no ties). types holds n codes
 * (0 first mode, 1 second); tol <= 0 and max_iter <= 0 select 1e-12 and
 * 10000. *eigenvalue receives the largest singular value, *connected 1 if
 * the network is connected. Replaces netcapi.h:762-771
 * (crates/capi/src/twomode.rs:293-320). */
NET_API int32_t net_twomode_eigenvector(const GraphHandle *h, const int32_t *types, double tol,
                                        int64_t max_iter, int32_t threads, double *out,
                                        double *eigenvalue, int32_t *connected, char *err,
                                        size_t err_len);

/* Newman's leading eigenvector communities of an undirected network with
 * at most 3000 nodes: 0-based labels (by first appearance) to
 * membership[0..n), the modularity on the input network to *q (NaN without
 * edges), the number of divisions to *splits. Weights (weighted != 0) must
 * be non-negative. Replaces netcapi.h:978-984 (crates/capi/src/groups.rs:334-356). */
NET_API int32_t net_leading_eigen(const GraphHandle *h, int32_t weighted, int64_t *membership,
                                  double *q, int64_t *splits, char *err, size_t err_len);

/* Component of every node, weak (kind 0) or strong (kind 1), as n labels in
 * membership; labels count up from 0 in the order of each component's
 * smallest node, and *count gets the number of components. An undirected
 * graph's strong components are its weak ones.
 * Replaces netcapi.h:517-520 (crates/capi/src/topography.rs:85-106). */
NET_API int32_t net_components(const GraphHandle *h, int32_t kind, int32_t *membership,
                               int64_t *count, char *err, size_t err_len);

/* Freeman centralization, one double to out. This library provides the
 * eigenvector measure (measure 3; igraph convention 0, direction ignored):
 * n max(c) - sum(c) over the unweighted eigenvector centrality c scaled
 * to max 1, divided by n - 2 when normalized (NaN below 3 nodes). The
 * other measures (0 degree, 1 betweenness, 2 closeness) fail with a
 * message. Replaces netcapi.h:534-539 (crates/capi/src/topography.rs:134-159). */
NET_API int32_t net_centralization(const GraphHandle *h, int32_t measure, int32_t mode,
                                   int32_t loops, int32_t normalized, int32_t convention,
                                   int32_t threads, double *out, char *err, size_t err_len);

/* ---- Extensions (no counterpart in the reference) ---------------------- */

/* What a solve did. */
typedef struct NetSolveInfo {
  int64_t iterations;      /* sweeps (PageRank) or matrix-vector products */
  int64_t iterations_fp32; /* of which in FP32 */
  double change;           /* last L1 change (PageRank) / residual (eigen) */
  double seconds;          /* device time of the solve */
  int32_t converged;
  int32_t kernel_launches; /* CUDA kernels the solve launched */
  double eigenvalue;
  int32_t connected;
  int32_t sweep_kernel;    /* PageRank: the sweep kernel used (net_set_tuning key 4 codes);
                              packed graphs: threads per CTA of the launch */
  int32_t long_row;        /* sliced sweeps: rows of at least this many arcs are long;
                              packed graphs: how many times the operator's launch graph
                              has been instantiated (a repeated batch replays it) */
  int32_t hot_columns;     /* FP32 values of the most gathered columns kept in L1;
                              packed graphs: CTAs per thread-block cluster that split
                              each large graph (1: no graph split; iterations_fp32
                              then counts the graphs split) */
} NetSolveInfo;

/* Precision codes: 0 = FP64, 1 = mixed (FP32 sweeps, then on the same
 * trajectory one FP64 anchor sweep and refinement sweeps that gather the
 * FP32 correction, or plain FP64 sweeps with tuning key 9 at 0, until the
 * reference's stopping rule holds in FP64), 2 = FP32 only. */
NET_API int32_t net_pagerank_ex(const GraphHandle *h, double damping, int32_t directed,
                        int32_t weighted, const double *personalization,
                        int32_t dangling, int32_t loops, double tol,
                        int64_t max_iter, int32_t precision, double *out,
                        NetSolveInfo *info, char *err, size_t err_len);

/* As net_pagerank_ex with device pointers for personalization and out. */
NET_API int32_t net_pagerank_device(const GraphHandle *h, double damping,
                            int32_t directed, int32_t weighted,
                            const double *d_personalization, int32_t dangling,
                            int32_t loops, double tol, int64_t max_iter,
                            int32_t precision, double *d_out,
                            NetSolveInfo *info, char *err, size_t err_len);

/* As net_eigenvector, with a precision code (0 = FP64, 1 = FP32
 * matrix-vector products with FP64 basis, dots and reorthogonalisation)
 * and the solve information. */
NET_API int32_t net_eigenvector_ex(const GraphHandle *h, int32_t mode, int32_t weighted,
                           int32_t scale, int32_t loops, double tol,
                           int64_t max_iter, int32_t precision, double *out,
                           double *eigenvalue, int32_t *connected,
                           NetSolveInfo *info, char *err, size_t err_len);

/* What a batched solve did. */
typedef struct NetBatchInfo {
  double seconds;                /* device time of the solve */
  int64_t sweeps;                /* batch sweeps (one SpMM each) */
  int64_t sweeps_fp32;           /* of which in FP32 */
  int64_t column_iterations;     /* sum over vectors of their own iteration counts */
  int64_t max_column_iterations;
  int32_t kernel_launches;
  int32_t refined;               /* mixed: 1 when the FP64 phase ran as one anchor sweep and
                                    refinement sweeps gathering the FP32 correction */
  double sweep_seconds;          /* device time of the sweeps alone (no copies, set-up) */
  int64_t column_iterations_fp32; /* of column_iterations, those in FP32 sweeps */
} NetBatchInfo;

/* Personalised PageRank for `batch` teleport vectors at once (one sparse
 * matrix times dense matrix product per sweep). personalization and out are
 * column-major n x batch: vector c at offset c * n. Each vector gets exactly
 * the result of net_pagerank with that personalization (own rescaling,
 * dangling mass and stopping sweep). precision 0 = FP64, 1 = mixed. */
NET_API int32_t net_pagerank_batch(const GraphHandle *h, double damping,
                           int32_t directed, int32_t weighted,
                           const double *personalization, int64_t batch,
                           int32_t dangling, int32_t loops, double tol,
                           int64_t max_iter, int32_t precision, double *out,
                           NetBatchInfo *info, char *err, size_t err_len);

/* As net_pagerank_batch with device pointers. */
NET_API int32_t net_pagerank_batch_device(const GraphHandle *h, double damping,
                                  int32_t directed, int32_t weighted,
                                  const double *d_personalization, int64_t batch,
                                  int32_t dangling, int32_t loops, double tol,
                                  int64_t max_iter, int32_t precision,
                                  double *d_out, NetBatchInfo *info, char *err,
                                  size_t err_len);

/* PageRank on every graph of a packed batch: the handle holds `count`
 * graphs side by side (graph k on nodes node_offsets[k] ..
 * node_offsets[k + 1] - 1, no edge between graphs, e.g. ego networks built
 * into one handle), and out receives, for every graph, what net_pagerank on
 * that graph alone returns. One persistent CUDA launch solves all graphs.
 * personalization is NULL (uniform per graph) or n values (rescaled per
 * graph); iterations (NULL or count values) receives each graph's
 * iteration count. */
NET_API int32_t net_pagerank_graphs(const GraphHandle *h, int64_t count,
                            const int64_t *node_offsets, double damping,
                            int32_t directed, int32_t weighted,
                            const double *personalization, int32_t dangling,
                            int32_t loops, double tol, int64_t max_iter,
                            double *out, int64_t *iterations,
                            NetSolveInfo *info, char *err, size_t err_len);

/* PageRank of the graph's structure with the edge weights d_weights (device,
 * m values in input edge order, nonnegative) instead of its own; device
 * pointers throughout. Weights are used as strengths (weighted PageRank). */
NET_API int32_t net_pagerank_weights_device(const GraphHandle *h,
                                    const double *d_weights, double damping,
                                    int32_t directed,
                                    const double *d_personalization,
                                    int32_t dangling, int32_t loops, double tol,
                                    int64_t max_iter, int32_t precision,
                                    double *d_out, NetSolveInfo *info,
                                    char *err, size_t err_len);

/* Gradient of a loss with respect to the edge weights of weighted PageRank:
 * given the scores d_scores (from net_pagerank_weights_device with the same
 * arguments) and dL/dscores in d_grad_scores, writes dL/dweights (m values,
 * input edge order) to d_grad_weights, by the adjoint solve
 * (I - d M - d jump 1_D^T)^T lambda = dL/dscores and
 * dL/dw_e = d f_e (x_j / s_j) (lambda_i - (M^T lambda)_j) for e = (j -> i).
 * d_lambda (NULL or n values) receives the adjoint vector. tol bounds the
 * L1 change of lambda relative to max(1, ||dL/dscores||_1). */
NET_API int32_t net_pagerank_grad_device(const GraphHandle *h,
                                 const double *d_weights, const double *d_scores,
                                 const double *d_grad_scores, double damping,
                                 int32_t directed,
                                 const double *d_personalization,
                                 int32_t dangling, int32_t loops, double tol,
                                 int64_t max_iter, double *d_grad_weights,
                                 double *d_lambda, NetSolveInfo *info,
                                 char *err, size_t err_len);

/* Builds a graph from device arrays: 32-bit endpoints and FP32 (d_w32) or
 * FP64 (d_w64) weights, either may be NULL. */
NET_API int32_t net_graph_new_device(int64_t n, const uint32_t *d_src,
                             const uint32_t *d_tgt, const float *d_w32,
                             const double *d_w64, int64_t m, int32_t directed,
                             GraphHandle **out, char *err, size_t err_len);

/* The graph of a frame's observed edge rows, as the reference's frame builder
 * makes it from a validated frame (graph_of, crates/engine/src/frame/
 * build.rs:106-121), built on the device from the resolved edge table:
 * endpoint node indices src[e], tgt[e] of every row over n nodes, weights
 * (NULL: none) and missing flags (NULL: every row observed; rows flagged 1
 * are left out). Edges keep row order; edge_rows (NULL or m values) receives
 * each graph edge's table row and *edge_count (NULL allowed) the number of
 * edges. The reference reaches this step through net_frame_build
 * (crates/capi/src/frame.rs:651), which takes a typed frame handle; this
 * entry point starts from the resolved indices. */
NET_API int32_t net_frame_graph(int64_t n, const int64_t *src, const int64_t *tgt,
                                const double *weights, const uint8_t *missing, int64_t m,
                                int32_t directed, GraphHandle **out, int64_t *edge_rows,
                                int64_t *edge_count, char *err, size_t err_len);

/* Every ego network of a frame at once (the reference's ego_subgraph,
 * crates/engine/src/frame/build.rs:153-194 and 220-238, reached one ego at
 * a time through net_frame_subgraph, crates/capi/src/frame.rs:952): ego k
 * has the nodes i with node_ego[i] == k, ascending, and the observed rows e
 * with edge_ego[e] == k whose endpoints are both in ego k, in row order
 * (labels outside 0..egos-1 mark a node or row of no ego; edge_ego NULL:
 * every row takes its source's ego, as the reference's resolved ego codes
 * do, crates/engine/src/frame/validate.rs:115-117). The egos are
 * packed back to back into one graph, ego k on nodes node_offsets[k] ..
 * node_offsets[k + 1] - 1 (egos + 1 values written), ready for
 * net_pagerank_graphs; node_ids (NULL or n values) receives the table's
 * node index of each packed node, edge_rows (NULL or m values) the table
 * row of each packed edge, *edge_count the number of edges. */
NET_API int32_t net_frame_egos(int64_t n, const int64_t *src, const int64_t *tgt,
                               const double *weights, const uint8_t *missing, int64_t m,
                               int32_t directed, const int64_t *node_ego, const int64_t *edge_ego,
                               int64_t egos, GraphHandle **out, int64_t *node_offsets,
                               int64_t *node_ids, int64_t *edge_rows, int64_t *edge_count,
                               char *err, size_t err_len);

/* Number of arcs of the out (which = 0), in (1) or undirected (2) CSR. */
NET_API int64_t net_graph_arc_count(const GraphHandle *h, int32_t which);

/* Copies a CSR to the host: off (n + 1), tgt and edge (the input edge of
 * each arc) and w (weighted graphs) hold one value per arc; any of tgt,
 * edge, w may be NULL. which: 0 out, 1 in, 2 directions ignored. */
NET_API int32_t net_graph_csr(const GraphHandle *h, int32_t which, uint32_t *off,
                      uint32_t *tgt, uint32_t *edge, double *w, char *err,
                      size_t err_len);

/* Copies the edge list (input order) to the host; w may be NULL. */
NET_API int32_t net_graph_edges(const GraphHandle *h, int64_t *src, int64_t *tgt,
                        double *w, char *err, size_t err_len);

/* Synthetic R-MAT graph (Chakrabarti, Zhan and Faloutsos 2004) built on the
 * device: m = edge_factor << scale draws; edge k takes `scale` 32-bit words
 * of Philox stream (seed, k), most significant level first, quadrant
 * a / b / c / d by comparing with floor(a 2^32), floor((a+b) 2^32),
 * floor((a+b+c) 2^32). clean != 0 removes self-loops and duplicates
 * (sorted); symmetrize != 0 also merges (u, v) and (v, u) and builds an
 * undirected graph. lognormal != 0 draws weights exp(N(0, 1)) rounded to
 * FP32 (Box-Muller on stream (wseed, e) of cleaned edge e). *m_out
 * receives the edge count. */
NET_API int32_t net_generate_rmat(int32_t scale, int64_t edge_factor, double a,
                          double b, double c, uint64_t seed, int32_t clean,
                          int32_t symmetrize, int32_t lognormal, uint64_t wseed,
                          GraphHandle **out, int64_t *m_out, char *err,
                          size_t err_len);

/* `count` G(n, m) graphs (the reference's generator, crates/engine/src/
 * generate.rs:255-290): graph k has n[k] nodes and m[k] distinct edges drawn
 * by Floyd's sampling from Philox stream (seed, k), sorted; its nodes are
 * numbered after those of graphs 0..k-1, so the edges of all graphs form
 * one packed batch for net_pagerank_graphs. src and tgt hold sum(m) values. */
NET_API int32_t net_generate_gnm(int64_t count, const int64_t *n, const int64_t *m,
                         int32_t directed, int32_t loops, uint64_t seed,
                         int64_t *src, int64_t *tgt, char *err, size_t err_len);

/* count sizes from the power law p(x) ~ x^-alpha on [lo, hi] (inverse
 * transform of the continuous law, floored), size k from stream (seed, k). */
NET_API int32_t net_power_law_sizes(int64_t count, double alpha, double lo,
                            double hi, uint64_t seed, int64_t *out, char *err,
                            size_t err_len);

/* Timing of the merge-path sweep kernel in the last PageRank solve of the
 * calling thread, when enabled with net_set_sweep_timing(1), for the FP32
 * (phase 0) or FP64 (phase 1) sweeps: launches, their total device
 * milliseconds (CUDA events) and the algorithmic bytes one sweep moves. */
NET_API int32_t net_sweep_timing(int32_t phase, int64_t *launches, double *total_ms,
                         double *bytes_per_launch);
NET_API void net_set_sweep_timing(int32_t on);

/* Process-wide tuning of the PageRank sweeps (results stay within the
 * documented tolerances whatever the setting): key 0 = merge-path items per
 * thread (0 automatic, 4, 8, 16); 1 = renumber nodes by gather frequency
 * (1, default) or not (0); 2 = mixed precision: leave FP32 once the change is
 * below tol times this factor (default 8192); 3 = ... or below this floor
 * (default 2e-6); 4 = sweep kernel (0 automatic, 1 one merge-path tile per
 * CTA, 2-5 one tile per warp, 6 and 7 persistent warp tiles with the most
 * gathered nodes in shared memory, 32 or 16 warps per SM, 8 warp tiles whose
 * gathers allocate in L1 only for the most gathered columns, 9 and 10 the
 * sliced layout: nodes renumbered by row length, long rows by whole warps,
 * the others one lane per row, with 48 or 64 resident warps per SM, 11 the
 * sliced layout with the most gathered values in shared memory, one CTA per
 * SM, 12 the sliced layout with its column and value streams staged in
 * shared memory by bulk copies; 0 lets the library choose: on operators of
 * at least 2^21 arcs the first solve times the candidates and keeps the
 * fastest); 5 = preferred
 * shared-memory carveout of the sweep (-1 just what the CTAs the kernel keeps
 * resident need, 0..100 percent);
 * 6 = threads per CTA of the packed-graph PageRank (0 tuned on first use,
 * 128, 256, 512, 1024); 7 = the most nodes kernels 6 and 7 keep in shared
 * memory (-1 as many as fit, 0 none), or the columns below which kernel 8
 * gathers allocate in L1 (-1: 24,576); 8 = warp-tile sweeps launch one warp
 * per tile (0) or only the CTAs that fit on the GPU at once, each warp
 * looping over tiles (1, default); 9 = mixed precision ends with one FP64
 * anchor sweep and refinement sweeps that gather the FP32 correction (1,
 * default) or with FP64 sweeps (0); 10 = sliced sweeps: rows of at least
 * this many arcs (1..65535) are taken by whole warps (0: automatic); 11 =
 * FP32 values kernel 11 keeps in shared memory (-1: 32,768); 12 = pick the
 * sweep kernel per operator by timing (1, default) or always use kernel 9
 * (0); 13 = CTAs per SM kernel 12 sizes its shared memory for (0: 4, 1..8);
 * 14 = for testing kernel 12's bounded waits: the chunk of the grid's first
 * warp whose copies are never issued, so that its wait runs out after about
 * one second and the solve fails with an error (-1, default: none);
 * 15 = packed graphs: graphs of at least this many nodes are each split
 * over a thread-block cluster (0, default: the larger of 4096 and the node
 * count over the launch's CTAs); 16 = packed graphs: CTAs per cluster for
 * those graphs (0 tuned with key 6 per batch, 1 none, 4, 8); 17 = FP64
 * PageRank (teleport vector, if any, in host memory) on at most this many
 * edges runs as one
 * packed-graph launch (default 262,144; 0 never; NetSolveInfo.sweep_kernel is
 * then 0). Setting key 0, 4, 7 or 10 also bypasses the timing.
 * Returns 1 for an unknown key or value. */
NET_API int32_t net_set_tuning(int32_t key, double value);

/* Eigenvalues (ascending, n doubles) and eigenvectors (the columns of the
 * row-major n x n `vectors`) of a symmetric n x n matrix (row-major, n at
 * most 20), computed by the device solver that eigenvector centrality's
 * Lanczos process runs on its projected matrices. Fails if the QL iteration
 * does not converge. */
NET_API int32_t net_projected_eigen(int64_t n, const double *a, double *values,
                                    double *vectors, char *err, size_t err_len);

/* PageRank (uniform teleport, weights as strengths when d_weights is not
 * NULL) of one graph given as device arrays of its in-arcs: d_offsets (n + 1)
 * and d_sources, d_weights (one per arc, or NULL), scores to d_out (n
 * doubles); on `stream` (NULL: the default stream). It allocates no device
 * memory, for callers that cannot call cudaMalloc (a host framework that has
 * reserved the device memory for its own allocator, or a path that must not
 * stall the device, which cudaMalloc and cudaFree may do): its scratch is a
 * static device array of the library holding graphs of up to 262,144 (2^18)
 * nodes (8 MiB, held on every device that loads the library); larger graphs
 * are rejected with an error. The kernel checks the arrays before it uses
 * them: offsets that decrease, a source outside [0, n) or a weight that is
 * negative or not finite fail the call with a message naming the first such
 * row or arc. Out-strengths are summed in a fixed order, so repeated calls
 * give identical scores. A tolerance or iteration cap that is not positive
 * (a NaN tolerance included) selects the defaults 1e-12 and 10000, as in
 * net_pagerank. The first call on a device looks up the array's address,
 * so it should come before any stream capture. All calls share the array:
 * calls that overlap on the GPU race and must be serialized by the caller.
 * No counterpart in the reference. */
NET_API int32_t net_pagerank_csr_static(int64_t n, const uint32_t *d_offsets,
                                const uint32_t *d_sources,
                                const double *d_weights, double damping,
                                double tol, int64_t max_iter, double *d_out,
                                int64_t *iterations, void *stream, char *err,
                                size_t err_len);

/* PageRank of one graph split over several GPUs by rows of its pull
 * operator (in-arcs with directed set on a directed graph, else all arcs),
 * one process per GPU. No counterpart in the reference, whose loop
 * (crates/engine/src/metrics/spectral.rs:247-280) runs in one process.
 *
 * net_shard_bounds writes parts + 1 row boundaries (0 first, n last) that
 * give each of `parts` ranks about an equal share of rows plus arcs. Each
 * rank then builds its shard with the same graph, options and boundaries
 * (net_shard_new; the options and their checks are net_pagerank's, with the
 * personalization vector, if any, given as n device doubles) and starts
 * from the uniform iterate. A sweep is: net_shard_sweep on every rank,
 * writing *payload_len doubles (device) -- the unnormalised scores of its
 * rows and their sum; an all-gather of the ranks' payloads in rank order
 * (parts * payload_len doubles, e.g. ncclAllGather); net_shard_finish on
 * every rank with the gathered payloads, which normalises the new iterate
 * over all nodes, returns its L1 change from the previous one in *change
 * (host; waits for the stream) and readies the next sweep. Every rank
 * computes the same iterate bit for bit, so all ranks stop on the same
 * sweep when the change reaches the tolerance, as net_pagerank does; the
 * caller runs that loop (and its iteration cap). net_shard_scores copies
 * the current iterate (n doubles) to host or device memory;
 * net_shard_restart returns the shard to the uniform iterate. The shard
 * lives on the current device and reads the graph's arrays, so the graph
 * must outlive it; its calls run on `stream` (NULL: the default stream),
 * which must order them (the sweep reads what the previous finish wrote),
 * and one shard must not be used by two threads at once.
 * The boundaries must not decrease and parts is at most 1024. */
typedef struct NetShard NetShard;
NET_API int32_t net_shard_bounds(const GraphHandle *h, int32_t directed,
                                 int32_t weighted, int32_t loops,
                                 int32_t parts, int64_t *bounds, char *err,
                                 size_t err_len);
NET_API int32_t net_shard_new(const GraphHandle *h, double damping,
                              int32_t directed, int32_t weighted,
                              const double *d_personalization,
                              int32_t dangling, int32_t loops,
                              const int64_t *bounds, int32_t parts,
                              int32_t rank, NetShard **shard,
                              int64_t *payload_len, char *err,
                              size_t err_len);
NET_API int32_t net_shard_sweep(NetShard *shard, double *d_payload,
                                void *stream, char *err, size_t err_len);
NET_API int32_t net_shard_finish(NetShard *shard, const double *d_gathered,
                                 double *change, void *stream, char *err,
                                 size_t err_len);
NET_API int32_t net_shard_scores(const NetShard *shard, double *out,
                                 int32_t out_on_device, void *stream,
                                 char *err, size_t err_len);
NET_API int32_t net_shard_restart(NetShard *shard, void *stream, char *err,
                                  size_t err_len);
NET_API void net_shard_free(NetShard *shard);

/* Calibration: random 4-byte gathers per second the whole GPU sustains,
 * from a device array of `words` FP32 values (source 0; an array that fits
 * in L2 gives the rate a sparse sweep's gathers of its iterate run into),
 * from each SM's own shared memory (source 1), or from the shared memory of
 * a thread-block cluster of 2, 4 or 8 CTAs (source 2, 4, 8). Takes tens of
 * milliseconds. */
NET_API int32_t net_measure_gather(int32_t source, int64_t words, double *gathers_per_second,
                                   char *err, size_t err_len);

/* Waits for the device; reports an asynchronous CUDA error if one occurred. */
NET_API int32_t net_device_sync(char *err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* KNAPPNET_H */
