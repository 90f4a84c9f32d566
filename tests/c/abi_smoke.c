/* C99 check of the library's C interface against the reference engine's.
 *
 * Built by tests/test_capi_c.py with `cc -std=c99 -Wall -Wextra -Werror`
 * against include/knappnet.h and linked to libknappnet_b200.so, as the
 * reference checks its own header (tools/check_c_abi.sh,
 * crates/capi/tests/c/smoke.c).
 *
 * Every entry point the library takes over from the reference is assigned
 * to a pointer whose type spells out the reference's prototype
 * (crates/capi/include/netcapi.h): if knappnet.h ever declares one of them
 * with other parameter or return types, this file no longer compiles.
 *
 *   abi_smoke cpu   calls that need no GPU (NULL handles, counts, argument
 *                   errors reported before any device work)
 *   abi_smoke gpu   builds the reference's five-node test network and checks
 *                   net_pagerank against the reference's hand values
 *                   (crates/engine/src/metrics/spectral.rs:948-979)
 */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "knappnet.h"

/* The reference's prototypes, one pointer type each. */
typedef int32_t (*graph_new_t)(int64_t, const int64_t *, const int64_t *, const double *,
                               int64_t, int32_t, GraphHandle **, char *, size_t);
typedef void (*graph_free_t)(GraphHandle *);
typedef int64_t (*graph_count_t)(const GraphHandle *);
typedef int32_t (*degree_t)(const GraphHandle *, int32_t, int32_t, int32_t, double *, char *,
                            size_t);
typedef int32_t (*pagerank_t)(const GraphHandle *, double, int32_t, int32_t, const double *,
                              int32_t, int32_t, double, int64_t, int32_t, double *, char *,
                              size_t);
typedef int32_t (*eigenvector_t)(const GraphHandle *, int32_t, int32_t, int32_t, int32_t, double,
                                 int64_t, int32_t, double *, double *, int32_t *, char *,
                                 size_t);
typedef int32_t (*katz_t)(const GraphHandle *, double, const double *, int64_t, int32_t, int32_t,
                          int32_t, int32_t, double, int64_t, int32_t, double *, char *, size_t);
typedef int32_t (*bonacich_t)(const GraphHandle *, double, int32_t, int32_t, int32_t, int32_t,
                              double, int64_t, int32_t, double *, char *, size_t);
typedef int32_t (*hits_t)(const GraphHandle *, int32_t, int32_t, int32_t, double, int64_t,
                          int32_t, double *, double *, double *, int32_t *, char *, size_t);
typedef int32_t (*components_t)(const GraphHandle *, int32_t, int32_t *, int64_t *, char *,
                                size_t);
typedef int32_t (*centralization_t)(const GraphHandle *, int32_t, int32_t, int32_t, int32_t,
                                    int32_t, int32_t, double *, char *, size_t);
typedef int32_t (*simplify_t)(const GraphHandle *, int32_t, int32_t, GraphHandle **, char *,
                              size_t);
typedef int32_t (*twomode_t)(const GraphHandle *, const int32_t *, double, int64_t, int32_t,
                             double *, double *, int32_t *, char *, size_t);
typedef int32_t (*leading_eigen_t)(const GraphHandle *, int32_t, int64_t *, double *, int64_t *,
                                   char *, size_t);

static int failures = 0;

static void check(int ok, const char *what) {
  if (!ok) {
    fprintf(stderr, "FAILED: %s\n", what);
    ++failures;
  }
}

static int run_cpu(void) {
  graph_free_t graph_free = net_graph_free;
  graph_count_t node_count = net_graph_node_count;
  graph_count_t edge_count = net_graph_edge_count;
  degree_t degree = net_degree;
  pagerank_t pagerank = net_pagerank;
  eigenvector_t eigenvector = net_eigenvector;
  katz_t katz = net_katz;
  bonacich_t bonacich = net_bonacich_power;
  hits_t hits = net_hits;
  components_t components = net_components;
  centralization_t centralization = net_centralization;
  simplify_t simplify = net_graph_simplify;
  twomode_t twomode = net_twomode_eigenvector;
  leading_eigen_t leading = net_leading_eigen;
  graph_new_t graph_new = net_graph_new;
  char err[256];
  double out[4], value = 0.0;
  int32_t flag = 0, memb[4] = {0, 0, 0, 0};
  int64_t count = 0, lmemb[4], splits = 0;
  GraphHandle *g = NULL;

  (void)graph_new;  /* its type is checked; building a graph needs a GPU */
  check(node_count(NULL) == -1, "node count of NULL is -1");
  check(edge_count(NULL) == -1, "edge count of NULL is -1");
  graph_free(NULL);
  /* every measure fails cleanly on a NULL handle, with a message */
  err[0] = 0;
  check(pagerank(NULL, 0.85, 1, 0, NULL, 0, 0, 0.0, 0, 0, out, err, sizeof err) != 0 &&
            strstr(err, "null") != NULL,
        "net_pagerank on NULL");
  check(degree(NULL, 1, 1, 0, out, err, sizeof err) != 0, "net_degree on NULL");
  check(eigenvector(NULL, 3, 0, 0, 0, 0.0, 0, 0, out, &value, &flag, err, sizeof err) != 0,
        "net_eigenvector on NULL");
  check(katz(NULL, 0.1, NULL, 0, 2, 0, 1, 1, 0.0, 0, 0, out, err, sizeof err) != 0,
        "net_katz on NULL");
  check(bonacich(NULL, 0.5, 1, 0, 2, 0, 0.0, 0, 0, out, err, sizeof err) != 0,
        "net_bonacich_power on NULL");
  check(hits(NULL, 0, 0, 0, 0.0, 0, 0, out, out, &value, &flag, err, sizeof err) != 0,
        "net_hits on NULL");
  check(components(NULL, 0, memb, &count, err, sizeof err) != 0, "net_components on NULL");
  check(centralization(NULL, 3, 3, 0, 1, 0, 0, out, err, sizeof err) != 0,
        "net_centralization on NULL");
  check(simplify(NULL, 0, 0, &g, err, sizeof err) != 0, "net_graph_simplify on NULL");
  check(twomode(NULL, memb, 0.0, 0, 0, out, &value, &flag, err, sizeof err) != 0,
        "net_twomode_eigenvector on NULL");
  check(leading(NULL, 0, lmemb, &value, &splits, err, sizeof err) != 0,
        "net_leading_eigen on NULL");
  /* the extensions check their arguments before any device work */
  const int64_t ends[2] = {0, 1};
  int64_t offs[3];
  GraphHandle *fg = NULL;
  err[0] = 0;
  check(net_frame_graph(2, ends, ends, NULL, NULL, 2, 1, NULL, NULL, NULL, err, sizeof err) != 0 &&
            strstr(err, "out is null") != NULL,
        "net_frame_graph without an output handle");
  check(net_frame_egos(2, ends, ends, NULL, NULL, 2, 1, ends, NULL, 2, &fg, NULL, NULL, NULL,
                       NULL, err, sizeof err) != 0 &&
            strstr(err, "node_offsets is null") != NULL && fg == NULL,
        "net_frame_egos without node offsets");
  check(net_frame_egos(2, ends, ends, NULL, NULL, 2, 1, NULL, NULL, 2, &fg, offs, NULL, NULL,
                       NULL, err, sizeof err) != 0 &&
            strstr(err, "node_ego is null") != NULL,
        "net_frame_egos without node ego labels");
  check(net_measure_gather(3, 1 << 20, &value, err, sizeof err) != 0 &&
            strstr(err, "gather source") != NULL,
        "net_measure_gather with an unknown source");
  check(net_projected_eigen(21, out, out, out, err, sizeof err) != 0 &&
            strstr(err, "between 0 and 20") != NULL,
        "net_projected_eigen beyond order 20");
  check(net_projected_eigen(0, NULL, NULL, NULL, err, sizeof err) == 0,
        "net_projected_eigen of order 0 does nothing");
  check(net_set_tuning(99, 0.0) != 0 && net_set_tuning(17, -1.0) != 0,
        "net_set_tuning rejects unknown keys and values");
  int64_t bounds[3] = {0, 1, 2}, plen = 0;
  NetShard *sh = NULL;
  check(net_shard_bounds(NULL, 1, 0, 0, 2, bounds, err, sizeof err) != 0 &&
            strstr(err, "graph handle is null") != NULL,
        "net_shard_bounds on NULL");
  check(net_shard_new(NULL, 0.85, 1, 0, NULL, 0, 0, bounds, 2, 0, &sh, &plen, err,
                      sizeof err) != 0 && sh == NULL,
        "net_shard_new on NULL");
  check(net_shard_sweep(NULL, out, NULL, err, sizeof err) != 0 &&
            strstr(err, "shard handle is null") != NULL,
        "net_shard_sweep on NULL");
  check(net_shard_finish(NULL, out, &value, NULL, err, sizeof err) != 0,
        "net_shard_finish on NULL");
  check(net_shard_scores(NULL, out, 0, NULL, err, sizeof err) != 0, "net_shard_scores on NULL");
  check(net_shard_restart(NULL, NULL, err, sizeof err) != 0, "net_shard_restart on NULL");
  net_shard_free(NULL);
  /* a message is cut to the buffer and NUL-terminated */
  char tiny[5];
  memset(tiny, 'x', sizeof tiny);
  check(pagerank(NULL, 0.85, 1, 0, NULL, 0, 0, 0.0, 0, 0, out, tiny, sizeof tiny) != 0 &&
            tiny[4] == 0,
        "message truncated with a terminating NUL");
  return failures;
}

static int run_gpu(void) {
  /* 0 -> 1, 0 -> 2, 1 -> 2, 2 -> 0, 3 -> 2, 2 -> 4; node 4 has no out-arcs */
  const int64_t src[] = {0, 0, 1, 2, 3, 2};
  const int64_t tgt[] = {1, 2, 2, 0, 2, 4};
  const double uniform[] = {0.2142011097, 0.1574496602, 0.3477339318, 0.0664141886,
                            0.2142011097};
  const double at_zero[] = {0.3928645968, 0.1669674536, 0.3088897892, 0.0, 0.1312781604};
  const double spread[] = {0.3166510816, 0.1629073936, 0.3254597594, 0.0283306839,
                           0.1666510816};
  const double p[] = {1.0, 0.0, 0.0, 0.0, 0.0};
  graph_new_t graph_new = net_graph_new;
  pagerank_t pagerank = net_pagerank;
  char err[256];
  double x[5];
  GraphHandle *g = NULL;
  err[0] = 0;
  check(graph_new(-1, NULL, NULL, NULL, 0, 1, &g, err, sizeof err) != 0 && err[0] != 0 &&
            g == NULL,
        "a negative node count fails with a message and no handle");
  if (graph_new(5, src, tgt, NULL, 6, 1, &g, err, sizeof err) != 0) {
    fprintf(stderr, "net_graph_new: %s\n", err);
    return 1;
  }
  check(net_graph_node_count(g) == 5 && net_graph_edge_count(g) == 6, "counts");
  const double *want[3] = {uniform, at_zero, spread};
  const double *pers[3] = {NULL, p, p};
  const int32_t dangling[3] = {0, 0, 1};
  for (int k = 0; k < 3; ++k) {
    if (pagerank(g, 0.85, 1, 0, pers[k], dangling[k], 0, 0.0, 0, 0, x, err, sizeof err) != 0) {
      fprintf(stderr, "net_pagerank: %s\n", err);
      ++failures;
      continue;
    }
    double worst = 0.0;
    for (int i = 0; i < 5; ++i) worst = fmax(worst, fabs(x[i] - want[k][i]));
    printf("pagerank case %d: largest difference from the hand values %.3e\n", k, worst);
    check(worst <= 1e-9, "PageRank within 1e-9 of the reference's hand values");
  }
  err[0] = 0;
  check(pagerank(g, 1.5, 1, 0, NULL, 0, 0, 0.0, 0, 0, x, err, sizeof err) != 0 && err[0] != 0,
        "damping 1.5 fails");
  net_graph_free(g);
  return failures;
}

int main(int argc, char **argv) {
  const char *mode = argc > 1 ? argv[1] : "cpu";
  int bad = strcmp(mode, "gpu") == 0 ? run_gpu() : run_cpu();
  printf("%s checks: %s\n", mode, bad ? "FAILED" : "ok");
  return bad ? 1 : 0;
}
