/*
 * vine_workloads.h -- seeded synthetic CSP workloads and file loaders.
 *
 * A workload is a directed graph in CSR form plus a list of queries
 * (source, sink, delay budget).  It stands in for the reference's input
 * layer: the graph loaders read_graph (include/io.hpp:22-93), the query
 * loaders task::read_query / task::load_query (include/task.hpp:27-76) and
 * the adjacency -> CSR conversion Graph::adj_to_csr (include/graph.hpp:136-167).
 * The generators are deterministic functions of their parameters (one
 * std::mt19937_64 stream per workload, fixed draw order).
 *
 * All functions return VINE_OK (0) or a negative vine_status code
 * (see vine.h); no exceptions cross this boundary.
 */
#ifndef VINE_WORKLOADS_H_
#define VINE_WORKLOADS_H_

#include <stdint.h>

#include "vine.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vine_workload vine_workload;

enum vine_workload_kind {
  VINE_WL_GRID = 1,          /* 4-neighbour grid, len/delay ~ U{1..100}          */
  VINE_WL_ROAD_LOGNORMAL = 2,/* jittered planar lattice, delay = len*lognormal    */
  VINE_WL_ROAD_ANTICORR = 3, /* same lattice, delay = 1e4/len * U[0.5,1.5)        */
  VINE_WL_CHUNGLU = 4,       /* Chung-Lu power law, len/delay ~ U{1..100}        */
  VINE_WL_ROAD_BATCH = 5     /* road (lognormal) graph, hop-sampled query batch  */
};

typedef struct {
  int32_t kind;        /* vine_workload_kind                                   */
  uint64_t seed;
  int32_t rows, cols;  /* grid / lattice shape (vertices = rows*cols)          */
  int64_t n;           /* Chung-Lu vertex count                                */
  int64_t m_target;    /* target number of arcs (road, Chung-Lu)               */
  double exponent;     /* Chung-Lu degree exponent                             */
  int32_t n_pairs;     /* number of source/sink pairs                          */
  int32_t n_alpha;     /* >0: each pair is used once per alpha[i];             */
  float alpha[4];      /*  0: one query per pair, alpha ~ U[alpha_lo,alpha_hi) */
  float alpha_lo, alpha_hi;
  int32_t hop_lo, hop_hi; /* sink sampled at a BFS hop distance in [lo,hi];    */
  int32_t hop_log_uniform;/* 0 = uniform random pairs when hop_hi == 0          */
  int32_t nthreads;    /* host threads for budgets / BFS (0 = all cores)       */
  uint64_t query_seed; /* 0: queries continue the graph's random stream;       */
                       /* else they come from their own stream with this seed */
} vine_workload_params;

/* Default parameters of the five benchmark workloads (config_id 1..5). */
int vine_workload_default_params(int32_t config_id, vine_workload_params *out);

/* Generates a workload.  The delay budget of a query with pair (s, t) and
 * fraction alpha is floor(dmin + alpha * (dlen - dmin)), where dmin is the
 * smallest s->t delay and dlen the delay of the shortest s->t path by length
 * (ties broken by smaller delay); unreachable sinks get budget -1. */
int vine_workload_generate(const vine_workload_params *p, vine_workload **out);

/* Reads a 5-column MatrixMarket-style edge list ("eid src snk len delay"
 * rows after a '%' header and an "n n m" line, as in the reference's
 * inputs/tech-*.mtx.txt).  Each row is added in both directions, as the
 * reference's type-1 loader does (include/io.hpp:30-60).  No queries. */
int vine_workload_load_mtx(const char *path, vine_workload **out);

/* Reads a COLA road graph ("N" then "u: v len delay v len delay ... -1"
 * lines, include/io.hpp:61-91) and optionally a COLA query file
 * ("u v cost_lower cost_upper cost_limit" rows; the budget is cost_limit,
 * include/task.hpp:61-76).  query_path may be NULL. */
int vine_workload_load_cola(const char *graph_path, const char *query_path,
                            vine_workload **out);

/* Appends n_pairs random distinct pairs with the given alphas (budget rule
 * as in vine_workload_generate). */
int vine_workload_add_random_queries(vine_workload *w, uint64_t seed, int32_t n_pairs,
                                     int32_t n_alpha, const float *alpha);

/* Borrowed views; valid until vine_workload_destroy. */
int vine_workload_graph(const vine_workload *w, int32_t *n, int64_t *m, const int64_t **row_ptr,
                        const int32_t **col, const float **len, const float **delay);
int vine_workload_queries(const vine_workload *w, int32_t *nq, const int32_t **src,
                          const int32_t **dst, const float **budget, const float **alpha);

void vine_workload_destroy(vine_workload *w);

#ifdef __cplusplus
}
#endif

#endif /* VINE_WORKLOADS_H_ */
