/*
 * vine.h -- C ABI of the B200 exact constrained-shortest-path (CSP) engine.
 *
 * Problem (the reference's CSP=1 instance): a label is a partial path
 * (vid, d, delay) from the source; expanding it over arc (u -> v, len, dly)
 * gives (v, d + len, delay + dly) (include/label.hpp:214-222); label a
 * dominates b when a.d <= b.d and a.delay <= b.delay
 * (include/label.hpp:234-236); a label is feasible when !(delay > budget)
 * (include/constraint.hpp:99-101).  A query asks for the feasible
 * source -> sink path of smallest cost d; ties are broken by smaller delay,
 * so the answer (cost, delay) is unique.
 *
 * The reference binds this path only through C++ templates -- the query class
 * cspp<Label_t, Edge_t> (algorithm/cspp.hpp:11-69) and its GPU driver
 * RUN_CSPP (algorithm/cspp.cuh:50-58, 69-325).  Each entry point below names
 * the reference interface it replaces.  include/vine/cspp.hpp layers the
 * reference's class shape on top of these functions.
 *
 * Conventions: every function returns a vine_status (0 = VINE_OK, negative =
 * error); no C++ exception crosses this boundary; output buffers are owned by
 * the caller; the last error message of the calling thread is available from
 * vine_last_error().  Weights must be finite and >= 0.  Optimal costs are
 * bit-exact (the same FP32 additions along the same path as the reference)
 * whenever the weights are integers whose path sums stay below 2^24.
 */
#ifndef VINE_H_
#define VINE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  VINE_OK = 0,
  VINE_ERR_INVALID = -1,   /* bad argument                                   */
  VINE_ERR_CAPACITY = -2,  /* a label pool / pile / table / output overflowed */
  VINE_ERR_CUDA = -3,      /* CUDA runtime error                             */
  VINE_ERR_TIMEOUT = -4,   /* a bounded device wait gave up                  */
  VINE_ERR_NO_DEVICE = -5, /* no usable CUDA device                          */
  VINE_ERR_IO = -6,        /* file could not be read / parsed                */
  VINE_ERR_INTERNAL = -7
} vine_status;

/* Thread-local text of the last error (never NULL). */
const char *vine_last_error(void);
/* Library version string. */
const char *vine_version(void);

/* ------------------------------------------------------------------ graph */

typedef struct vine_graph vine_graph;

/* Uploads a CSR graph to `device` (SoA: row_ptr[n+1], col[m], len[m],
 * delay[m]; arcs of vertex u are col[row_ptr[u] .. row_ptr[u+1])).  Also
 * builds the reverse CSR used by the lower-bound searches.
 * Replaces Graph::adj_to_csr + Graph::make_gpu_graph
 * (include/graph.hpp:136-195) and the gpuGraph device struct
 * (include/gpu_graph.hpp:5-35). */
int vine_graph_create(int32_t device, int32_t n, int64_t m, const int64_t *row_ptr,
                      const int32_t *col, const float *len, const float *delay,
                      vine_graph **out);
void vine_graph_destroy(vine_graph *g);
/* n, m, and 1 when every weight is an integer < 2^24 (exactness regime). */
int vine_graph_info(const vine_graph *g, int32_t *n, int64_t *m, int32_t *integral);

/* ----------------------------------------------------------------- config */

enum vine_engine {
  VINE_ENGINE_BATCH = 0, /* persistent kernel, one query per CTA worker     */
  VINE_ENGINE_PLAIN = 1  /* one query at a time, whole GPU, host-driven     */
};
enum vine_mode {
  VINE_MODE_OPTIMAL = 0, /* prune by the incumbent; answer = lex-min label  */
  VINE_MODE_PARETO = 1   /* no incumbent / bounds: full sink Pareto set     */
};
enum vine_policy {
  VINE_POLICY_FIXED = 0, /* constant bucket width                           */
  VINE_POLICY_AR = 1,    /* AR(3) (Burg) forecast of the frontier size      */
  VINE_POLICY_MLP = 2    /* learned 16-64-64-2 scheduler (needs cfg.mlp)    */
};

typedef struct vine_mlp vine_mlp;

typedef struct {
  int32_t engine;          /* vine_engine                                     */
  int32_t mode;            /* vine_mode                                       */
  int32_t policy;          /* vine_policy                                     */
  int32_t use_bounds;      /* reverse lower bounds (delay and A* cost)        */
  int32_t block_threads;   /* batch engine: threads per query worker (CTA)    */
  int32_t ctas_per_sm;     /* batch engine: resident workers per SM (0=auto)  */
  int32_t table_log2;      /* shared-memory bucket table entries (log2)       */
  int32_t spill_log2;      /* reserved (overflow chains have no fixed size)   */
  float bucket_width;      /* bucket width in cost units (0 = auto)           */
  int32_t split_threshold; /* max labels expanded per round (0 = auto)        */
  int64_t pool_labels;     /* label arena capacity (0 = auto)                 */
  int64_t far_capacity;    /* per-worker far-pile entries (0 = auto)          */
  int32_t use_cuda_graph;  /* replay the batch launch sequence as a graph     */
  int32_t order_queries;   /* batch engine: largest budget first              */
  const vine_mlp *mlp;     /* model for VINE_POLICY_MLP                       */
  int32_t trace;           /* record per-bucket scheduler traces              */
  int32_t max_workers;     /* batch engine: cap on resident workers (0 = all) */
  int32_t sync_rounds;     /* batch engine: 1 = block-synchronous expansion
                              rounds of at most split_threshold labels;
                              0 = warps pull labels from the bucket's queue */
  int32_t band_mult;       /* batch engine: near far-pile band (64 key bins),
                              in bucket widths (0 = 16)                       */
  float ar_scale;          /* AR / MLP policies: multiplier applied to the AR
                              rule's width (0 = 1)                            */
  int32_t wait_limit;      /* every bounded device wait (lock attempts, polls
                              of the bucket queue) gives up after this many
                              tries and fails its query with VINE_ERR_TIMEOUT
                              (0 = 2^26)                                      */
  int32_t time_limit_ms;   /* per-query time limit, measured on the device's
                              global timer (host clock for the plain engine):
                              a query still running after it stops with
                              VINE_ERR_TIMEOUT (0 = 600000, i.e. 10 minutes;
                              < 0 = no limit)                                 */
  int32_t split_staging;   /* batch engine: 1 = when a bucket opens, stream its
                              far-bin / rest-pile label tiles into shared
                              memory with bulk copies (cp.async.bulk) instead
                              of per-thread loads; costs 64 bytes of shared
                              memory (taken from L1) per thread            */
} vine_config;

void vine_config_default(vine_config *cfg);

/* ---------------------------------------------------------------- results */

enum vine_stat {
  VINE_STAT_EXPANDED = 0, /* labels popped and expanded                      */
  VINE_STAT_RELAXED,      /* arcs relaxed                                    */
  VINE_STAT_INSERTED,     /* labels accepted into a store / pile             */
  VINE_STAT_DOMINATED,    /* candidates rejected by dominance                */
  VINE_STAT_BUCKETS,      /* buckets processed                               */
  VINE_STAT_ROUNDS,       /* expansion rounds                                */
  VINE_STAT_SPILLS,       /* labels stored in per-vertex HBM overflow chains */
  VINE_STAT_CYCLES,       /* device clock cycles spent on the query          */
  VINE_STAT_ABORT_SITE,   /* where a failed query stopped (0 = it did not)   */
  VINE_STAT_BOUND_ROUNDS, /* rounds of the reverse bound searches            */
  VINE_STAT_BOUND_CYCLES, /* device clock cycles of the reverse searches     */
  VINE_STAT_CHAIN_STEPS,  /* overflow-chain labels read by dominance tests   */
  VINE_STAT_SPLIT_CYCLES, /* device clock cycles opening buckets (far piles) */
  VINE_STAT_SPLIT_ITEMS,  /* far-pile labels scanned while opening buckets   */
  VINE_STAT_POLICY_CYCLES,/* device clock cycles settling + scheduler steps  */
  VINE_STAT_LOAD_CYCLES,  /* device clock cycles loading round labels + scan */
  VINE_STAT_RELAX_CYCLES, /* device clock cycles relaxing the round's arcs   */
  VINE_STAT_START_NS,     /* batch engine: device global timer (ns) when the
                             query started on its worker                     */
  VINE_STAT_TIME_NS,      /* batch engine: the query's duration on its worker
                             in ns (device global timer)                     */
  VINE_STAT_REST_ITEMS,   /* batch engine: rest-pile labels rescanned when the
                             band was rebuilt (part of SPLIT_ITEMS)          */
  VINE_STAT_IDLE_CYCLES,  /* batch engine: warp-cycles (summed over warps) of
                             polling an empty bucket queue                   */
  VINE_STAT_PUBLISH_CYCLES,/* batch engine: warp-cycles waiting to publish
                             queue entries in reservation order              */
  VINE_STAT_COUNT = 22
};

/* Values of stats[VINE_STAT_ABORT_SITE]: where a failed query stopped. */
enum vine_abort_site {
  VINE_SITE_NONE = 0,
  VINE_SITE_ARENA = 1,       /* label arena exhausted (chunk request)         */
  VINE_SITE_ARENA_ALLOC = 2, /* label arena exhausted (slot)                  */
  VINE_SITE_NEAR = 3,        /* the open bucket outgrew the near ring         */
  VINE_SITE_BAND = 4,        /* far band / bound-search pile full             */
  VINE_SITE_REST = 5,        /* rest pile full                                */
  VINE_SITE_SINK = 6,        /* sink label list full (Pareto mode)            */
  VINE_SITE_LOCK = 7,        /* a lock wait reached wait_limit                */
  VINE_SITE_ROUNDS = 8,      /* round / bucket count bound                    */
  VINE_SITE_PATH = 9,        /* path arena full                               */
  VINE_SITE_CHUNKS = 10,     /* arena chunk list full                         */
  VINE_SITE_INVALID = 11,    /* query arguments out of range                  */
  VINE_SITE_ASYNC = 12,      /* a bucket-queue wait reached wait_limit        */
  VINE_SITE_TIME = 13,       /* time_limit_ms reached                         */
  VINE_SITE_RING = 14,       /* a queue entry failed its range check          */
  VINE_SITE_TILE = 15        /* a staged label tile's copy did not land within
                                wait_limit polls (the worker then stops)      */
};

typedef struct {
  float *cost;            /* [nq] optimal cost (+inf when infeasible)        */
  float *delay;           /* [nq] delay of that path                         */
  int32_t *found;         /* [nq] 1 = feasible path exists                   */
  int32_t *status;        /* [nq] per-query vine_status                      */
  int64_t *path_offsets;  /* [nq+1] or NULL: path of q is                    */
  int32_t *path;          /*   path[path_offsets[q] .. path_offsets[q+1])    */
  int64_t path_capacity;  /*   capacity of `path` in vertices                */
  float *pareto_d;        /* [nq*pareto_stride] or NULL (VINE_MODE_PARETO)  */
  float *pareto_delay;    /* [nq*pareto_stride]                              */
  int32_t *pareto_n;      /* [nq] size of the sink Pareto set                */
  int32_t pareto_stride;
  int64_t *stats;         /* [nq*VINE_STAT_COUNT] or NULL                    */
  int32_t retried;        /* out (vine_solve): queries solved again, with
                             roomier structures and fewer workers at once,
                             after a capacity overflow                        */
} vine_results;

/* Solves nq queries (source src[q], sink dst[q], delay budget budget[q]) from
 * HOST buffers; copies in, runs, copies results out.  Replaces
 * cspp<c_label,c_edge>::solve (algorithm/cspp.hpp:48-53) -> RUN_CSPP
 * (algorithm/cspp.cuh:69-325), which returned nothing; this fills cost,
 * delay, path and (in Pareto mode) the sink's Pareto set.  Queries whose
 * status is VINE_ERR_CAPACITY are re-run, up to four times, with larger
 * piles and arena and with fewer of them running at once, before the call
 * gives up.  Returns the first per-query error, or VINE_OK. */
int vine_solve(vine_graph *g, int32_t nq, const int32_t *src, const int32_t *dst,
               const float *budget, const vine_config *cfg, vine_results *out);

/* Device-resident variant: src/dst/budget and every output pointer are device
 * pointers; work is enqueued on `stream` (a cudaStream_t; NULL means the
 * legacy default stream) and the call returns without waiting.  Paths are
 * packed in query order: out->path_offsets (nq+1 entries) receives their
 * offsets and out->path the vertices; the caller sizes `path` (up to the
 * number of vertices per query).  With cfg->use_cuda_graph the launch
 * sequence is captured once and replayed while the call's shape, buffers and
 * configuration stay the same.  Not retried on capacity errors. */
int vine_solve_device(vine_graph *g, int32_t nq, const int32_t *src, const int32_t *dst,
                      const float *budget, const vine_config *cfg, vine_results *out,
                      void *stream);

/* Splits one batch over several GPUs: graphs[k] is the same graph created on
 * device k (vine_graph_create per device).  Queries are independent, so
 * there is no exchange between devices: each solves its share with
 * vine_solve on its own host thread, and results land in `out` in query
 * order (paths packed as in vine_solve; out->retried sums the shares).
 * Shares are chosen longest-first by budget, so every device gets a similar
 * mix of heavy and light queries.  The reference runs one device
 * (main.cu:50); this is the query-replica scaling of its query loop
 * (algorithm/cspp.cuh:134-296). */
int vine_solve_multi(vine_graph **graphs, int32_t ngraphs, int32_t nq, const int32_t *src,
                     const int32_t *dst, const float *budget, const vine_config *cfg,
                     vine_results *out);

/* ---------------------------------------------------------- label variants */

/* The reference's other label types (include/label.hpp:46-465 with
 * include/constraint.hpp:21-187), chosen there at compile time by the CSP
 * macro, here per call. */
enum vine_label_kind {
  VINE_LABEL_CSP = 1,     /* (d, delay): delay <= L (CSP=1; CSP=4 is the same) */
  VINE_LABEL_HOP = 2,     /* (d, delay, hop): delay <= L and hop <= H (CSP=2)  */
  VINE_LABEL_MAXCOST = 3, /* (d, delay, hop, maxcost = largest arc length):
                             delay <= L, hop <= H, maxcost <= M (CSP=3)        */
  VINE_LABEL_QOS = 6      /* (d, bandwidth = smallest arc delay on the path,
                             21474836 at the source): bandwidth >= L          */
};

/* Solves nq queries of label kind `kind` on the GPU (host buffers) with the
 * variant engine: every label is checked against all stored labels of its
 * vertex under the kind's dominance, so any number of criteria is exact.
 * delay_limit[q] is L (the bandwidth floor for QoS); hop_limit[q] (H,
 * default 100 when NULL) and maxcost_limit[q] (M, default 10000 when NULL)
 * as in the reference's constraints.  The answer is the best feasible sink
 * label: lexicographically smallest (d, delay, hop, maxcost); for QoS the
 * smallest d, then the largest bandwidth.  out->cost / delay receive its d
 * and delay (QoS: bandwidth); extra[2q], extra[2q+1] (may be NULL) its hop
 * count and maxcost.  Paths as in vine_solve; Pareto outputs are not
 * filled.  cfg: bucket_width, block_threads (default 256), max_workers,
 * pool_labels, far_capacity, wait_limit, time_limit_ms are used.
 * Replaces cspp<c_label,c_edge>::solve for a reference built with CSP=2, 3
 * or the QoS label (algorithm/cspp.hpp:48-53). */
int vine_solve_labels(vine_graph *g, int32_t kind, int32_t nq, const int32_t *src,
                      const int32_t *dst, const float *delay_limit, const float *hop_limit,
                      const float *maxcost_limit, const vine_config *cfg, vine_results *out,
                      float *extra);

/* Multi-core CPU engine (host arrays only, no device): the reference's
 * OpenMP solver RUN_CSPP_OMP (algorithm/cspp_cpu.hpp:127-213), behind
 * cspp::solve_omp / solve_cpu (algorithm/cspp.hpp:55-61), with its data
 * races removed: each round expands the frontier in parallel, then every
 * vertex's dominance list is updated by the one thread that owns the vertex.
 * It is a separate, explicitly chosen solver; the GPU entry points never
 * fall back to it.  Fills cost / delay / found / status, and when given the
 * packed paths (path_offsets[nq+1], path, path_capacity) and the sink Pareto
 * sets (pareto_d / pareto_delay / pareto_n / pareto_stride) of out.
 * nthreads 0 = all cores; across_queries = 0 runs the queries one after the
 * other, each expanded by all threads (as the reference does); 1 gives each
 * thread its own queries.  Same answers either way and for every nthreads.
 * A query that would hold more labels than a cap (a quarter of physical
 * memory shared by the queries in flight, about 96 bytes a label; the
 * environment variable VINE_HOST_MAX_LABELS, read per call, overrides it)
 * stops with status VINE_ERR_CAPACITY and no answer; the others finish. */
int vine_solve_host(int32_t n, int64_t m, const int64_t *row_ptr, const int32_t *col,
                    const float *len, const float *delay, int32_t nq, const int32_t *src,
                    const int32_t *dst, const float *budget, int32_t nthreads,
                    int32_t across_queries, vine_results *out);

/* ------------------------------------------------------- learned scheduler */

#define VINE_MLP_IN 16
#define VINE_MLP_HIDDEN 64
#define VINE_MLP_OUT 2
/* Number of FP32 parameters: W1[64x16] b1[64] W2[64x64] b2[64] W3[2x64] b3[2]. */
#define VINE_MLP_PARAMS (64 * 16 + 64 + 64 * 64 + 64 + 2 * 64 + 2)

/* Creates a model on `device` with parameters initialised from `seed`
 * (or copied from `params` when not NULL). */
int vine_mlp_create(int32_t device, uint64_t seed, const float *params, vine_mlp **out);
void vine_mlp_destroy(vine_mlp *m);
int vine_mlp_get_params(const vine_mlp *m, float *params);
int vine_mlp_set_params(vine_mlp *m, const float *params);
/* y[n x 2] = MLP(x[n x 16]) on the GPU (host buffers). */
int vine_mlp_forward(const vine_mlp *m, int32_t n, const float *x, float *y);
/* Mean squared error over n rows and its gradient w.r.t. every parameter,
 * computed by the GPU forward + backward kernels (host buffers). */
int vine_mlp_loss_grad(const vine_mlp *m, int32_t n, const float *x, const float *y_target,
                       float *loss, float *grad);
/* No-allocation variant of vine_mlp_loss_grad (this entry point has no
 * counterpart in the reference, which has no learned scheduler).  Same
 * arguments and results, plus `stream` (a cudaStream_t; NULL = the legacy
 * default stream): the inputs are staged into a fixed device scratch area
 * that is part of the library image, the forward + backward kernel runs on
 * `stream`, and the call waits for that stream only.  It makes no device
 * allocation and frees nothing.  It exists for callers that must not
 * allocate: a loop that refines the scheduler while a batch solve is running
 * on another stream (cudaFree waits for all work on the device, which would
 * stall it behind a persistent kernel that runs for seconds), and processes
 * whose HBM is already handed to the label arena.
 * Limits: 1 <= n <= VINE_MLP_NOALLOC_MAX_ROWS, else VINE_ERR_INVALID with the
 * limit in vine_last_error().  The scratch area is one per device and per
 * process: calls that overlap in time on the same device (other threads or
 * streams) race on it and must be serialised by the caller.  The first call
 * on each device looks the scratch address up (cudaGetSymbolAddress); make
 * that first call before any stream capture begins.  The gradient and loss
 * accumulators in the scratch area are zeroed by every call on `stream`
 * before the kernel, so nothing has to start at zero on the caller's side. */
#define VINE_MLP_NOALLOC_MAX_ROWS 4096
int vine_mlp_loss_grad_noalloc(const vine_mlp *m, int32_t n, const float *x,
                               const float *y_target, float *loss, float *grad, void *stream);
/* `epochs` passes of mini-batch Adam over (x, y_target) on the GPU; returns
 * the final mean loss.  Mini-batches are drawn in a seeded order. */
int vine_mlp_train(vine_mlp *m, int32_t n, const float *x, const float *y_target,
                   int32_t epochs, int32_t batch, float lr, uint64_t seed, float *final_loss);

/* Scheduler traces recorded by the last vine_solve on `g` with cfg.trace=1:
 * one row per processed bucket.  Each row has VINE_TRACE_COLS floats:
 * [0..15] the 16 scheduler features, [16] query index, [17] bucket width
 * used, [18] labels expanded in the bucket, [19] rounds in the bucket. */
#define VINE_TRACE_COLS 20
int vine_trace_fetch(vine_graph *g, int64_t *rows, float *buf, int64_t capacity);

/* --------------------------------------------------------------- autotune */

/* Times candidate (block_threads, table_log2, bucket_width, split_threshold)
 * settings of the batch engine on the given sample of queries and writes the
 * fastest into *best (other fields copied from *base).  `cache_path` (may be
 * NULL) stores / reuses results keyed by a fingerprint of the graph. */
int vine_autotune(vine_graph *g, int32_t nq, const int32_t *src, const int32_t *dst,
                  const float *budget, const vine_config *base, const char *cache_path,
                  vine_config *best);

#ifdef __cplusplus
}
#endif

#endif /* VINE_H_ */
