/*
 * smx -- a B200-native subgraph-matching engine behind the filter / order /
 * explore plugin surface of Orrinn/SubgraphMatching (the reference).
 *
 * Plain C ABI: opaque handles, plain pointers and sizes, status codes.  Every
 * entry point names the reference interface it replaces (file:line within the
 * reference project).  Device memory is owned by the handles; every handle is
 * released by its smx_*_destroy.  One CUDA stream per data graph; calls on one
 * graph (and the candidate sets built from it) are not thread-safe, calls on
 * different graphs are.
 *
 * Counts follow the reference's semantics (explore.h:516-608): injective,
 * label-preserving, edge-preserving (non-induced) mappings of the query into
 * the data graph, every automorphic copy counted; a limit caps the count the
 * way output_limit does (explore.h:587-590), reported as min(count, limit).
 */
#ifndef SMX_H_
#define SMX_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SMX_MAX_QUERY_VERTEX 64 /* MAX_QUERY_VERTEX, common_type.h:29 */

typedef enum {
    SMX_OK = 0,
    SMX_EMPTY_CANDIDATES = 1, /* a filter left some query vertex without candidates (filter.h:87-89, :222-230) */
    SMX_INVALID_ORDER = 2,    /* order is not a permutation or has a vertex without an earlier neighbour (order.h:104-124, code_gen.h:743-746) */
    SMX_TOO_LARGE = 3,        /* query above SMX_MAX_QUERY_VERTEX, or a size above a stated maximum */
    SMX_TIMEOUT = 4,          /* the time budget ran out; the count is partial */
    SMX_CUDA_ERROR = 5,       /* a CUDA call failed; smx_last_error() has the message */
    SMX_BAD_ARGUMENT = 6,
    SMX_BAD_FORMAT = 7,       /* text graph does not parse or its degrees disagree with its edges */
    SMX_IO_ERROR = 8,
    SMX_STOPPED = 9,          /* the caller's stop word was set; the count is partial */
    SMX_NO_DEVICE = 10
} smx_status;

typedef struct smx_graph smx_graph; /* data graph resident in HBM (Graph, graph.h:51-380) */
typedef struct smx_query smx_query; /* query graph (Query, graph.h:382-495) */
typedef struct smx_cand smx_cand;   /* candidate sets + edge tables (CandidateParam, api.h:9-164) */

typedef enum { SMX_FILTER_NLF = 0, SMX_FILTER_GQL = 1 } smx_filter_kind;

typedef enum {
    /* explore_Intersection_Recursive<CandidatesBuffer> (explore.h:613-670):
     * candidates come from edge-table rows intersected per backward neighbour. */
    SMX_EXPLORE_CANDIDATES = 0,
    /* explore_Intersection_Cache_DAF_Filter (explore.h:1073-1129): raw
     * adjacency prefix intersections reused across depths (PlanIR,
     * code_gen.h:682-847), filter applied as a membership test, DAF
     * failing-set pruning (prune.h:82-171). */
    SMX_EXPLORE_CACHE_DAF = 1
} smx_explore_kind;

/* Enumeration options.  smx_enum_opts_default() fills defaults. */
typedef struct {
    int32_t explore;          /* smx_explore_kind */
    int32_t warps_per_block;  /* 0 = auto (8) */
    int32_t blocks_per_sm;    /* 0 = auto (occupancy); >= 3 also selects a build capped at 80 registers */
    int32_t task_grab;        /* tasks a warp takes per queue access; 0 = auto */
    int32_t stage_chunk;      /* elements per warp staged in shared memory for merge intersection */
    int32_t gallop_ratio;     /* long/short length ratio above which binary-search (galloping) intersection is used */
    int32_t bitmap_min;       /* candidate-table mode: |G| (the last depth's list without the row of depth n-2)
                                 from which G is marked in a bitmap that lanes probe; 0 = auto (32), -1 = never */
    int32_t use_tma;          /* stage rows with cp.async.bulk (1) or plain loads (0) */
    int32_t failing_sets;     /* DAF failing-set pruning in SMX_EXPLORE_CACHE_DAF (1 = on) */
    int32_t lane_depth;       /* candidate-table mode: depth (>= 2) from which each lane enumerates a
                                 subtree of its own; 0 = off (default), -1 = chosen from the query */
    double time_budget_ms;    /* 0 = unlimited; on expiry SMX_TIMEOUT with a partial count */
    int32_t budget_per_query; /* smx_enumerate_batch: 1 = the budget applies to each query from its first
                                 task (per-query status SMX_TIMEOUT), 0 = to the whole launch */
    int32_t reserved0;
} smx_enum_opts;

/* Per-call statistics (the reference's Profiler counters, common_type.h:185-189,
 * plus device work counters). */
typedef struct {
    uint64_t count;           /* min(embeddings, limit) */
    uint64_t raw_count;       /* embeddings counted before the limit stopped the search */
    uint64_t intersections;   /* set intersections performed (Profiler::total_intersection) */
    uint64_t nodes;           /* search-tree extensions (sum of total_iter_count) */
    uint64_t bytes;           /* algorithmic bytes read by the enumerator (list elements touched * 4 + row/candidate reads) */
    uint64_t pruned;          /* sibling subtrees skipped by failing sets (Profiler::daf_fp.cnt) */
    uint64_t tasks;           /* work items executed */
    double kernel_ms;         /* device time of the enumeration launch(es) */
    int32_t limit_reached;
    int32_t status;           /* smx_status of the device run */
} smx_stats;

/* ------------------------------------------------------------ errors */
const char* smx_status_str(int status);
const char* smx_last_error(void); /* thread-local message of the last failing call */
int smx_device_count(void);

/* Device-time markers on the graph's stream (CUDA events): begin records,
 * end records, waits and returns the elapsed device time in ms. */
int smx_mark_begin(smx_graph* g);
int smx_mark_end(smx_graph* g, double* ms);
/* Number of kernels this library has launched in the process so far. */
uint64_t smx_launch_count(void);

/* ------------------------------------------------------------ data graph */
/* Graph from a host CSR (rows strictly ascending, no self loops).
 * Replaces Graph::Load's in-memory result (graph.h:190-266). labels may be NULL (all 0).
 * device < 0 keeps the graph on the host only (I/O and generation without a GPU). */
int smx_graph_create(const uint64_t* offsets, const uint32_t* neighbors, const uint32_t* labels,
                     uint32_t num_vertices, uint64_t num_directed_edges, int device, smx_graph** out);
/* Graph::Load (graph.h:190-266): reference text format "t N M" / "v id label deg" / "e u v". */
int smx_graph_load_text(const char* path, int device, smx_graph** out);
/* Seeded Chung-Lu power-law graph: n vertices, m undirected edges (exact, no loops or
 * duplicates), degree exponent gamma; num_labels > 1 draws labels Zipf(zipf_s). */
int smx_graph_generate(uint32_t n, uint64_t m, double gamma, uint32_t num_labels, double zipf_s,
                       uint64_t seed, int device, smx_graph** out);
int smx_graph_info(const smx_graph* g, uint32_t* num_vertices, uint64_t* num_directed_edges,
                   uint32_t* max_degree, uint32_t* label_count);
/* Copy the host CSR out (offsets n+1, neighbors 2m, labels n); any pointer may be NULL. */
int smx_graph_export(const smx_graph* g, uint64_t* offsets, uint32_t* neighbors, uint32_t* labels);
int smx_graph_save_text(const smx_graph* g, const char* path);
void smx_graph_destroy(smx_graph* g);

/* ------------------------------------------------------------ query graph */
/* Query from a host CSR (Query, graph.h:382-495; at most SMX_MAX_QUERY_VERTEX vertices). */
int smx_query_create(const uint32_t* offsets, const uint32_t* neighbors, const uint32_t* labels,
                     uint32_t num_vertices, smx_query** out);
/* Query::Load (graph.h:474-478). */
int smx_query_load_text(const char* path, smx_query** out);
/* Seeded query of num_vertices vertices taken from the data graph, labels inherited.
 * dense == 0: a random walk's vertices with only the edges the walk traversed;
 * dense != 0: a randomized greedy-densest growth from a seeded start, induced subgraph
 * (retried until the average degree exceeds 3, else the densest attempt). */
int smx_query_generate(const smx_graph* g, uint32_t num_vertices, int dense, uint64_t seed, smx_query** out);
int smx_query_info(const smx_query* q, uint32_t* num_vertices, uint32_t* num_edges, uint32_t* max_degree);
int smx_query_export(const smx_query* q, uint32_t* offsets, uint32_t* neighbors, uint32_t* labels);
/* Query::getKCoreValue (graph.h:491) for every vertex. */
int smx_query_kcore(const smx_query* q, uint32_t* core);
int smx_query_save_text(const smx_query* q, const char* path);
void smx_query_destroy(smx_query* q);

/* ------------------------------------------------------------ orders (host) */
/* Order_RI (order.h:1138-1281). */
int smx_order_ri(const smx_query* q, uint32_t* order);
/* Order_GQL (order.h:563-597), from the candidate counts of c. */
int smx_order_gql(const smx_query* q, const smx_cand* c, uint32_t* order);
/* isValid (order.h:104-124) plus a permutation check: 1 valid, 0 not. */
int smx_order_valid(const smx_query* q, const uint32_t* order);

/* ------------------------------------------------------------ filtering (device) */
/* Filter_NLF / Filter_GQL (filter.h:1049-1063) including FilterParamConstruct
 * (filter.h:60-78): sorted candidate sets and the candidate-edge tables of
 * buildTables (table.h:7-139).  With build_tables == 0 the tables are skipped
 * (SMX_EXPLORE_CACHE_DAF needs none).  Returns SMX_EMPTY_CANDIDATES (with *out
 * still set) where the reference filter returns false. */
int smx_filter(smx_graph* g, const smx_query* q, int kind, int build_tables, smx_cand** out);
/* candidates_count[u] for every query vertex (api.h:12). */
int smx_cand_counts(const smx_cand* c, uint32_t* counts);
/* candidates[u] (api.h:11), ascending vertex ids; out holds counts[u] entries. */
int smx_cand_export(const smx_cand* c, uint32_t u, uint32_t* out);
/* edge_matrix[a][b] (api.h:13, graph.h:13-49): returns SMX_BAD_ARGUMENT if (a, b)
 * has no table.  offsets has v_cnt+1 entries, edge / edge_v e_cnt. */
int smx_table_info(const smx_cand* c, uint32_t a, uint32_t b, uint32_t* v_cnt, uint32_t* e_cnt, uint32_t* max_degree);
int smx_table_export(const smx_cand* c, uint32_t a, uint32_t b, uint32_t* offsets, uint32_t* edge, uint32_t* edge_v);
/* Device time of the last smx_filter stages, ms: [0] NLF, [1] GQL rounds, [2] compaction, [3] tables. */
int smx_cand_timing(const smx_cand* c, double* ms4);
void smx_cand_destroy(smx_cand* c);

/* ------------------------------------------------------------ enumeration (device) */
void smx_enum_opts_default(smx_enum_opts* o);
/* explore_* (explore.h:613, :1073): count embeddings along `order` (NULL = RI order).
 * limit 0 = unlimited.  stop (may be NULL; host memory registered or allocated as
 * mapped) is polled by the device; setting it non-zero ends the run with SMX_STOPPED. */
int smx_enumerate(smx_graph* g, const smx_query* q, const smx_cand* c, const uint32_t* order,
                  const smx_enum_opts* opts, uint64_t limit, volatile uint32_t* stop, smx_stats* out);

/* Stop word for smx_enumerate: pinned, device-mapped host memory holding one
 * uint32 (initially 0); the counterpart of the reference's
 * std::atomic<bool> stop_flag (explore.h:600-602).  Another host thread sets
 * *flag = 1 to end a running enumeration with SMX_STOPPED. */
int smx_stop_flag_create(int device, volatile uint32_t** flag);
void smx_stop_flag_destroy(volatile uint32_t* flag);

/* ------------------------------------------------------------ batched enumeration */
/* Many queries against one data graph in one persistent work-stealing launch,
 * captured in a CUDA graph and replayed.  orders may be NULL (RI) or hold nq
 * pointers (NULL entries = RI).  counts[nq] out (min(count, limit) each); stats
 * aggregate; query_status[nq] (may be NULL) out: SMX_OK or SMX_TIMEOUT per query. */
int smx_enumerate_batch(smx_graph* g, const smx_query* const* qs, const smx_cand* const* cs,
                        const uint32_t* const* orders, uint32_t nq, const smx_enum_opts* opts,
                        uint64_t limit, uint64_t* counts, smx_stats* out, int32_t* query_status);

/* ------------------------------------------------------------ learned matching order */
/* No counterpart in the reference (its orders are rule-based, order.h:1138-1281,
 * or analytic cost models, order.h:1391-1645).  A 64-256-256-1 MLP (ReLU, BF16
 * weights and activations, FP32 accumulation; Adam on FP32 master weights)
 * predicts the enumeration work of a (query, order) pair from
 * smx_order_features; smx_order_learned picks the order of a beam with the
 * smallest prediction.  An order never changes a count, only the work. */
#define SMX_MLP_INPUTS 64
#define SMX_MLP_HIDDEN 256
/* parameters, fp32: W1[256][64] b1[256] W2[256][256] b2[256] W3[256] b3[1] */
#define SMX_MLP_PARAMS 82689
typedef struct smx_mlp smx_mlp;
size_t smx_mlp_param_count(void);
/* He-normal weights from `seed`; batches of 1..max_batch rows. */
int smx_mlp_create(int device, uint32_t max_batch, uint64_t seed, smx_mlp** out);
int smx_mlp_set_params(smx_mlp* m, const float* params, size_t n); /* also resets the Adam state */
int smx_mlp_get_params(const smx_mlp* m, float* params, size_t n);
/* y[i] = model(x[i]) for n rows of SMX_MLP_INPUTS floats (host buffers). */
int smx_mlp_forward(smx_mlp* m, const float* x, uint32_t n, float* y);
/* Gradients of sum_i (y_i - t_i)^2 / (2n) in the parameter layout, and that loss; no update. */
int smx_mlp_gradients(smx_mlp* m, const float* x, const float* t, uint32_t n, float* grads, float* loss);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on that loss; *loss = loss before the step. */
int smx_mlp_train_step(smx_mlp* m, const float* x, const float* t, uint32_t n, float lr, float* loss);
void smx_mlp_destroy(smx_mlp* m);
/* The model's 64 inputs for `order` (valid order of q; candidate counts from c). */
int smx_order_features(const smx_query* q, const smx_cand* c, const uint32_t* order, float* out);
/* Up to `beam` distinct valid orders into orders[beam][n]: RI, GQL, then seeded
 * randomized greedy orders; *produced = how many. */
int smx_order_beam(const smx_query* q, const smx_cand* c, uint32_t beam, uint64_t seed, uint32_t* orders,
                   uint32_t* produced);
/* The beam order with the smallest predicted work (beam <= the model's max_batch). */
int smx_order_learned(smx_mlp* m, const smx_query* q, const smx_cand* c, uint32_t beam, uint64_t seed,
                      uint32_t* order, float* predicted);

/* ------------------------------------------------------------ enumeration without allocation */
/* No counterpart in the reference.  smx_enumerate allocates device memory on
 * every call (its plans, and scratch that grows with the query); some callers
 * cannot allow that -- a framework whose own caching allocator has already
 * reserved the GPU's memory, code that must not pay cudaMalloc's implicit
 * device synchronisation or risk its failure mid-run, or a service that has
 * to keep a fixed device footprint after start-up.  smx_enumerate_noalloc
 * counts like smx_enumerate (same arguments, same counts and statistics;
 * kernel_ms is host-timed) but calls no cudaMalloc/cudaFree or other
 * allocating routine: its control block, plan and per-warp scratch live in
 * one static device array of SMX_NOALLOC_SCRATCH_BYTES that every GPU loading
 * this library reserves until the process exits.  The caller still passes the
 * graph, query and candidate handles (made by the allocating calls above) and
 * receives the result in *out.
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) with that device current; make that first call
 *    before any stream capture on the graph's stream.
 *  - Every call shares the array, which keeps the last call's contents; each
 *    call clears what must start at zero.  Two calls whose GPU work overlapped
 *    would race on it, so calls are serialised by a process-wide lock and each
 *    waits for its own launch before returning.
 *  - It launches only as many warps as the array holds; a query whose one
 *    block of warps_per_block warps needs more than the array returns
 *    SMX_TOO_LARGE with the sizes in smx_last_error(). */
#define SMX_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)
int smx_enumerate_noalloc(smx_graph* g, const smx_query* q, const smx_cand* c, const uint32_t* order,
                          const smx_enum_opts* opts, uint64_t limit, volatile uint32_t* stop, smx_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* SMX_H_ */
