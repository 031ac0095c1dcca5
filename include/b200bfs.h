/*
 * b200bfs.h -- C ABI of the B200-native direction-optimizing BFS engine.
 *
 * The engine replaces the BFS hot path of Graph500-BFS, i.e. the member
 * surface of `class BfsBase` (mpi/bfs.hpp:48-172) that the benchmark driver
 * reaches through `typedef BfsBase BfsOnCPU` (mpi/bfs_cpu.hpp:13).  Each entry
 * point below names the reference interface it stands in for.  The 2D MPI
 * partition of the reference collapses to one device-resident CSR on one GPU.
 *
 * Conventions
 *  - Every function returns an int status: B200BFS_OK (0) or an error code;
 *    b200bfs_last_error() gives the message of the last failure on a handle.
 *    (The reference throws `const char*`, std::runtime_error or calls
 *    MPI_Abort; a C ABI cannot, so errors become status codes.)
 *  - Vertex ids are the ORIGINAL (scrambled) global ids of the generator.
 *  - pred entries follow the reference encoding
 *    `pred[v] = (uint64(level & 0xFFFF) << 48) | (parent & 0xFFFFFFFFFFFF)`,
 *    -1 for unreached vertices (mpi/validate.hpp:982-992); with CoreBFS,
 *    pruned tree vertices carry level 0xFFFF as in
 *    mpi/corebfs_adaptor.hpp:285-301.
 *  - Host pointers are plain host memory (pinned or pageable); device
 *    pointers are only used where the name says `_device`.
 *  - A handle is not thread-safe; calls on one handle come from one thread,
 *    as the reference driver calls BfsBase from its main thread only.
 */
#ifndef B200BFS_H_
#define B200BFS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------ status codes ----------------------------- */
enum {
  B200BFS_OK = 0,
  B200BFS_ERR_INVALID = 1,   /* bad argument (null pointer, range, size)    */
  B200BFS_ERR_CUDA = 2,      /* a CUDA call failed                          */
  B200BFS_ERR_OOM = 3,       /* device memory or the HBM budget exhausted   */
  B200BFS_ERR_STATE = 4,     /* call out of order (e.g. run before build)   */
  B200BFS_ERR_TIMEOUT = 5,   /* a bounded device wait gave up               */
  B200BFS_ERR_OVERFLOW = 6,  /* more than 0xFFFE levels, or > 32 prunings   */
  B200BFS_ERR_NOT_FOUND = 7  /* unknown graph / request id                  */
};

/* ------------------------------ build flags ------------------------------ */
enum {
  /* CoreBFS forest pruning (main.cc -C; bfs.hpp:116-139). */
  B200BFS_BUILD_COREBFS = 1 << 0,
  /* Degree-ordered reordering within groups of 2^16 original ids
   * (SMALL_REORDER_BIT, graph_constructor.hpp:594-732) instead of one global
   * degree order (VERTEX_REORDERING=2, :632-637). */
  B200BFS_BUILD_GROUP_REORDER = 1 << 1,
  /* The edge list given is already symmetric (each undirected edge present
   * in both directions, as the sym_edge_list passed to BfsBase::construct);
   * without this flag every edge is mirrored, as make_symmetry_edge_list
   * (benchmark_helper.hpp:383-497) does. */
  B200BFS_BUILD_INPUT_SYMMETRIC = 1 << 2
};

typedef struct b200bfs_handle b200bfs_handle;

typedef struct b200bfs_config {
  int device;                 /* CUDA device ordinal                          */
  int reserved;               /* must be 0                                    */
  uint64_t hbm_budget_bytes;  /* 0: no limit besides the device's memory      */
} b200bfs_config;

/* Graph facts the driver reads from `benchmark->graph_`
 * (main.cc:441, 693; benchmark_helper.hpp:532-533, 567-573). */
typedef struct b200bfs_graph_info {
  int32_t scale;                 /* estimated SCALE, log_orig_global_verts_   */
  int32_t reorder_bits;          /* reorder_bits_ (16 with group reorder)     */
  int64_t pred_size;             /* pred_size(): length of pred[]             */
  int64_t num_global_edges;      /* directed entries after de-duplication     */
  int64_t num_global_verts;      /* vertices with at least one edge           */
  int64_t num_rows;              /* rows of the device CSR                    */
  int64_t num_input_edges;       /* edges given to the builder                */
  int64_t device_bytes;          /* device memory held by the graph           */
  int32_t corebfs;               /* 1 when built with CoreBFS                 */
  int32_t prune_rounds;          /* CoreBFS pruning rounds                    */
  int64_t core_vertices;         /* 2-core vertices (CoreBFS)                 */
  int64_t tree_vertices;         /* pruned vertices that keep a parent        */
} b200bfs_graph_info;

/* Per-run statistics (the reference's VERVOSE_MODE counters,
 * bfs.hpp:3459-3526, and PROFILE_REGIONS TD/BU split, utils.hpp:3736-3755). */
typedef struct b200bfs_run_stats {
  int32_t levels;                /* last current_level_ (AUTO_LEVEL)         */
  int32_t num_td_levels;
  int32_t num_bu_levels;
  int32_t kernel_launches;       /* engine kernels launched by the run       */
  uint64_t bu_level_mask;        /* bit L: level L ran bottom-up (L < 64)    */
  int64_t visited;               /* vertices reached, root included          */
  int64_t edges_scanned_td;      /* adjacency entries read top-down          */
  int64_t edges_scanned_bu;      /* adjacency entries read bottom-up         */
  int64_t algorithmic_bytes;     /* bytes the search must move (roofline)    */
  int64_t td_bytes;              /* of which in top-down expansion kernels   */
  int64_t bu_bytes;              /* of which in bottom-up kernels            */
  double device_ms;              /* CUDA-event time of the whole run         */
  double td_ms;                  /* CUDA-event time of the top-down kernels  */
  double bu_ms;                  /* CUDA-event time of the bottom-up kernels */
  int64_t pred_bytes;            /* bytes of the pred assembly pass (0: none) */
  double pred_ms;                /* CUDA-event time of the pred assembly pass */
} b200bfs_run_stats;

/* One level of the last search (the per-level report of the reference's
 * VERVOSE_MODE, bfs.hpp:3459-3526). */
typedef struct b200bfs_level_stats {
  int32_t level;                 /* current_level_                           */
  int32_t bottom_up;             /* 1: bottom-up step, 0: top-down           */
  int64_t input;                 /* frontier rows (top-down) or unvisited rows (bottom-up) */
  int64_t discovered;            /* vertices found in the level (NQ)         */
  int64_t scanned;               /* adjacency entries read                   */
  int64_t algorithmic_bytes;
  double ms;                     /* CUDA-event time of the level's kernel    */
} b200bfs_level_stats;

/* Statistics of the last batched search (b200bfs_run_batch). */
typedef struct b200bfs_batch_stats {
  int32_t num_roots;             /* roots in the batch                        */
  int32_t levels;                /* last level of the deepest root            */
  int32_t num_td_levels;         /* levels with a top-down expansion          */
  int32_t num_bu_levels;         /* levels with a bottom-up sweep             */
  int32_t kernel_launches;
  int32_t reserved;
  int64_t edges_scanned_td;      /* adjacency entries read top-down           */
  int64_t edges_scanned_bu;      /* adjacency entries read bottom-up          */
  int64_t algorithmic_bytes;     /* bytes the batch must move (roofline)      */
  int64_t bu_bytes;              /* of which in the bottom-up kernel          */
  double ms;                     /* CUDA-event time of the whole batch        */
  double bu_ms;                  /* CUDA-event time of the bottom-up kernels  */
  double td_ms;                  /* CUDA-event time of the top-down parts     */
} b200bfs_batch_stats;

/* --------------------------- lifetime / errors --------------------------- */

/* Replaces `new BfsOnCPU()` (main.cc:433). */
int b200bfs_create(const b200bfs_config* config, b200bfs_handle** out);
/* Replaces `delete benchmark` (main.cc:711) and frees every device buffer. */
int b200bfs_destroy(b200bfs_handle* h);
/* Message of the last failed call on h (never NULL). */
const char* b200bfs_last_error(const b200bfs_handle* h);
/* Replaces BfsBase::printInformation (main.cc:410): writes a one-line
 * description of the engine and device into buf. */
int b200bfs_print_information(b200bfs_handle* h, char* buf, size_t len);

/* -------------------------------- graph ---------------------------------- */

/* Replaces BfsBase::construct(scale, corebfs_enabled, sym_edge_list)
 * (bfs.hpp:116-139) together with make_symmetry_edge_list when the input is
 * not symmetric.  `edges` holds nedges (v0, v1) pairs of int64 in host memory.
 * scale is the SCALE of the id space (0: estimate it from the ids, as
 * make_symmetry_edge_list does).  flags: B200BFS_BUILD_*. */
int b200bfs_build_from_edges(b200bfs_handle* h, const int64_t* edges,
                             int64_t nedges, int scale, int flags);

/* Same, for the reference's 12-byte UnweightedPackedEdge records
 * (mpi/primitives.hpp:54-86: v0_low, v1_low, high = v0>>32 | (v1>>32)<<16),
 * i.e. the EdgeListStorage<UnweightedPackedEdge> chunks main.cc holds. */
int b200bfs_build_from_packed(b200bfs_handle* h, const uint32_t* packed,
                              int64_t nedges, int scale, int flags);

/* Replaces generate_graph_spec2010 + make_symmetry_edge_list + construct
 * (main.cc:412-435): the Kronecker edges of RmatGraphGenerator<...,5700,1900>
 * (generator/graph_generator.hpp:781-892) with user seeds (seed1, seed2)
 * are generated on the device in chunks and streamed into the CSR, so no
 * host edge list exists (needed at SCALE 28). */
int b200bfs_generate_graph(b200bfs_handle* h, int scale, int edgefactor,
                           uint64_t seed1, uint64_t seed2, int flags);

/* Copies edges [start, end) of the device generator (same generator and
 * seeds as b200bfs_generate_graph) into host memory as int64 pairs; used to
 * check the generator against the reference and to feed the validator. */
int b200bfs_generate_edges(b200bfs_handle* h, int scale, uint64_t seed1,
                           uint64_t seed2, int64_t start, int64_t end,
                           int64_t* edges_out);

int b200bfs_graph_info_get(b200bfs_handle* h, b200bfs_graph_info* out);

/* Copies the searched CSR (the 2-core with CoreBFS) to host memory:
 * row_ptr[num_rows + 1], col[num_global_edges] (row ids), inv[num_rows]
 * (row -> original id) and mdeg[num_rows] (pre-dedup degree, the
 * reference's degree_).  Any output pointer may be NULL.  The counterpart of
 * reading Graph2DCSR's arrays (graph_constructor.hpp:291-332). */
int b200bfs_get_csr(b200bfs_handle* h, int64_t* row_ptr, int32_t* col, int32_t* inv,
                    int32_t* mdeg);

/* Replaces BfsBase::has_edge (bfs.hpp:167-170). */
int b200bfs_has_edge(b200bfs_handle* h, int64_t v, int* out);
/* has_edge for every vertex at once: out[pred_size] (0/1). */
int b200bfs_has_edge_all(b200bfs_handle* h, uint8_t* out);

/* find_roots (mpi/benchmark_helper.hpp:527-562): the driver's search-key
 * sampler with user seeds (2 + r1, 3 + r2) over has_edge; writes num_roots
 * vertex ids.  main.cc calls it with r1 = root seed (+1 per re-pick), r2 = 0. */
int b200bfs_find_roots(b200bfs_handle* h, int num_roots, int r1, int r2, int64_t* roots);

/* --------------------------------- BFS ----------------------------------- */

/* Replaces BfsBase::prepare_bfs (bfs.hpp:141-151): allocates the search
 * buffers; with CoreBFS also resets unreachable tree parents
 * (corebfs_adaptor.hpp:228-249). */
int b200bfs_prepare(b200bfs_handle* h, int edgefactor, double alpha,
                    double beta);

/* Replaces BfsBase::run_bfs (bfs.hpp:3214-3232) including
 * initialize_memory, the level loop with the alpha/beta direction switch
 * (bfs.hpp:3413-3457) and the CoreBFS tree climb and fill-in.  pred stays on
 * the device until b200bfs_get_pred.  auto_tuning_data (host, 9 int64 slots,
 * parameters.h:260-270) receives the slots run_bfs writes; may be NULL.
 * Blocks until the search is complete. */
int b200bfs_run(b200bfs_handle* h, int64_t root, int edgefactor, double alpha,
                double beta, int64_t* auto_tuning_data);

/* The driver's -A mode, auto_tuning of mpi/main.cc:361-391: searches every
 * root, then moves alpha and afterwards beta one switch level at a time while
 * the moved root gets faster (auto_tuning_each, main.cc:45-311).  nedge[i] is
 * the TEPS numerator of roots[i] (the reference uses pf_nedge[SCALE]).
 * *alpha and *beta are read and tuned in place; *teps (may be NULL) receives
 * the harmonic-mean TEPS of the final measurement.  Search times are
 * CUDA-event times of the engine's stream. */
int b200bfs_auto_tune(b200bfs_handle* h, const int64_t* roots, int num_roots,
                      const double* nedge, int edgefactor, double* alpha, double* beta,
                      double* teps);

/* Replaces BfsBase::get_pred (bfs.hpp:161-163): copies pred[pred_size] of the
 * last run to host memory. */
int b200bfs_get_pred(b200bfs_handle* h, int64_t* pred);

/* Exact per-vertex BFS level of the last run (-1 if unreached), with the
 * levels of CoreBFS tree vertices filled in: levels[pred_size]. */
int b200bfs_get_levels(b200bfs_handle* h, int32_t* levels);

/* Per-level records of the last run or batch (a batch level with both a
 * top-down and a bottom-up part gives two records; there `discovered` is the
 * number of roots in that part): up to max entries into out, the number of
 * records in *count. */
int b200bfs_get_level_stats(b200bfs_handle* h, b200bfs_level_stats* out, int max, int* count);

/* Statistics of the last run. */
int b200bfs_get_run_stats(b200bfs_handle* h, b200bfs_run_stats* out);

/* ------------------------------ engine tuner ------------------------------ */

enum {
  B200BFS_TUNE_FORMS = 1 << 0,        /* bottom-up and top-down kernel forms   */
  B200BFS_TUNE_BATCH_ALPHA = 1 << 1,  /* alpha of b200bfs_run_batch            */
  B200BFS_TUNE_SWITCH = 1 << 2        /* single-source alpha/beta, refined     */
};

typedef struct b200bfs_tune_report {
  int32_t bu_kernel;             /* chosen "bu_kernel" option                 */
  int32_t td_kernel;             /* chosen "td_kernel" option                 */
  double batch_alpha;            /* chosen "batch_alpha" option               */
  double single_ms;              /* mean search time with the chosen forms    */
  double batch_ms;               /* batch time with the chosen alpha          */
  int32_t searches;              /* single-source searches the tuner ran      */
  int32_t batches;               /* batches the tuner ran                     */
  double alpha, beta;            /* single-source switch parameters: refined
                                    with B200BFS_TUNE_SWITCH, else the input   */
} b200bfs_tune_report;

/* No counterpart in the reference, whose equivalents are compile-time
 * constants of parameters.h: picks, for the resident graph, the bottom-up
 * and top-down kernel forms (timing each on up to 16 of the roots with
 * alpha/beta) and the batched search's alpha (timing 64-root batches with
 * 10..400), and keeps the fastest in the engine's options ("bu_kernel",
 * "td_kernel", "batch_alpha").  With B200BFS_TUNE_SWITCH it also refines
 * the given alpha/beta (for instance the -A tuner's) by timing the same
 * searches with each scaled by 0.5, 0.7, 1.4 and 2, one after the other,
 * keeping a change only when it is more than 1 % faster; the result is
 * returned in out->alpha / out->beta for the caller to pass to b200bfs_run.
 * what: B200BFS_TUNE_* bits.  Levels and parent validity do not depend on
 * the choices.  out may be NULL. */
int b200bfs_tune_engine(b200bfs_handle* h, const int64_t* roots, int num_roots, int edgefactor,
                        double alpha, double beta, int what, b200bfs_tune_report* out);

/* Engine tuning knobs (no counterpart in the reference, whose equivalents
 * are compile-time constants of parameters.h): "bu_kernel" (1..4, bottom-up
 * kernel form), "td_kernel" (1..7, top-down kernel form; 4 and 7 pick per
 * level), "bu_probe" (1..64, neighbours probed per lane by bottom-up form
 * 1), "bu_first" (1: bottom-up forms 2-4 probe the first neighbour from a
 * dense per-row array first, the default), "bu_sparse" (1: on levels with
 * few unvisited rows bottom-up forms 2-4 skip full bitmap words 32 at a time,
 * the default; 0: every word steps through the row search), "bu_spec" (1: on
 * levels where more than half of the rows are unvisited bottom-up forms 2-4
 * load every row's first-neighbour entry beside its bitmap word, the
 * default; 0: only the unvisited rows' entries, after the word), "td_unroll" (1, 2 or 4: 32-entry
 * steps a lane of top-down form 5 handles together), "pred_assemble" (1:
 * the levels write a row-order buffer and one pass over the original ids
 * writes pred, the default; after a search of this kind the pass leaves out
 * the ids whose entries cannot change (no edge, or a CoreBFS tree vertex off
 * both climbs); 0: the levels write pred by original id),
 * "force_direction" (0 = alpha/beta rule, 1 = top-down only, 2 = bottom-up
 * from level 2),
 * "single_graph" (1: b200bfs_run runs its level loop as a CUDA graph on the
 * device, one host synchronisation per search, with bottom-up form 4 and
 * top-down forms 1, 3, 4 or 5; per-level kernel times are then not
 * recorded; 0: host loop, the default),
 * "batch_graph" (1: b200bfs_run_batch runs its level loop as a CUDA graph on
 * the device, 0: the host launches each level and per-level times are
 * recorded), "batch_alpha" (the alpha b200bfs_run_batch uses when given
 * alpha <= 0; default 30), "batch_probe" (4, 8, 16, 32, 64, 128, 256 or
 * 1024: neighbours a lane of the batched bottom-up sweep probes before the
 * warp sweeps its row; default 128) and "batch_round" (4 or 8: of them
 * loaded together; default 4).  None of them changes levels or the validity
 * of parents. */
int b200bfs_set_option(b200bfs_handle* h, const char* name, int64_t value);

/* The CUDA stream (a cudaStream_t) the engine launches its kernels on, for
 * callers that time or order work around b200bfs_run with CUDA events. */
int b200bfs_get_stream(b200bfs_handle* h, void** stream);

/* Replaces BfsBase::end_bfs (bfs.hpp:165): frees the search buffers. */
int b200bfs_end(b200bfs_handle* h);

/* Graph500 validation of the last run on the device, following
 * BfsValidation::validate (validate.hpp:607-976) against the graph's input
 * edges (the device generator's edges for b200bfs_generate_graph).  Returns
 * the error count in *errors and the traversed input-edge count (the TEPS
 * numerator) in *edge_visit_count. */
int b200bfs_validate(b200bfs_handle* h, int64_t root, int64_t* errors,
                     int64_t* edge_visit_count);

/* Replaces validate_bfs_result (validate.hpp:1269-1277, called by main.cc:647)
 * for a pred the caller holds: the same Graph500 rules as b200bfs_validate,
 * applied to pred[pred_size] (host or device memory, read only) from root
 * against the graph's resident input edges.  corebfs != 0 selects the
 * CoreBFS mode of the reference (tree entries with level 0xFFFF, depths
 * rebuilt from parents).  Needs a built graph, not a search; *errors is 0
 * for a valid pred. */
int b200bfs_validate_pred(b200bfs_handle* h, int64_t root, const int64_t* pred, int corebfs,
                          int64_t* errors, int64_t* edge_visit_count);

/* ---------------------------- batched search ------------------------------ */

#define B200BFS_BATCH_MAX 64

/* No single counterpart in the reference, which runs one root per run_bfs
 * call (main.cc:610-640); this is that loop over roots done in one
 * traversal.  Searches from roots[0..num_roots), 1 <= num_roots <= 64, in
 * one multi-source traversal: every vertex carries a 64-bit mask of the roots
 * that reached it, so one read of an adjacency row serves all roots.  Each
 * root switches between top-down and bottom-up on its own, with the rule of
 * bfs.hpp:3413-3457 applied to that root's frontier (alpha <= 0 selects the
 * engine's "batch_alpha" option, default 30; beta as for b200bfs_run).  Per-root levels equal those
 * of b200bfs_run from the same root.  Requires b200bfs_prepare; with CoreBFS
 * each root climbs to the 2-core first, as b200bfs_run does.  stats may be
 * NULL. */
int b200bfs_run_batch(b200bfs_handle* h, const int64_t* roots, int num_roots, int edgefactor,
                      double alpha, double beta, b200bfs_batch_stats* stats);

/* auto_tuning_data[AUTO_LEVEL] of every root of the last batch, as
 * b200bfs_run would leave it for that root alone: the first level at which
 * the root's frontier is empty (its deepest level + 1; 0 for a root outside
 * the searched graph).  The quantity find_roots_in_large_graph
 * (main.cc:334-359) tests against REMOVE_ROOTS_LEVEL_THED, for all roots of
 * one batch at once.  auto_level[num_roots] (host). */
int b200bfs_batch_root_levels(b200bfs_handle* h, int64_t* auto_level);

/* Makes root `index` of the last batch the engine's current result: pred is
 * rebuilt on the device from the batch's levels (parent = a neighbour one
 * level nearer the root, a valid BFS parent), so b200bfs_get_pred,
 * b200bfs_get_levels and b200bfs_validate then report that root. */
int b200bfs_batch_select(b200bfs_handle* h, int index);

/* -------------------------------- serving --------------------------------- */

/* No counterpart in the reference (a batch benchmark).  A BFS server keeps
 * several graphs resident on one GPU and answers (graph, root) queries as
 * they arrive, with continuous batching: every graph has a few batch slots,
 * each served by its own worker thread and CUDA stream; a free slot takes up
 * to max_batch queued roots of its graph into one b200bfs_run_batch-style
 * traversal, so requests that arrive while other batches are on the GPU are
 * admitted as soon as a slot frees, and batches of different graphs (and of
 * one graph on different slots) overlap on the device.  Graphs and slots are
 * admitted against one HBM budget.  Each request's levels are those of a
 * single-source search from its root, whatever batch it was served in.
 * All server calls are thread-safe. */
typedef struct b200bfs_server b200bfs_server;

typedef struct b200bfs_server_config {
  int device;                 /* CUDA device ordinal                          */
  int max_batch;              /* roots per batch, 1..64 (0: 64)               */
  int slots_per_graph;        /* concurrent batches per graph (0: 2)          */
  int keep_results;           /* 1: a finished request keeps its levels on the
                                 device until b200bfs_server_release          */
  uint64_t hbm_budget_bytes;  /* graphs + slots together (0: device memory)   */
  double alpha;               /* batch switch alpha (<= 0: 30)                */
  double beta;                /* batch switch beta (<= 0: 14)                 */
} b200bfs_server_config;

enum {
  B200BFS_REQ_QUEUED = 0,
  B200BFS_REQ_RUNNING = 1,
  B200BFS_REQ_DONE = 2,
  B200BFS_REQ_FAILED = 3,
  B200BFS_REQ_CANCELLED = 4
};

typedef struct b200bfs_request_info {
  int32_t state;                 /* B200BFS_REQ_*                             */
  int32_t graph_id;
  int64_t root;
  int32_t depth;                 /* deepest level reached from the root       */
  int32_t batch_size;            /* roots in the batch that served it         */
  double latency_ms;             /* submit -> done, host clock                */
  double queue_ms;               /* submit -> start of its batch              */
} b200bfs_request_info;

typedef struct b200bfs_server_stats {
  int64_t submitted;
  int64_t completed;
  int64_t failed;
  int64_t batches;
  double mean_batch_size;
  double p50_ms;                 /* latency percentiles of completed requests */
  double p99_ms;
  double max_ms;
  double bfs_per_s;              /* completed / (last completion - first submit) */
  uint64_t device_bytes;         /* held by graphs and slots                  */
  int32_t graphs;
  int32_t slots;
} b200bfs_server_stats;

/* Starts a server (no graphs yet). */
int b200bfs_server_start(const b200bfs_server_config* config, b200bfs_server** out);
/* Generates and prepares a Graph500 graph on the device (as
 * b200bfs_generate_graph + b200bfs_prepare with edgefactor's switch
 * parameters) and makes it servable; B200BFS_ERR_OOM when it or its first
 * slot does not fit the budget.  *graph_id receives its id. */
int b200bfs_server_add_graph(b200bfs_server* srv, int scale, int edgefactor, uint64_t seed1,
                             uint64_t seed2, int flags, int* graph_id);
int b200bfs_server_graph_info(b200bfs_server* srv, int graph_id, b200bfs_graph_info* out);
/* Roots of a served graph drawn as b200bfs_find_roots does (uniform among
 * vertices with an edge), for load generators and tests. */
int b200bfs_server_find_roots(b200bfs_server* srv, int graph_id, int num_roots, int r1, int r2,
                              int64_t* roots);
/* Queues a query; returns at once with its id. */
int b200bfs_server_submit(b200bfs_server* srv, int graph_id, int64_t root, int64_t* request_id);
/* State of a request, without waiting. */
int b200bfs_server_poll(b200bfs_server* srv, int64_t request_id, b200bfs_request_info* info);
/* Waits up to timeout_s seconds for a request to finish;
 * B200BFS_ERR_TIMEOUT if it has not. */
int b200bfs_server_wait(b200bfs_server* srv, int64_t request_id, double timeout_s,
                        b200bfs_request_info* info);
/* Levels of a finished request (keep_results = 1), levels[pred_size] in
 * original vertex ids, -1 for unreached vertices. */
int b200bfs_server_get_levels(b200bfs_server* srv, int64_t request_id, int32_t* levels);
/* Forgets a request; a finished request's slot can then be reused. */
int b200bfs_server_release(b200bfs_server* srv, int64_t request_id);
int b200bfs_server_get_stats(b200bfs_server* srv, b200bfs_server_stats* out);
/* Restarts the latency and throughput statistics. */
int b200bfs_server_reset_stats(b200bfs_server* srv);
const char* b200bfs_server_last_error(const b200bfs_server* srv);
/* Stops the workers (queued requests are cancelled, running batches finish)
 * and frees every graph. */
int b200bfs_server_stop(b200bfs_server* srv);

/* ------------------------- allocation-free search ------------------------ */

/* Largest graph b200bfs_bfs_noalloc accepts (rows of the CSR). */
#define B200BFS_NOALLOC_MAX_ROWS (1 << 24)

/* No counterpart in the reference: an entry point for callers that may not
 * allocate device memory -- applications whose caching allocator owns the
 * device memory (a framework's pool that must not be bypassed) and hosts that
 * give the library a fixed memory budget at start-up.  It searches a CSR the
 * caller already holds on the device (row_ptr[nrows + 1] int64,
 * col[row_ptr[nrows]] int32 row ids, rows sorted or not) from `root` and
 * writes pred[nrows] (device memory, same encoding as pred above with row ids
 * as vertex ids, -1 unreached); *num_levels (host, may be NULL) receives the
 * last level, as AUTO_LEVEL.  The CSR must be symmetric (every edge stored
 * in both directions, as the engine's own CSR is): the search is bottom-up
 * only and takes any neighbour visited before a level as the parent, which
 * gives BFS levels only on an undirected graph.  Column ids outside
 * [0, nrows) are ignored.  stream is a cudaStream_t (NULL = legacy default
 * stream); the host reads a counter after every level, so the call
 * synchronises the stream once per level and returns once the search is
 * complete; a stream that is being captured is refused with
 * B200BFS_ERR_INVALID before anything is enqueued.
 * It allocates nothing: its scratch (two visited bitmaps and a counter) lives
 * in one fixed device array of B200BFS_NOALLOC_MAX_ROWS / 4 bytes that every
 * GPU loading the library keeps until exit.  Graphs with more rows are
 * rejected with B200BFS_ERR_INVALID.  The first call on a device looks up
 * that array's device address.  All calls share the array: calls that overlap
 * on the GPU (other threads or streams) race and must be serialised by the
 * caller. */
int b200bfs_bfs_noalloc(const int64_t* row_ptr, const int32_t* col, int64_t nrows,
                        int64_t root, int64_t* pred, void* stream, int32_t* num_levels);

/* ------------------------------ measurement ------------------------------ */

/* No counterpart in the reference (a measurement aid): the rate at which
 * this GPU's SMs issue independent random 4-byte accesses into `words`, a
 * caller-owned device buffer of 2^log2_words uint32 (10 <= log2_words <= 30;
 * its contents are overwritten when kind is 1): kind 0 loads, kind 1
 * non-returning ORs.  These are the accesses a top-down level is made of (a
 * visited-bitmap probe per adjacency entry, an OR per claim), so with a
 * buffer the size of the visited bitmap the result is the ceiling the
 * top-down kernels are measured against.  Enqueued on `stream` (a
 * cudaStream_t, NULL = legacy default stream) and synchronised; *per_s
 * receives accesses per second (the best of three launches after one
 * warm-up).  Allocates nothing. */
int b200bfs_random_access_rate(void* words, int log2_words, int kind, void* stream,
                               double* per_s);

#ifdef __cplusplus
}
#endif

#endif /* B200BFS_H_ */
