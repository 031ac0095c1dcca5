/*
 * CPU oracle for the direction-optimizing BFS hot path of Graph500-BFS.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path (the CUDA library
 * under graph500-bfs_b200/) links or calls this code; it is loaded by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and
 * only as the checker / the timed CPU restatement.
 *
 * Every function restates the reference's algorithm in plain C (OpenMP for
 * speed) and cites the reference file:line it follows.  Parity of this
 * restatement is pinned by
 *   - the reference's own known-answer table pf_nedge[SCALE]
 *     (mpi/utils.hpp:3687-3733), reproduced exactly by
 *     generate -> symmetrize -> BFS -> validate edge counting, and
 *   - golden edge / random-number vectors produced by the reference's own
 *     generator sources compiled unchanged (oracle/ref/, see tests/golden/).
 */
#ifndef B200BFS_ORACLE_H_
#define B200BFS_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- MRG (generator/splittable_mrg.{h,c}) ------------------ */

typedef struct orc_mrg_state {
  uint32_t z[5]; /* z[0] = z1 (most recent output) ... z[4] = z5 */
} orc_mrg_state;

/* generator/graph_generator.hpp:494-500 make_mrg_seed */
void orc_mrg_seed_from_user(uint64_t userseed1, uint64_t userseed2,
                            orc_mrg_state* st);
/* generator/splittable_mrg.c:324-327 mrg_get_uint_orig */
uint32_t orc_mrg_next(orc_mrg_state* st);
/* generator/splittable_mrg.c:330-337 mrg_get_double_orig */
double orc_mrg_next_double(orc_mrg_state* st);
/* generator/splittable_mrg.c:228-245 mrg_skip: advance by the 192-bit exponent
 * (hi, mid, lo). */
void orc_mrg_skip(orc_mrg_state* st, uint64_t hi, uint64_t mid, uint64_t lo);
/* The 5x5 transition matrix A^(2^k), row-major, k in [0, 192). */
void orc_mrg_pow2_matrix(int k, uint32_t out[25]);

/* generator/graph_generator.hpp:506-520 make_random_numbers */
void orc_make_random_numbers(int64_t nvalues, uint64_t userseed1,
                             uint64_t userseed2, int64_t position,
                             double* result);

/* -------------- Kronecker generator (graph_generator.hpp) --------------- */

/* Scramble constants of GraphGeneratorBase (graph_generator.hpp:541-551). */
void orc_scramble_values(uint64_t userseed1, uint64_t userseed2,
                         uint64_t* val0, uint64_t* val1);
/* graph_generator.hpp:625-637 scramble */
int64_t orc_scramble(int64_t v, int scale, uint64_t val0, uint64_t val1);

/* RmatGraphGenerator<...,5700,1900>::generateRange
 * (graph_generator.hpp:781-892): writes edges [start, end) as interleaved
 * (v0, v1) int64 pairs into out[2*(end-start)]. */
void orc_generate_edges(int scale, uint64_t userseed1, uint64_t userseed2,
                        int64_t start, int64_t end, int64_t* out);

/* ------------------------- graph (symmetric CSR) ------------------------- */

typedef struct orc_graph {
  int64_t nverts;      /* 2^scale */
  int scale;           /* estimated SCALE (benchmark_helper.hpp:488-494) */
  int64_t* row_ptr;    /* nverts + 1 */
  int64_t* col;        /* sorted, de-duplicated neighbours */
  int64_t* multideg;   /* pre-dedup symmetric degree (graph_constructor.hpp:572-592) */
  int64_t num_edges;   /* post-dedup directed entries (num_global_edges_) */
  int64_t num_verts;   /* vertices with >= 1 edge (num_global_verts_) */
} orc_graph;

/* make_symmetry_edge_list (benchmark_helper.hpp:383-497) followed by the
 * CSR de-duplication of GraphConstructor2DCSR (graph_constructor.hpp:1986-2128).
 * edges are interleaved (v0, v1) pairs; self-loops are dropped. */
orc_graph* orc_graph_build(const int64_t* edges, int64_t nedges, int scale);
/* Build from an explicit symmetric CSR (used for the 2-core). */
void orc_graph_free(orc_graph* g);

/* ------------------ direction-optimizing BFS (bfs.hpp) ------------------ */

enum {
  ORC_AUTO_NUM = 9 /* parameters.h:260-270 */
};

typedef struct orc_bfs_stats {
  int levels;             /* last value of current_level_ (AUTO_LEVEL) */
  int64_t edges_td;       /* adjacency entries examined top-down */
  int64_t edges_bu;       /* adjacency entries examined bottom-up */
  int64_t visited;        /* vertices reached (including the root) */
  uint32_t direction_mask; /* bit L set: level L ran bottom-up (L < 32) */
} orc_bfs_stats;

/* BfsBase::run_bfs_core (bfs.hpp:3238-3609): writes pred[nverts]
 * ((level << 48) | parent, -1 unreached) and auto_tuning_data[9].
 * root_level offsets every level (CoreBFS).  Returns 0 on success. */
int orc_bfs(const orc_graph* g, int64_t root, int64_t root_level,
            int edgefactor, double alpha, double beta, int64_t* pred,
            int64_t* auto_tuning_data, orc_bfs_stats* stats);

/* The same search over an int32-column CSR whose rows are renumbered
 * vertices (the engine's CSR copied to host memory): row r is original vertex
 * inv[r]; pred[npred] is written in original ids.  Used as the timed CPU
 * restatement of the reference's search on the benchmark graph. */
int orc_bfs_csr32(int64_t nrows, const int64_t* row_ptr, const int32_t* col,
                  const int32_t* mdeg, const int32_t* inv, int64_t npred,
                  int64_t root_row, int edgefactor, double alpha, double beta,
                  int64_t* pred, int64_t* auto_tuning_data, orc_bfs_stats* stats);

/* Per-vertex BFS level with a plain queue BFS (the debugging oracle
 * bfs_local, external/indexed_bfs/bfs/corebfs.hpp:217-261): -1 if unreached. */
int orc_bfs_levels_simple(const orc_graph* g, int64_t root, int32_t* level);

/* ---------------------- validation (validate.hpp) ------------------------ */

/* BfsValidation::validate (validate.hpp:607-976).  edges are the ORIGINAL
 * generated (non-symmetrised) edges.  Writes depths into the high 16 bits of
 * pred when corebfs_enabled (build_bfs_depth_map).  Returns the number of
 * errors (0 = valid) and the traversed-edge count. */
int64_t orc_validate(const int64_t* edges, int64_t nedges, int64_t nglobalverts,
                     int64_t nlocalverts, int corebfs_enabled, int64_t root,
                     int64_t* pred, int64_t* edge_visit_count);

/* --------------------------- CoreBFS (-C) -------------------------------- */

typedef struct orc_core {
  orc_graph* core;        /* induced 2-core graph (same vertex ids) */
  int64_t* tree_parent;   /* parent of a pruned vertex, -1 otherwise */
  int32_t* peel_round;    /* 1.. round in which the vertex was pruned, 0 = kept */
  int rounds;             /* number of peeling rounds that removed a vertex */
} orc_core;

/* corebfs_adaptor::preprocess + decomposition::prune_trees
 * (corebfs_adaptor.hpp:328-357, decomposition.hpp:350-572).
 * Returns NULL if more than 32 rounds are needed (OR_DIE at :401). */
orc_core* orc_core_build(const orc_graph* g);
/* corebfs_index::reset_unreachable (corebfs_adaptor.hpp:228-249,
 * postprocess.hpp:106-154). */
int orc_core_reset_unreachable(orc_core* c, int edgefactor, double alpha,
                               double beta);
/* BfsBase::has_edge with CoreBFS (bfs.hpp:167-170). */
int orc_core_has_edge(const orc_core* c, int64_t v);
/* BfsBase::run_bfs with CoreBFS (bfs.hpp:3214-3232): bfs_tree climb,
 * run_bfs_core on the 2-core with the level offset, write_tree_parents. */
int orc_core_run_bfs(const orc_core* c, int64_t root, int edgefactor,
                     double alpha, double beta, int64_t* pred,
                     int64_t* auto_tuning_data, orc_bfs_stats* stats);
void orc_core_free(orc_core* c);

/* ------------------------- roots (main.cc) -------------------------------- */

/* find_roots (benchmark_helper.hpp:527-562) over a has_edge table
 * (has_edge[v] != 0).  Returns the number of roots found. */
int orc_find_roots(const uint8_t* has_edge, int64_t nglobalverts,
                   int num_roots, int r1, int r2, int64_t* roots);

/* Thread count used by the OpenMP loops (for the CPU baseline report). */
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif

#endif /* B200BFS_ORACLE_H_ */
