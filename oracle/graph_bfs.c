/*
 * Oracle: symmetric CSR, direction-optimizing BFS, Graph500 validation and
 * root sampling.  TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include "oracle.h"

int orc_num_threads(void) { return omp_get_max_threads(); }

static int cmp_i64(const void* a, const void* b) {
  int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
  return (x > y) - (x < y);
}

static int msb_index(uint64_t v) { return v ? 63 - __builtin_clzll(v) : -1; }

/* make_symmetry_edge_list (mpi/benchmark_helper.hpp:383-497): self-loops are
 * dropped, each edge is emitted in both directions and the SCALE is estimated
 * from the OR of all endpoints.  The CSR rows are then sorted and
 * de-duplicated as GraphConstructor2DCSR::sortEdgesInner does
 * (mpi/graph_constructor.hpp:1986-2056); multideg keeps the pre-dedup count
 * that DegreeCalculation::calc_degree accumulates (:572-592). */
orc_graph* orc_graph_build(const int64_t* edges, int64_t m, int scale) {
  uint64_t orv = 0;
#pragma omp parallel for reduction(| : orv)
  for (int64_t i = 0; i < m; ++i) {
    int64_t a = edges[2 * i], b = edges[2 * i + 1];
    if (a != b) orv |= (uint64_t)(a | b);
  }
  int est = msb_index(orv) + 1;
  if (scale <= 0) scale = est;
  orc_graph* g = (orc_graph*)calloc(1, sizeof(orc_graph));
  g->scale = est;
  const int64_t n = INT64_C(1) << scale;
  g->nverts = n;
  g->multideg = (int64_t*)calloc(n, sizeof(int64_t));
  int64_t* raw_ptr = (int64_t*)calloc(n + 1, sizeof(int64_t));
#pragma omp parallel for
  for (int64_t i = 0; i < m; ++i) {
    int64_t a = edges[2 * i], b = edges[2 * i + 1];
    if (a == b) continue;
    __atomic_fetch_add(&g->multideg[a], 1, __ATOMIC_RELAXED);
    __atomic_fetch_add(&g->multideg[b], 1, __ATOMIC_RELAXED);
  }
  for (int64_t v = 0; v < n; ++v) raw_ptr[v + 1] = raw_ptr[v] + g->multideg[v];
  int64_t* cursor = (int64_t*)malloc(n * sizeof(int64_t));
  memcpy(cursor, raw_ptr, n * sizeof(int64_t));
  int64_t* raw = (int64_t*)malloc((raw_ptr[n] + 1) * sizeof(int64_t));
#pragma omp parallel for
  for (int64_t i = 0; i < m; ++i) {
    int64_t a = edges[2 * i], b = edges[2 * i + 1];
    if (a == b) continue;
    raw[__atomic_fetch_add(&cursor[a], 1, __ATOMIC_RELAXED)] = b;
    raw[__atomic_fetch_add(&cursor[b], 1, __ATOMIC_RELAXED)] = a;
  }
  free(cursor);
  int64_t* dlen = (int64_t*)calloc(n, sizeof(int64_t));
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < n; ++v) {
    int64_t b = raw_ptr[v], e = raw_ptr[v + 1];
    if (e - b > 1) qsort(raw + b, e - b, sizeof(int64_t), cmp_i64);
    int64_t k = 0;
    for (int64_t j = b; j < e; ++j)
      if (k == 0 || raw[b + k - 1] != raw[j]) raw[b + k++] = raw[j];
    dlen[v] = k;
  }
  g->row_ptr = (int64_t*)malloc((n + 1) * sizeof(int64_t));
  g->row_ptr[0] = 0;
  int64_t nv = 0;
  for (int64_t v = 0; v < n; ++v) {
    g->row_ptr[v + 1] = g->row_ptr[v] + dlen[v];
    nv += dlen[v] > 0;
  }
  g->num_edges = g->row_ptr[n];
  g->num_verts = nv;
  g->col = (int64_t*)malloc((g->num_edges + 1) * sizeof(int64_t));
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < n; ++v)
    memcpy(g->col + g->row_ptr[v], raw + raw_ptr[v], dlen[v] * sizeof(int64_t));
  free(dlen);
  free(raw);
  free(raw_ptr);
  return g;
}

void orc_graph_free(orc_graph* g) {
  if (!g) return;
  free(g->row_ptr);
  free(g->col);
  free(g->multideg);
  free(g);
}

/* --------------------------------- BFS ----------------------------------- */

#define AUTO_GLOBAL_NQ_EDGES 0
#define AUTO_NUM_GLOBAL_EDGES 1
#define AUTO_T2B_LEVEL 2
#define AUTO_GLOBAL_NQ_SIZE 3
#define AUTO_NUM_GLOBAL_VERTS 4
#define AUTO_B2T_LEVEL 5
#define AUTO_PRE_GLOBAL_NQ_EDGES 6
#define AUTO_PRE_GLOBAL_NQ_SIZE 7
#define AUTO_LEVEL 8

#define BIT_TEST(bm, v) (((bm)[(v) >> 6] >> ((v)&63)) & 1)

#define BFS_NAME bfs_impl64
#define COL_T int64_t
#define MDEG_T int64_t
#include "bfs_body.inc"
#undef BFS_NAME
#undef COL_T
#undef MDEG_T
#define BFS_NAME bfs_impl32
#define COL_T int32_t
#define MDEG_T int32_t
#include "bfs_body.inc"
#undef BFS_NAME
#undef COL_T
#undef MDEG_T

int orc_bfs(const orc_graph* g, int64_t root, int64_t root_level,
            int edgefactor, double alpha, double beta, int64_t* pred,
            int64_t* at, orc_bfs_stats* stats) {
  return bfs_impl64(g->nverts, g->row_ptr, g->col, g->multideg, g->num_edges,
                    g->num_verts, NULL, g->nverts, root, root_level, edgefactor,
                    alpha, beta, pred, at, stats);
}

int orc_bfs_csr32(int64_t nrows, const int64_t* row_ptr, const int32_t* col,
                  const int32_t* mdeg, const int32_t* inv, int64_t npred,
                  int64_t root_row, int edgefactor, double alpha, double beta,
                  int64_t* pred, int64_t* at, orc_bfs_stats* stats) {
  return bfs_impl32(nrows, row_ptr, col, mdeg, row_ptr[nrows], nrows, inv, npred,
                    root_row, 0, edgefactor, alpha, beta, pred, at, stats);
}

int orc_bfs_levels_simple(const orc_graph* g, int64_t root, int32_t* level) {
  const int64_t n = g->nverts;
  for (int64_t i = 0; i < n; ++i) level[i] = -1;
  int64_t* q = (int64_t*)malloc((n + 1) * sizeof(int64_t));
  int64_t h = 0, t = 0;
  level[root] = 0;
  q[t++] = root;
  while (h < t) {
    int64_t v = q[h++];
    for (int64_t j = g->row_ptr[v]; j < g->row_ptr[v + 1]; ++j) {
      int64_t u = g->col[j];
      if (level[u] < 0) {
        level[u] = level[v] + 1;
        q[t++] = u;
      }
    }
  }
  free(q);
  return 0;
}

/* ------------------------------ validation -------------------------------- */

static inline int64_t pe_parent(int64_t x) { return (int64_t)((uint64_t)x << 16) >> 16; }
static inline uint16_t pe_depth(int64_t x) { return (uint16_t)(((uint64_t)x >> 48) & 0xFFFF); }
static inline void pe_set_depth(int64_t* x, uint16_t d) {
  *x = (int64_t)(((uint64_t)*x & UINT64_C(0xFFFFFFFFFFFF)) | ((uint64_t)d << 48));
}

/* BfsValidation::validate (mpi/validate.hpp:607-976) for one rank, with
 * check_value_ranges (:994-1016), check_pred_depth (:1018-1034),
 * build_bfs_depth_map (:1040-1141) and
 * check_bfs_depth_map_using_predecessors (:1145-1254). */
int64_t orc_validate(const int64_t* edges, int64_t m, int64_t nglobalverts,
                     int64_t nlocalverts, int corebfs, int64_t root,
                     int64_t* pred, int64_t* edge_visit_count) {
  int64_t err = 0;
  *edge_visit_count = 0;
#pragma omp parallel for reduction(+ : err)
  for (int64_t i = 0; i < nlocalverts; ++i) {
    int64_t p = pe_parent(pred[i]);
    if (p < -1 || p >= nglobalverts) ++err;
  }
  if (root < 0 || root >= nglobalverts) ++err;
  if (err) return err;
  if (pe_parent(pred[root]) != root) return 1;
#pragma omp parallel for reduction(+ : err)
  for (int64_t i = 0; i < nlocalverts; ++i)
    if (i != root && pe_parent(pred[i]) != -1 && pe_parent(pred[i]) == i) ++err;
  if (err) return err;

  if (corebfs) {
    pe_set_depth(&pred[root], 0);
    for (int iter = 0;; ++iter) {
      int changes = 0;
#pragma omp parallel for reduction(+ : err) reduction(| : changes)
      for (int64_t i = 0; i < nlocalverts; ++i) {
        if (i == root) continue;
        int64_t p = pe_parent(pred[i]);
        if (p < 0 || pe_depth(pred[i]) != 0xFFFF) continue;
        uint16_t dp = pe_depth(pred[p]);
        if (dp != 0xFFFF) {
          pe_set_depth(&pred[i], (uint16_t)(dp + 1));
          changes = 1;
        }
      }
      if (!changes) break;
    }
  } else {
    if (pe_depth(pred[root]) != 0) ++err;
#pragma omp parallel for reduction(+ : err)
    for (int64_t i = 0; i < nlocalverts; ++i) {
      int64_t p = pe_parent(pred[i]);
      uint16_t d = pe_depth(pred[i]);
      if (p == -1 && d != 0xFFFF) ++err;
      else if (p != -1 && d == 0xFFFF) ++err;
      if (i == root || p == -1) continue;
      uint16_t dp = pe_depth(pred[p]);
      if (dp == 0xFFFF) ++err;
      if ((int)d != (int)dp + 1) ++err;
    }
  }
  if (err) return err;

  uint8_t* pred_valid = (uint8_t*)calloc(nlocalverts, 1);
  int64_t count = 0;
#pragma omp parallel for reduction(+ : err, count)
  for (int64_t i = 0; i < m; ++i) {
    const int64_t s = edges[2 * i], t = edges[2 * i + 1];
    const int64_t ps = pred[s], pt = pred[t];
    const int sd = pe_depth(ps), td = pe_depth(pt);
    if (sd != 0xFFFF && td == 0xFFFF) ++err;
    else if (sd == 0xFFFF && td != 0xFFFF) ++err;
    else if (sd - td < -1 || sd - td > 1) ++err;
    else if (sd != 0xFFFF) ++count;
    if (pe_parent(ps) == t) {
      if (s != t && td + 1 != sd) ++err;
      pred_valid[s] = 1;
    }
    if (pe_parent(pt) == s) {
      if (s != t && sd + 1 != td) ++err;
      pred_valid[t] = 1;
    }
  }
#pragma omp parallel for reduction(+ : err)
  for (int64_t i = 0; i < nlocalverts; ++i) {
    if (pe_parent(pred[i]) == -1 || i == root) continue;
    if (!pred_valid[i]) ++err;
  }
  free(pred_valid);
  *edge_visit_count = count;
  return err;
}

/* ------------------------------- roots ------------------------------------ */

/* find_roots (mpi/benchmark_helper.hpp:527-562) with USERSEED1/2 = 2/3. */
int orc_find_roots(const uint8_t* has_edge, int64_t nglobalverts, int num_roots,
                   int r1, int r2, int64_t* roots) {
  int64_t counter = 0;
  int idx;
  for (idx = 0; idx < num_roots; ++idx) {
    int64_t root;
    for (;;) {
      double d[2];
      orc_make_random_numbers(2, 2 + r1, 3 + r2, counter, d);
      root = (int64_t)((d[0] + d[1]) * nglobalverts) % nglobalverts;
      counter += 2;
      if (counter > 2 * nglobalverts) break;
      int dup = 0;
      for (int i = 0; i < idx; ++i)
        if (roots[i] == root) {
          dup = 1;
          break;
        }
      if (dup) continue;
      if (has_edge[root]) break;
    }
    roots[idx] = root;
  }
  return idx;
}
