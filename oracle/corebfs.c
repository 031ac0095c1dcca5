/*
 * Oracle: CoreBFS forest pruning.  TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Restates external/indexed_bfs/bfs/corebfs/decomposition.hpp:350-572
 * (prune_trees), postprocess.hpp:106-154 (reset_unreachable),
 * corebfs.hpp:125-157 (bfs_tree_with_callback) and
 * mpi/corebfs_adaptor.hpp:228-301 (reset_unreachable, bfs_tree,
 * write_tree_parents) for a single rank.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

/* Leaf peeling: in each round every vertex whose number of live neighbours is
 * exactly one (a leaf) takes that neighbour, live at the start of the round,
 * as its parent; the leaf is then removed and its parent loses one neighbour,
 * being removed without a parent when that count reaches zero
 * (find_leaves / find_mark_twigs / update_by_source / update_by_target,
 * decomposition.hpp:137-313).  More than 32 rounds abort (:401). */
orc_core* orc_core_build(const orc_graph* g) {
  const int64_t n = g->nverts;
  int64_t* deg = (int64_t*)malloc(n * sizeof(int64_t));
  uint8_t* live = (uint8_t*)malloc(n);
  uint8_t* snap = (uint8_t*)malloc(n);
  int64_t* leaves = (int64_t*)malloc(n * sizeof(int64_t));
  orc_core* c = (orc_core*)calloc(1, sizeof(orc_core));
  c->tree_parent = (int64_t*)malloc(n * sizeof(int64_t));
  c->peel_round = (int32_t*)calloc(n, sizeof(int32_t));
  for (int64_t v = 0; v < n; ++v) {
    deg[v] = g->row_ptr[v + 1] - g->row_ptr[v];
    live[v] = deg[v] > 0;
    c->tree_parent[v] = -1;
  }
  int rounds = 0;
  for (int iter = 1;; ++iter) {
    if (iter > 32) {
      free(deg); free(live); free(snap); free(leaves);
      orc_core_free(c);
      return NULL;
    }
    int64_t nl = 0;
    for (int64_t v = 0; v < n; ++v)
      if (deg[v] == 1) leaves[nl++] = v;
    if (nl == 0) break;
    rounds = iter;
    memcpy(snap, live, n);
    int64_t* par = (int64_t*)malloc(nl * sizeof(int64_t));
    for (int64_t i = 0; i < nl; ++i) {
      int64_t s = leaves[i];
      par[i] = -1;
      for (int64_t j = g->row_ptr[s]; j < g->row_ptr[s + 1]; ++j)
        if (snap[g->col[j]]) {
          par[i] = g->col[j];
          break;
        }
    }
    for (int64_t i = 0; i < nl; ++i) {
      int64_t s = leaves[i];
      if (par[i] < 0) continue;
      deg[s] = 0;
      c->tree_parent[s] = par[i];
      c->peel_round[s] = iter;
      live[s] = 0;
    }
    for (int64_t i = 0; i < nl; ++i) {
      int64_t t = par[i];
      if (t < 0) continue;
      if (deg[t] > 0) {
        if (--deg[t] == 0) {
          live[t] = 0;
          c->peel_round[t] = iter;
        }
      }
    }
    free(par);
  }
  c->rounds = rounds;

  /* The 2-core: edges whose two endpoints are still live
   * (remove_removed, decomposition.hpp:315-332). */
  orc_graph* k = (orc_graph*)calloc(1, sizeof(orc_graph));
  k->nverts = n;
  k->scale = g->scale;
  k->row_ptr = (int64_t*)malloc((n + 1) * sizeof(int64_t));
  k->multideg = (int64_t*)calloc(n, sizeof(int64_t));
  k->row_ptr[0] = 0;
  for (int64_t v = 0; v < n; ++v) {
    int64_t d = 0;
    if (live[v])
      for (int64_t j = g->row_ptr[v]; j < g->row_ptr[v + 1]; ++j) d += live[g->col[j]];
    k->row_ptr[v + 1] = k->row_ptr[v] + d;
    k->multideg[v] = d;
    k->num_verts += d > 0;
  }
  k->num_edges = k->row_ptr[n];
  k->col = (int64_t*)malloc((k->num_edges + 1) * sizeof(int64_t));
  for (int64_t v = 0; v < n; ++v) {
    int64_t o = k->row_ptr[v];
    if (live[v])
      for (int64_t j = g->row_ptr[v]; j < g->row_ptr[v + 1]; ++j)
        if (live[g->col[j]]) k->col[o++] = g->col[j];
  }
  c->core = k;
  free(deg);
  free(live);
  free(snap);
  free(leaves);
  return c;
}

void orc_core_free(orc_core* c) {
  if (!c) return;
  orc_graph_free(c->core);
  free(c->tree_parent);
  free(c->peel_round);
  free(c);
}

/* BFS from the highest-degree core vertex; tree vertices whose parent chain
 * does not end in a reached core vertex lose their parent. */
int orc_core_reset_unreachable(orc_core* c, int edgefactor, double alpha,
                               double beta) {
  const orc_graph* k = c->core;
  const int64_t n = k->nverts;
  int64_t best = 0;
  for (int64_t v = 1; v < n; ++v)
    if (k->multideg[v] > k->multideg[best]) best = v;
  int64_t* pred = (int64_t*)malloc(n * sizeof(int64_t));
  int64_t at[ORC_AUTO_NUM];
  orc_bfs(k, best, 0, edgefactor, alpha, beta, pred, at, NULL);
  uint8_t* reach = (uint8_t*)malloc(n);
  for (int64_t v = 0; v < n; ++v) reach[v] = pred[v] != -1;
  for (int changed = 1; changed;) {
    changed = 0;
    for (int64_t v = 0; v < n; ++v) {
      int64_t p = c->tree_parent[v];
      if (p >= 0 && !reach[v] && reach[p]) {
        reach[v] = 1;
        changed = 1;
      }
    }
  }
  for (int64_t v = 0; v < n; ++v)
    if (c->tree_parent[v] >= 0 && !reach[v]) c->tree_parent[v] = -1;
  free(reach);
  free(pred);
  return 0;
}

int orc_core_has_edge(const orc_core* c, int64_t v) {
  return c->core->row_ptr[v + 1] > c->core->row_ptr[v] || c->tree_parent[v] >= 0;
}

static inline int64_t pred_entry(int64_t parent, int64_t level) {
  return (int64_t)(((uint64_t)(level & 0xFFFF) << 48) |
                   ((uint64_t)parent & UINT64_C(0xFFFFFFFFFFFF)));
}

int orc_core_run_bfs(const orc_core* c, int64_t root, int edgefactor,
                     double alpha, double beta, int64_t* pred, int64_t* at,
                     orc_bfs_stats* stats) {
  /* Climb from the root to the 2-core; every vertex on the way takes the
   * previous one as its parent (bfs_tree_with_callback). */
  int64_t path_v[64], path_e[64];
  int np = 0;
  int64_t u = root, p = root;
  int64_t lv = 0;
  for (;; ++lv) {
    if (np >= 64) return -1;
    path_v[np] = p;
    path_e[np] = pred_entry(u, lv);
    ++np;
    u = p;
    p = c->tree_parent[u];
    if (p < 0) break;
  }
  orc_bfs(c->core, u, lv, edgefactor, alpha, beta, pred, at, stats);
  /* write_tree_parents: pruned vertices get their tree parent with the
   * unknown level 0xFFFF; the climbed path overrides them. */
  const int64_t n = c->core->nverts;
  for (int64_t v = 0; v < n; ++v)
    if (c->tree_parent[v] >= 0) pred[v] = pred_entry(c->tree_parent[v], 0xFFFF);
  for (int i = 0; i < np; ++i) pred[path_v[i]] = path_e[i];
  return 0;
}
