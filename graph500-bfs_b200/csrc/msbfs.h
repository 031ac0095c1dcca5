// Batched multi-source BFS: up to 64 roots traversed together.
#pragma once

#include "bfs_internal.h"

namespace b200bfs {

constexpr int kBatchMax = 64;        // roots per batch (one bit each of a uint64 mask)
constexpr int kBatchHist = 256;      // per-level records kept on the device
constexpr double kBatchAlpha = 30.0; // default top-down -> bottom-up threshold of a batch

// Counters of the level being computed (device).
struct BatchCounters {
  unsigned long long active;      // OR of the root bits found in the level (exact)
  unsigned long long scanned_bu;  // adjacency entries read bottom-up
  unsigned long long rows_bu;     // rows with unseen bottom-up bits
  unsigned long long qsize;       // rows of the top-down queue
  unsigned long long qedges;      // adjacency entries of the top-down queue rows
  unsigned long long cnt[kBatchMax];  // per-root frontier rows (sampled estimate)
  unsigned long long edg[kBatchMax];  // per-root pre-dedup degree sum (sampled estimate)
};

struct BatchLevelRec {
  unsigned long long td_roots;    // roots expanded top-down in the level
  unsigned long long bu_roots;    // roots searched bottom-up in the level
  unsigned long long active;      // roots that found a vertex in the level
  unsigned long long scanned_bu;
  unsigned long long rows_bu;
  unsigned long long qsize;
  unsigned long long qedges;
};

// Control block of a batched search, resident on the device.  The level
// kernels read their plan (level, masks, plane pointers) from it, and the
// control kernel writes the next plan, so the same launch sequence serves
// a host-driven loop and a device-side loop in a CUDA graph.
struct BatchCtl {
  // fixed during a search
  unsigned long long* planes;  // [capacity][R]: bit k of planes[L][v] <=> level_k(v) == L
  unsigned long long* seen;    // [R]: bits of the roots that reached v
  // [capacity][wstride]: bitmap of the rows of planes[L] that may be
  // non-zero (a superset of them), per plane.  A level clears only those rows
  // of its plane, so a plane a batch leaves mostly zero costs the next batch
  // little to reuse.
  uint32_t* rowbits;
  long long wstride;           // words per plane bitmap (>= (R + 31) / 32, multiple of 4)
  long long R;
  long long capacity;          // planes allocated
  long long nedges;            // num_global_edges (alpha test)
  long long nverts;            // num_global_verts (beta test)
  double alpha, beta;
  int edgefactor;
  int K;
  int root_row[kBatchMax];     // row where root k enters the searched graph, -1: none
  int root_lv[kBatchMax];      // level at which it enters (CoreBFS climb), 0 otherwise
  // plan of the level being computed
  long long level;
  unsigned long long td_mask;  // roots expanded top-down
  unsigned long long bu_mask_active;  // roots searched bottom-up (with a frontier)
  int has_td, has_bu;
  int done;                    // 0 running, 1 finished, 2 needs more planes, 3 level overflow
  int pad;
  // per-root switch state (the reference rule, bfs.hpp:3413-3457, per root)
  unsigned long long bu_mask, growing, pending;
  long long prev_cnt[kBatchMax];
  long long last_level[kBatchMax];  // deepest level at which root k found a vertex, -1 none
  BatchCounters c;
  BatchLevelRec hist[kBatchHist];
};

struct BatchState {
  bool allocated = false;
  int64_t R = 0;
  int64_t capacity = 0;
  int64_t nblk = 0;
  unsigned long long* planes = nullptr;
  unsigned long long* seen = nullptr;
  uint32_t* rowbits = nullptr;  // [capacity][wstride], see BatchCtl
  int64_t wstride = 0;
  int32_t* queue = nullptr;  // top-down queue rows
  int64_t* qdeg = nullptr;   // its degree prefix
  int64_t* blk_cnt = nullptr;
  int64_t* blk_deg = nullptr;
  BatchCtl* ctl = nullptr;   // device
  BatchCtl* hctl = nullptr;  // pinned mirror
  int* hdone = nullptr;      // pinned copy of ctl->done
  void* d_arg = nullptr;     // device copy of the batch arguments
  void* h_arg = nullptr;     // pinned staging of the batch arguments
  std::vector<cudaEvent_t> ev;
  // The level loop as one CUDA graph (a WHILE conditional node around the
  // level kernels), built on first use and rebuilt when a buffer it names
  // changes.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<const void*> graph_key;
  // last batch
  // neighbours a lane probes in the bottom-up sweep before the warp sweeps
  // its row (4 .. 1024), bu_round of them loaded together (4 or 8).  SCALE 28,
  // 64 roots: 8 / 32 / 128 / 1024 probes give 29.0 / 26.2 / 24.3 / 24.6 ms.
  int bu_probe = 128;
  int bu_round = 4;
  // planes[0] is zero except at plane0_rows (the last batch's level-0 root
  // rows); false after allocation and while a batch runs
  bool plane0_clean = false;
  std::vector<int32_t> plane0_rows;
  int K = 0;
  int64_t levels = 0;                 // planes in use = last level + 1
  std::vector<int64_t> roots;         // original ids
  std::vector<int64_t> entry_vertex;  // vertex where each root enters the searched graph
  std::vector<int32_t> entry_level;   // level of that vertex (CoreBFS climb length)
  std::vector<std::vector<int64_t>> path_v, path_e;  // CoreBFS climb of each root
  std::vector<b200bfs_level_stats> level_records;   // per level of the last batch
  cudaEvent_t event(size_t i);
  void release(DeviceArena& arena);
};

// Runs one batched search from roots[0..k) over g.csr.  alpha <= 0 selects
// kBatchAlpha.  use_graph: run the level loop as a CUDA graph on the device
// (one host synchronisation per batch); otherwise the host launches each
// level and records per-level timings.  The CoreBFS climb of each root is applied as in
// BfsBase::run_bfs (bfs.hpp:3214-3232).
// A BatchState shares nothing mutable with other BatchStates of the same
// graph, so batches on different states and streams may run concurrently.
void run_batch(DeviceArena& arena, const Graph& g, BatchState& bs, cudaStream_t s,
               int sms, const int64_t* roots, int k, int edgefactor, double alpha, double beta,
               bool use_graph, b200bfs_batch_stats* stats);

// The graph the batched search runs on: g.csr, or for a group-reordered
// graph its view in global degree order (hub rows together, so the masks the
// bottom-up sweep probes most stay in a few cache lines).
inline const Csr& batch_csr(const Graph& g) { return g.bview_built ? g.bview : g.csr; }
// Builds that view once (no-op unless the graph is group-reordered); not
// thread-safe: call it before concurrent batches.
void ensure_batch_view(DeviceArena& arena, Graph& g, cudaStream_t s, int sms);
void free_batch_view(DeviceArena& arena, Graph& g);

// Allocates bs for g (level planes, masks, queue, control block) ahead of
// its first batch.
void batch_reserve(DeviceArena& arena, const Graph& g, BatchState& bs);

// Writes root `index` of the last batch into st.pred in the reference
// encoding: level from the planes, parent = a neighbour one level closer to
// the root (any such neighbour is a valid BFS parent).
void batch_select(const Graph& g, BfsState& st, const BatchState& bs, cudaStream_t s, int sms,
                  int index);

}  // namespace b200bfs
