// Search state and level loop of the single-source BFS.
#pragma once

#include "engine.h"

namespace b200bfs {

// Per-level counters written by the kernels and read by the host.
struct Counters {
  unsigned long long nq;        // vertices discovered in the level (global_nq_size_)
  unsigned long long nq_edges;  // their pre-dedup degree sum (global_nq_edges_)
  unsigned long long scanned;   // adjacency entries read bottom-up
  unsigned long long qsize;     // length of the frontier queue
  unsigned long long qedges;    // CSR degree sum of the frontier queue
  int error;
  unsigned int blocks_done;     // blocks of the level's last kernel that finished
};

// Device-driven level loop of the single-source search (CUDA graph mode).
constexpr int kSgHist = 128;  // per-level records kept on the device
struct SgRec {
  int32_t level, bottom_up;
  int64_t input, discovered, scanned, bytes;
};
// Per-search arguments, written by the host before each graph launch.
struct SgArg {
  long long root, prev_root, root_level;
  double alpha, beta;
  int edgefactor, want_at;
  int sparse, pad;  // sparse pred assembly (see BfsState::asm_sparse)
  long long at[9];
};
// Control block: the state the host loop keeps in local variables.
struct SingleCtl {
  long long level;
  int forward, next_forward, growing, cur, done, pad;
  long long global_nq_size, global_nq_edges, visited, qsize, prev_nq;
  long long at[9];
  long long num_td, num_bu;
  unsigned long long bu_mask;
  long long scanned_td, scanned_bu, td_bytes, bu_bytes, bytes;
  int nrec, pad2;
  SgRec rec[kSgHist];
};

struct BfsState {
  bool allocated = false;
  int64_t R = 0, W = 0, pred_size = 0, nblk = 0;
  uint32_t* vis[2] = {nullptr, nullptr};  // visited bitmaps (double-buffered)
  uint32_t* fr = nullptr;                 // bits discovered in the last level
  int32_t* queue = nullptr;               // frontier rows for top-down
  int64_t* qdeg = nullptr;                // degree prefix of queue
  int64_t* blk_cnt = nullptr;
  int64_t* blk_deg = nullptr;
  int64_t* pred = nullptr;                // [pred_size], original ids
  Counters* ctr = nullptr;
  // The level counters as the device publishes them at the end of a level,
  // in host-mapped memory (hpub; dpub is its device address), with the
  // level's sequence number written last; the host waits for it by polling
  // instead of a copy and a stream synchronisation.
  struct Published {
    Counters c;
    unsigned long long seq;
  };
  Published* hpub = nullptr;
  Published* dpub = nullptr;
  unsigned long long pub_seq = 0;
  int asm_ev = -1;                        // event pair of the last assembly pass
  std::vector<cudaEvent_t> ev;            // per-level kernel timing events
  std::vector<b200bfs_level_stats> levels;  // per-level record of the last search
  // pred holds exactly the last search's result (-1 everywhere else), so the
  // next search only resets what it leaves unreached; false after
  // allocation and whenever pred was written by other code.
  bool pred_clean = false;
  int64_t prev_root = -1;                 // the last search's root entry
  // CoreBFS: pred holds the tree parents (level 0xFFFF) of all pruned
  // vertices except the last climb, whose vertices carry their levels.
  bool tree_clean = false;
  std::vector<int64_t> prev_path_v;
  // pred assembly (RunOptions::pred_assemble): the levels write rp[row]
  // (row order) and a final pass writes all of pred through pmap (one entry
  // per original id: row, -1, or -(tree parent + 2)).
  int64_t* rp = nullptr;                  // [R] row-order pred entries
  int32_t* pmap = nullptr;                // [pred_size]
  bool assembled = false;                 // the last search used the assembly
  // and wrote only the 4-id groups holding a searched row (the others kept
  // their entries from the search before); core_groups counts those groups
  bool asm_sparse = false;
  int64_t core_groups = 0;
  // device-driven level loop (graph mode)
  SingleCtl* sctl = nullptr;
  SingleCtl* hsctl = nullptr;             // pinned mirror
  SgArg* sarg = nullptr;
  uint32_t** d_vis = nullptr;             // device copy of vis[2]
  SgArg* hsarg = nullptr;                 // pinned staging
  cudaGraph_t sgraph = nullptr;
  cudaGraphExec_t sgexec = nullptr;
  std::vector<const void*> skey;

  cudaEvent_t event(size_t i);            // creates events on demand

  void allocate(DeviceArena& arena, const Graph& g);
  void release(DeviceArena& arena);
};

struct RunOptions {
  // Bottom-up form.  1: bu_kernel (one word per warp step); 2, 3, 4:
  // bu_wide_kernel with 2 words at 8 or 6 resident CTAs per SM, or 4 words
  // at 4 per SM.  Form 2 is the fastest measured at SCALE 28 (2.57 against
  // 2.69 ms per search for forms 3 and 4 on the headline graph) and within
  // 1 % of the best (form 3) at SCALE 24.
  int bu_kernel = 2;
  // Top-down form.  1: td_expand_kernel, 2: td_wide_kernel, 3: td_chunk_kernel,
  // 4: form 5 while the frontier grows, form 3 after the switch back from
  // bottom-up (measured best at SCALE 24 and 28), 5: td_expand_kernel with a
  // warp-wide search for each tile's first row, 6: td_vec_kernel (128-entry
  // warp steps, four neighbours per lane inside a row), 7: form 6 while the
  // frontier grows, form 3 after the switch back.
  int td_kernel = 4;
  int bu_probe = 8;         // bu_kernel: neighbours each lane probes before the warp sweep
  int bu_first = 1;         // bottom-up form 4: probe the dense first-neighbour array first
  // bottom-up forms 2-4 on levels with fewer unvisited rows than a quarter of
  // the bitmap words: skip full words 32 at a time (1) or step through every
  // word (0)
  int bu_sparse = 1;
  // bottom-up forms 2-4 on levels where more than half of the rows are still
  // unvisited: load every row's first-neighbour entry beside its bitmap
  // word (1) or only the unvisited rows' entries once the word is in (0)
  int bu_spec = 1;
  int td_unroll = 1;        // td form 5: 32-entry steps per lane handled together (1, 2, 4)
  int force_direction = 0;  // 0: alpha/beta rule, 1: top-down only, 2: bottom-up after level 1
  // pred output.  1: the level kernels write a row-order buffer and one
  // pass over the original ids assembles pred (sequential pred writes); 0:
  // they write pred by original id (a random 32-byte sector per entry).
  // Measured at SCALE 28: 3.2 against 4.2 ms per search with group
  // reordering and CoreBFS, 4.4 against 6.4 ms on the plain graph.
  int pred_assemble = 1;
  int batch_graph = 1;      // batched search: level loop in a CUDA graph (0: host loop)
  // single-source search: level loop on the device in a CUDA graph (default
  // forms only: bottom-up form 4, top-down forms 1, 3, 4, 5); 0: host loop
  // with per-level kernel timings
  int single_graph = 0;
  double batch_alpha = 30;  // batched search: alpha used when the caller passes alpha <= 0
};

void run_bfs_core(const Graph& g, BfsState& st, cudaStream_t s, int sms, int64_t root,
                  int64_t root_level, int edgefactor, double alpha, double beta, int64_t* at,
                  const RunOptions& opt, b200bfs_run_stats* stats);

void levels_from_pred(const BfsState& st, cudaStream_t s, int sms, int32_t* d_levels);

inline bool use_pred_assembly(const Graph&, const RunOptions& o) { return o.pred_assemble != 0; }
// Allocates rp and pmap (if needed) and fills pmap from the current row map
// and tree parents; synchronises the stream.
void build_pred_assembly(DeviceArena& arena, const Graph& g, BfsState& st, cudaStream_t s,
                         int sms);
int64_t assembly_bytes(const BfsState& st, int64_t visited, bool sparse);
// After the search's stream work is complete: the assembly pass time.
void finish_run_stats(BfsState& st, b200bfs_run_stats* stats);

}  // namespace b200bfs
