// Internal interfaces of the B200 BFS engine (not part of the C ABI).
#pragma once

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/b200bfs.h"

namespace b200bfs {

// ------------------------------- generator ---------------------------------
cudaError_t launch_generate(int scale, uint64_t seed1, uint64_t seed2, int64_t start, int64_t end,
                            uint2* out, cudaStream_t stream);
void host_seed_state(uint64_t s1, uint64_t s2, uint32_t z[5]);
void host_mrg_skip(uint32_t z[5], uint64_t hi, uint64_t mid, uint64_t lo);
uint32_t host_mrg_next(uint32_t z[5]);
void host_scramble_values(uint64_t s1, uint64_t s2, uint64_t* v0, uint64_t* v1);
double host_random_double(uint64_t s1, uint64_t s2, int64_t position);
void find_roots_host(const uint8_t* has_edge, int64_t nglobal, int num_roots, int r1, int r2,
                     int64_t* roots);

// Error carrying a status code and message through the engine.
struct Error {
  int code;
  std::string msg;
};

// A device-memory budget shared by several arenas (the graphs of a server).
struct SharedBudget {
  uint64_t limit = 0;
  std::atomic<uint64_t> used{0};
};

// Device memory with an optional budget (b200bfs_config.hbm_budget_bytes)
// and an optional budget shared with other arenas.  Allocations carry a
// sequence number so that a failed build can release everything it
// allocated (mark / rollback).  Thread-safe.
class DeviceArena {
 public:
  explicit DeviceArena(uint64_t budget = 0) : budget_(budget) {}
  void set_shared(SharedBudget* sb) { shared_ = sb; }
  void* alloc(size_t bytes, const char* what);  // throws Error
  void free(void* p);
  uint64_t mark() const { return seq_; }
  void rollback(uint64_t mark);  // frees every allocation made after mark
  uint64_t in_use() const { return in_use_; }
  uint64_t budget() const { return budget_; }
  void set_budget(uint64_t b) { budget_ = b; }

 private:
  struct Block {
    void* p;
    size_t bytes;
    uint64_t seq;
  };
  uint64_t budget_;
  uint64_t in_use_ = 0;
  uint64_t seq_ = 0;
  std::vector<Block> live_;
  SharedBudget* shared_ = nullptr;
  std::mutex mu_;
};

template <typename T>
T* arena_alloc(DeviceArena& a, int64_t n, const char* what) {
  return static_cast<T*>(a.alloc((size_t)(n > 0 ? n : 1) * sizeof(T), what));
}

void check_cuda(cudaError_t e, const char* what);  // throws Error on failure

// A CSR over reordered vertex ids ("rows").  Row r holds the de-duplicated
// neighbours of original vertex inv[r], highest pre-dedup degree first; rows
// are in descending order of the pre-dedup degree (optionally within groups
// of 2^reorder_bits original ids, when the neighbour order is the global
// degree order rather than the row order), so without groups low row ids
// are the high-degree vertices and neighbour lists are ascending.
struct Csr {
  int64_t nrows = 0;           // R: vertices with >= 1 edge
  int64_t nedges = 0;          // E: directed entries after de-duplication
  int64_t* row_ptr = nullptr;  // [R + 1]
  int32_t* col = nullptr;      // [E]
  int32_t* inv = nullptr;      // [R]     row -> original id
  int32_t* rank = nullptr;     // [nverts] original id -> row, -1 if no edge
  int32_t* mdeg = nullptr;     // [R]     pre-dedup degree (degree_, graph_constructor.hpp:572-592)
  // [R] first (highest-degree) neighbour of each row, kept apart so that a
  // bottom-up probe of it is one coalesced 4-byte read per row (the
  // reference keeps each row's first edge apart too: isolated_edges_,
  // graph_constructor.hpp:1224-1348)
  int32_t* first = nullptr;
  // [R] (first[r], inv[first[r]]): the first neighbour and its original
  // id in one 8-byte entry, so that the single-root bottom-up search gets
  // both with one load and a parent found by the first probe needs neither
  // a second load nor a random gather into inv[] (null in the batch view)
  int2* first_pair = nullptr;
  int64_t max_degree = 0;
};

// CoreBFS index on the device.
struct CoreIndex {
  bool enabled = false;
  int rounds = 0;                      // peeling rounds that removed a vertex
  int32_t* tree_parent = nullptr;      // [nverts] original ids, -1 = none
  std::vector<int32_t> h_tree_parent;  // host copy for the root climb
  int2* tree_list = nullptr;           // [tree_vertices] (vertex, parent), original ids
  int64_t core_vertices = 0;
  int64_t tree_vertices = 0;
};

struct Graph {
  bool built = false;
  int scale = 0;               // estimated SCALE (log_orig_global_verts_)
  int64_t nverts = 0;          // 2^scale
  int64_t pred_size = 0;       // max(2^scale, 2^16) (graph_constructor.hpp:1085-1094)
  int64_t num_input_edges = 0;
  bool group_reorder = false;
  int reorder_bits = 0;
  Csr csr;                     // the searched graph (the 2-core with CoreBFS)
  CoreIndex core;
  uint2* input_edges = nullptr;  // device copy of the input edges, for validation
  // The searched graph renumbered in global degree order, for the batched
  // search on group-reordered graphs (built on first use; csr otherwise).
  Csr bview;
  int32_t* b_of_row = nullptr;   // [csr.nrows] row -> bview row
  bool bview_built = false;
  bool input_symmetric = false;
  int64_t device_bytes = 0;
};

// Fills c.first from c.row_ptr and c.col, and c.first_pair when parent_ids.
void build_first(DeviceArena& arena, cudaStream_t s, Csr& c, int sms, bool parent_ids = true);

// Builds g.csr from nedges device edges (each a (v0, v1) pair of uint32 ids).
void build_csr(DeviceArena& arena, cudaStream_t s, const uint2* edges, int64_t nedges,
               bool mirror, bool group_reorder, int scale_hint, Graph& g, int num_sms);

}  // namespace b200bfs
