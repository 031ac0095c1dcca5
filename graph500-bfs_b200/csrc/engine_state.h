// The engine behind one b200bfs_handle: a device-resident graph, the
// single-source search state and the batched-search state.
#pragma once

#include <string>
#include "bfs_internal.h"
#include "corebfs.h"
#include "msbfs.h"

namespace b200bfs {

struct Engine {
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t run_ev[2] = {nullptr, nullptr};  // b200bfs_run start / end
  DeviceArena arena;
  Graph g;
  BfsState st;
  BatchState bs;
  bool prepared = false;
  bool have_run = false;
  int64_t last_root = -1;
  b200bfs_run_stats last_stats{};
  RunOptions opt;
  std::string last_error = "no error";

  void free_graph() {
    if (st.allocated) st.release(arena);
    bs.release(arena);
    prepared = false;
    have_run = false;
    free_batch_view(arena, g);
    free_core(arena, g);
    arena.free(g.csr.row_ptr);
    arena.free(g.csr.col);
    arena.free(g.csr.inv);
    arena.free(g.csr.rank);
    arena.free(g.csr.mdeg);
    arena.free(g.csr.first);
    arena.free(g.csr.first_pair);
    arena.free(g.input_edges);
    g = Graph();
  }

  void finish_build(uint2* d_edges, int64_t m, int scale_hint, int flags) {
    const bool mirror = !(flags & B200BFS_BUILD_INPUT_SYMMETRIC);
    g.input_edges = d_edges;
    g.num_input_edges = m;
    g.input_symmetric = !mirror;
    build_csr(arena, stream, d_edges, m, mirror, (flags & B200BFS_BUILD_GROUP_REORDER) != 0,
              scale_hint, g, sms);
    if (flags & B200BFS_BUILD_COREBFS) build_core(arena, stream, g, sms);
    g.built = true;
    g.device_bytes = (int64_t)arena.in_use();
  }

  // Runs a graph build; on failure every allocation of the build is released
  // and the handle is left without a graph.
  template <typename F>
  void build_guarded(F&& f) {
    free_graph();
    const uint64_t m = arena.mark();
    try {
      f();
    } catch (...) {
      cudaStreamSynchronize(stream);
      cudaGetLastError();
      arena.rollback(m);
      g = Graph();
      throw;
    }
  }
};

}  // namespace b200bfs

// The opaque handle of the C ABI.
struct b200bfs_handle {
  b200bfs::Engine e;
};
