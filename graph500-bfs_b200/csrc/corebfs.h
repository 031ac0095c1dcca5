// CoreBFS forest pruning on the device.
#pragma once

#include "bfs_internal.h"

namespace b200bfs {

// Peels degree-1 trees off g.csr and replaces g.csr by the 2-core.
void build_core(DeviceArena& arena, cudaStream_t s, Graph& g, int sms);
void free_core(DeviceArena& arena, Graph& g);
// corebfs_index::reset_unreachable (mpi/corebfs_adaptor.hpp:228-249).
void core_reset_unreachable(DeviceArena& arena, cudaStream_t s, int sms, Graph& g, BfsState& st,
                            int edgefactor, double alpha, double beta, const RunOptions& opt);
// BfsBase::run_bfs with CoreBFS (mpi/bfs.hpp:3214-3232).
void core_run_bfs(const Graph& g, BfsState& st, cudaStream_t s, int sms, int64_t root,
                  int edgefactor, double alpha, double beta, int64_t* at, const RunOptions& opt,
                  b200bfs_run_stats* stats);
// The climb of bfs_tree_with_callback (corebfs.hpp:125-157) from root to the
// searched 2-core: the path's vertices and pred entries, the vertex where it
// enters the core and the level there.
void core_climb(const Graph& g, int64_t root, std::vector<int64_t>& path_v,
                std::vector<int64_t>& path_e, int64_t* entry, int64_t* entry_level);
// write_tree_parents (corebfs_adaptor.hpp:285-301): pruned vertices get their
// tree parent with level 0xFFFF, then the climbed path.  Returns launches.
int core_write_tree(const Graph& g, int64_t* pred, const std::vector<int64_t>& path_v,
                    const std::vector<int64_t>& path_e, cudaStream_t s, int sms);
// Exact levels of pruned vertices from their parents (d_levels holds the
// levels taken from pred, 0xFFFF for pruned vertices).
void core_fill_levels(const Graph& g, const BfsState& st, cudaStream_t s, int sms,
                      int32_t* d_levels);
// has_edge for every vertex (bfs.hpp:167-170).
void has_edge_all(const Graph& g, cudaStream_t s, int sms, uint8_t* d_out);

}  // namespace b200bfs
