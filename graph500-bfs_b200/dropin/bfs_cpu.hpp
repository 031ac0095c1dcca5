/*
 * bfs_cpu.hpp -- drop-in replacement for the reference's mpi/bfs_cpu.hpp.
 *
 * The reference's file (mpi/bfs_cpu.hpp:8-15) names the engine that main.cc
 * drives: `typedef BfsBase BfsOnCPU;`.  This file keeps its include guard and
 * its include of bfs.hpp (main.cc also includes bfs.hpp itself) and names the
 * B200 engine instead.  Placed at mpi/bfs_cpu.hpp, with graph500-bfs_b200/ on
 * the include path and libb200bfs.so linked, it leaves main.cc,
 * benchmark_helper.hpp (find_roots, find_max_used_vertex), validate.hpp and
 * logfile.h unchanged: they see `benchmark->graph_` as the reference's
 * Graph2DCSR and call construct / prepare_bfs / run_bfs / get_pred /
 * end_bfs / has_edge as they do on BfsBase.
 */

#ifndef BFS_CPU_HPP_
#define BFS_CPU_HPP_

#include "bfs.hpp"
#include <bfs_on_b200.hpp>

typedef BfsOnB200 BfsOnCPU;

#endif /* BFS_CPU_HPP_ */
