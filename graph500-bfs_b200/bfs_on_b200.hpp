// bfs_on_b200.hpp -- header-only C++ adapter with the member surface of the
// reference's `class BfsBase` (mpi/bfs.hpp:48-172) over the C ABI of
// include/b200bfs.h.
//
// Drop-in use with the reference driver: replace the single line of
// mpi/bfs_cpu.hpp:13 (`typedef BfsBase BfsOnCPU;`) by
//
//     #include "bfs_on_b200.hpp"
//     typedef BfsOnB200 BfsOnCPU;
//
// and link libb200bfs.so; main.cc's root sampling (find_roots), timing
// (run_bfs between MPI_Wtime calls), validation (validate_bfs_result on the
// pred that get_pred fills) and result printing run unchanged.  Errors are
// thrown as std::runtime_error, as the reference throws.
#ifndef B200BFS_BFS_ON_B200_HPP_
#define B200BFS_BFS_ON_B200_HPP_

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/b200bfs.h"

class BfsOnB200 {
 public:
  // The part of Graph2DCSR main.cc and benchmark_helper.hpp read
  // (graph_constructor.hpp:187-333: pred_size(), has_edge(v),
  // log_orig_global_verts_, reorder_bits_).
  struct GraphFacade {
    int log_orig_global_verts_ = 0;
    int reorder_bits_ = 0;
    int64_t num_global_edges_ = 0;
    int64_t num_global_verts_ = 0;
    std::vector<uint8_t> has_edge_;
    int64_t pred_size_ = 0;

    int pred_size() const { return (int)pred_size_; }
    int log_orig_global_verts() const { return log_orig_global_verts_; }
    bool has_edge(int64_t v, bool = false) const {
      return v >= 0 && v < (int64_t)has_edge_.size() && has_edge_[(size_t)v];
    }
  };

  explicit BfsOnB200(int device = 0, uint64_t hbm_budget_bytes = 0) {
    b200bfs_config cfg{device, 0, hbm_budget_bytes};
    check(b200bfs_create(&cfg, &h_), "b200bfs_create");
  }
  ~BfsOnB200() { b200bfs_destroy(h_); }
  BfsOnB200(const BfsOnB200&) = delete;
  BfsOnB200& operator=(const BfsOnB200&) = delete;

  // BfsBase::printInformation (main.cc:410).
  static void printInformation(int validation_level, bool pre_exec, bool real_benchmark) {
    BfsOnB200 probe;
    char buf[512];
    if (b200bfs_print_information(probe.h_, buf, sizeof(buf)) == B200BFS_OK)
      fprintf(stderr, "%s (validation level %d, pre-exec %d, real benchmark %d)\n", buf,
              validation_level, (int)pre_exec, (int)real_benchmark);
  }

  // BfsBase::construct (bfs.hpp:116-139): sym_edge_list is the symmetric
  // EdgeListStorage<UnweightedPackedEdge> of make_symmetry_edge_list; its
  // chunks are gathered and handed over as 12-byte packed records.
  template <typename EdgeList>
  void construct(int scale, bool corebfs_enabled, EdgeList* sym_edge_list) {
    std::vector<uint32_t> packed;
    const int nchunks = sym_edge_list->beginRead(false);
    for (int c = 0; c < nchunks; ++c) {
      typename EdgeList::edge_type* chunk = nullptr;
      const int n = sym_edge_list->read(&chunk);
      const uint32_t* words = reinterpret_cast<const uint32_t*>(chunk);
      static_assert(sizeof(typename EdgeList::edge_type) == 12, "UnweightedPackedEdge expected");
      packed.insert(packed.end(), words, words + 3 * (size_t)n);
    }
    sym_edge_list->endRead();
    const int flags = B200BFS_BUILD_INPUT_SYMMETRIC | (corebfs_enabled ? B200BFS_BUILD_COREBFS : 0)
#ifdef SMALL_REORDER_BIT
                      | B200BFS_BUILD_GROUP_REORDER
#endif
        ;
    check(b200bfs_build_from_packed(h_, packed.data(), (int64_t)(packed.size() / 3), scale, flags),
          "construct");
    refresh_graph();
  }

  // Builds the benchmark graph on the device without a host edge list
  // (generate_graph_spec2010 + make_symmetry_edge_list + construct).
  void construct_generated(int scale, int edgefactor, bool corebfs_enabled,
                           bool group_reorder = false, uint64_t seed1 = 2, uint64_t seed2 = 3) {
    const int flags = (corebfs_enabled ? B200BFS_BUILD_COREBFS : 0) |
                      (group_reorder ? B200BFS_BUILD_GROUP_REORDER : 0);
    check(b200bfs_generate_graph(h_, scale, edgefactor, seed1, seed2, flags), "construct");
    refresh_graph();
  }

  // BfsBase::prepare_bfs (bfs.hpp:141-151).
  void prepare_bfs(int validation_level, bool pre_exec, bool real_benchmark, int edgefactor,
                   double alpha, double beta, int64_t* pred) {
    (void)validation_level;
    (void)pre_exec;
    (void)real_benchmark;
    (void)pred;
    check(b200bfs_prepare(h_, edgefactor, alpha, beta), "prepare_bfs");
  }

  // BfsBase::run_bfs (bfs.hpp:3214): blocks until the search is done; pred
  // is filled by get_pred, as the reference's GPU path did.
  void run_bfs(int64_t root, int64_t* pred, int edgefactor, double alpha, double beta,
               int64_t* auto_tuning_data) {
    (void)pred;
    check(b200bfs_run(h_, root, edgefactor, alpha, beta, auto_tuning_data), "run_bfs");
  }

  // BfsBase::get_pred (bfs.hpp:161-163).
  void get_pred(int64_t* pred) { check(b200bfs_get_pred(h_, pred), "get_pred"); }

  // BfsBase::end_bfs (bfs.hpp:165).
  void end_bfs() { check(b200bfs_end(h_), "end_bfs"); }

  // BfsBase::has_edge (bfs.hpp:167-170).
  bool has_edge(int64_t root) const { return graph_.has_edge(root); }

  b200bfs_handle* handle() { return h_; }

  GraphFacade graph_;

 private:
  void refresh_graph() {
    b200bfs_graph_info gi;
    check(b200bfs_graph_info_get(h_, &gi), "graph info");
    graph_.log_orig_global_verts_ = gi.scale;
    graph_.reorder_bits_ = gi.reorder_bits;
    graph_.num_global_edges_ = gi.num_global_edges;
    graph_.num_global_verts_ = gi.num_global_verts;
    graph_.pred_size_ = gi.pred_size;
    graph_.has_edge_.assign((size_t)gi.pred_size, 0);
    check(b200bfs_has_edge_all(h_, graph_.has_edge_.data()), "has_edge");
  }

  void check(int rc, const char* what) const {
    if (rc != B200BFS_OK)
      throw std::runtime_error(std::string(what) + ": " + b200bfs_last_error(h_));
  }

  b200bfs_handle* h_ = nullptr;
};

#endif  // B200BFS_BFS_ON_B200_HPP_
