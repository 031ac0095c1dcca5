// bfs_on_b200.hpp -- header-only C++ adapter with the member surface of the
// reference's `class BfsBase` (mpi/bfs.hpp:48-172) over the C ABI of
// include/b200bfs.h.
//
// Drop-in use with the reference driver: graph500-bfs_b200/dropin/bfs_cpu.hpp
// replaces mpi/bfs_cpu.hpp (`typedef BfsBase BfsOnCPU;`, bfs_cpu.hpp:13) by
// `typedef BfsOnB200 BfsOnCPU;`.  Compiled there, after the reference's
// graph_constructor.hpp, `graph_` is the reference's own Graph2DCSR
// (graph_constructor.hpp:115-333), filled so that its has_edge(v),
// pred_size() and log_orig_global_verts_ answer for the engine's graph; so
// benchmark_helper.hpp's find_roots (`const Graph2DCSR& g =
// benchmark.graph_`, :532) and find_max_used_vertex (:565-582) compile and run
// unchanged, as do main.cc's timing around run_bfs, validate.hpp on the pred
// that get_pred fills, and the result printing.  Outside the reference tree
// (runnable.cc) `graph_` is a small struct with the same members.  Errors are
// thrown as std::runtime_error, as the reference throws.
#ifndef B200BFS_BFS_ON_B200_HPP_
#define B200BFS_BFS_ON_B200_HPP_

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/b200bfs.h"

// The part of Graph2DCSR that main.cc and benchmark_helper.hpp read
// (graph_constructor.hpp:187-333), for builds outside the reference tree.
struct B200GraphFacade {
  int log_orig_global_verts_ = 0;
  int reorder_bits_ = 0;
  int64_t num_orig_local_verts_ = 0;
  int64_t num_global_edges_ = 0;
  int64_t num_global_verts_ = 0;
  std::vector<uint8_t> has_edge_;

  int pred_size() const { return (int)num_orig_local_verts_; }
  int log_orig_global_verts() const { return log_orig_global_verts_; }
  bool has_edge(int64_t v, bool = false) const {
    return v >= 0 && v < (int64_t)has_edge_.size() && has_edge_[(size_t)v];
  }
};

class BfsOnB200 {
 public:
#ifdef GRAPH_CONSTRUCTOR_HPP_
  typedef Graph2DCSR GraphType;  // the reference's graph type
#else
  typedef B200GraphFacade GraphType;
#endif

  explicit BfsOnB200(int device = 0, uint64_t hbm_budget_bytes = 0) {
#ifdef GRAPH_CONSTRUCTOR_HPP_
    // Graph2DCSR's constructor leaves invert_map_ unset and clean() frees it.
    graph_.invert_map_ = NULL;
#endif
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
  bool has_edge(int64_t root) const {
    return root >= 0 && root < (int64_t)has_edge_.size() && has_edge_[(size_t)root];
  }

  b200bfs_handle* handle() { return h_; }

  GraphType graph_;

 private:
  void refresh_graph() {
    b200bfs_graph_info gi;
    check(b200bfs_graph_info_get(h_, &gi), "graph info");
    has_edge_.assign((size_t)gi.pred_size, 0);
    check(b200bfs_has_edge_all(h_, has_edge_.data()), "has_edge");
    fill_graph(gi);
  }

#ifdef GRAPH_CONSTRUCTOR_HPP_
  // Gives the reference's Graph2DCSR an identity vertex layout over the
  // engine's has-edge flags: one process owns every vertex, local id = global
  // id (vertex_local, graph_constructor.hpp:29), reorder_map_ maps each id to
  // itself (within its group of 2^reorder_bits_ ids under SMALL_REORDER_BIT),
  // and has_edge_bitmap_ has bit v set iff v has an edge.  Graph2DCSR::has_edge
  // (:251-280) then returns the engine's answer in both reorder modes.  The
  // CSR arrays stay NULL: the engine holds the graph on the device.
  void fill_graph(const b200bfs_graph_info& gi) {
    Graph2DCSR& g = graph_;
    g.clean();
    const int64_t n = gi.pred_size;
    g.log_orig_global_verts_ = gi.scale;
    g.num_orig_local_verts_ = n;
    g.num_global_edges_ = gi.num_global_edges;
    g.num_global_verts_ = gi.num_global_verts;
    int id_bits = 0;  // bits of a local id: pred_size is a power of two
    while ((int64_t(1) << id_bits) < n) ++id_bits;
    g.local_bits_ = id_bits;
    g.orig_local_bits_ = id_bits;
    g.r_bits_ = 0;
    g.num_local_verts_ = n;
    g.reorder_map_ = static_cast<LocalVertex*>(malloc(sizeof(LocalVertex) * (size_t)(n > 0 ? n : 1)));
    const int64_t words = (n + 63) / 64;
    g.has_edge_bitmap_ = static_cast<BitmapType*>(calloc((size_t)(words > 0 ? words : 1), sizeof(BitmapType)));
    if (g.reorder_map_ == NULL || g.has_edge_bitmap_ == NULL)
      throw std::runtime_error("graph_: host allocation failed");
#ifdef SMALL_REORDER_BIT
    if (gi.reorder_bits <= 0 || gi.reorder_bits > 16 || (n & ((int64_t(1) << gi.reorder_bits) - 1)) != 0)
      throw std::runtime_error("graph_: group reordering needs groups of 2^1..2^16 ids dividing pred_size");
    g.reorder_bits_ = gi.reorder_bits;
    g.num_group_verts_ = int32_t(1) << gi.reorder_bits;
    g.num_groups_ = n >> gi.reorder_bits;
    const int64_t mask = (int64_t(1) << gi.reorder_bits) - 1;
    for (int64_t v = 0; v < n; ++v) g.reorder_map_[v] = (LocalVertex)(v & mask);
#else
    for (int64_t v = 0; v < n; ++v) g.reorder_map_[v] = (LocalVertex)v;
#endif
    for (int64_t v = 0; v < n; ++v)
      if (has_edge_[(size_t)v]) g.has_edge_bitmap_[v >> 6] |= BitmapType(1) << (v & 63);
#ifdef BFS_HPP_
    // main.cc:519-533 reports the all-to-all buffer sizes in units of the
    // global a2a_buf_unit (it divides by it), which BfsBase sets when it
    // allocates (bfs.hpp:218).  The engine uses no such buffers, so
    // max_num_buffers stays 0 and the proposed size printed is 0.
    a2a_buf_unit = g.num_local_verts_ * (int64_t)sizeof(int32_t);
#endif
  }
#else
  void fill_graph(const b200bfs_graph_info& gi) {
    graph_.log_orig_global_verts_ = gi.scale;
    graph_.reorder_bits_ = gi.reorder_bits;
    graph_.num_orig_local_verts_ = gi.pred_size;
    graph_.num_global_edges_ = gi.num_global_edges;
    graph_.num_global_verts_ = gi.num_global_verts;
    graph_.has_edge_ = has_edge_;
  }
#endif

  void check(int rc, const char* what) const {
    if (rc != B200BFS_OK)
      throw std::runtime_error(std::string(what) + ": " + b200bfs_last_error(h_));
  }

  b200bfs_handle* h_ = nullptr;
  std::vector<uint8_t> has_edge_;  // 1 per original id with an edge
};

#endif  // B200BFS_BFS_ON_B200_HPP_
