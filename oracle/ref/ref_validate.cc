// Runs the reference's own validator, validate_bfs_result (mpi/validate.hpp:
// 1269-1277), on pred arrays read from files, over the reference's own graph:
// main.cc's flow up to prepare_bfs (generate_graph_spec2010,
// redistribute_edge_2d, make_symmetry_edge_list, BfsOnCPU::construct with the
// stock BfsBase, find_max_used_vertex), then, for each file, the same call
// main.cc:647 makes.  Prints one line per file: "<valid 0/1> <edge_visit_count>".
//
// usage: ref_validate SCALE ROOT [-C] PRED_FILE...   (int64[pred_size] each)
// Test infrastructure: it pins the Graph500 verdicts of the oracle's and the
// device's validators to the reference's; built by oracle/ref/Makefile.
#define main graph500_reference_main
#include "main.cc"
#undef main

#include <cstdio>
#include <string>
#include <vector>

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s SCALE ROOT [-C] PRED_FILE...\n", argv[0]);
    return 2;
  }
  const int SCALE = atoi(argv[1]);
  const int64_t root = atoll(argv[2]);
  int first = 3;
  bool corebfs_enabled = false;
  if (std::string(argv[3]) == "-C") {
    corebfs_enabled = true;
    first = 4;
  }
  const int edgefactor = DEFAULT_EDGE_FACTOR;
  setup_globals(argc, argv, SCALE, edgefactor);
  {
    EdgeListStorage<UnweightedPackedEdge> edge_list((int64_t(1) << SCALE) * edgefactor / mpi.size_2d,
                                                    getenv("TMPFILE"));
    generate_graph_spec2010(&edge_list, SCALE, edgefactor);
    EdgeListStorage<UnweightedPackedEdge> sym_edge_list(
        (int64_t(1) << SCALE) * edgefactor / mpi.size_2d * 2, getenv("TMPFILE"), "-sym");
    redistribute_edge_2d(&edge_list);
    const auto estimated_scale = make_symmetry_edge_list(&edge_list, &sym_edge_list);
    BfsOnCPU* benchmark = new BfsOnCPU();
    benchmark->construct(estimated_scale, corebfs_enabled, &sym_edge_list);
    const int64_t max_used_vertex = find_max_used_vertex(benchmark->graph_);
    const int64_t nlocalverts = benchmark->graph_.pred_size();
    int64_t* pred = static_cast<int64_t*>(cache_aligned_xmalloc(nlocalverts * sizeof(pred[0])));
    for (int a = first; a < argc; ++a) {
      FILE* f = fopen(argv[a], "rb");
      if (f == NULL || fread(pred, sizeof(int64_t), (size_t)nlocalverts, f) != (size_t)nlocalverts) {
        fprintf(stderr, "ref_validate: cannot read %" PRId64 " entries from %s\n", nlocalverts,
                argv[a]);
        return 1;
      }
      fclose(f);
      int64_t count = 0;
      const bool ok = validate_bfs_result(&edge_list, max_used_vertex + 1, nlocalverts,
                                          corebfs_enabled, root, pred, &count);
      printf("%d %" PRId64 "\n", ok ? 1 : 0, count);
      fflush(stdout);
    }
    free(pred);
    delete benchmark;
  }
  cleanup_globals();
  return 0;
}
