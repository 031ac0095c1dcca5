// Golden-output harness over the reference's own driver code.  It includes
// mpi/main.cc unchanged (its main() renamed) and repeats graph500_bfs's flow
// (main.cc:393-470, 610-660): generate_graph_spec2010, redistribute_edge_2d,
// make_symmetry_edge_list, BfsOnCPU::construct (the stock BfsBase), root
// selection by find_roots_in_large_graph or, with -A, the auto_tuning α/β
// tuner (main.cc:334-391), then run_bfs + get_pred + validate_bfs_result for
// every root.  Instead of timing, it writes what the searches produced:
//
//   OUTDIR/meta.txt     scale, edgefactor, alpha, beta (after -A), corebfs,
//                       reorder bits, pred size, num_global_edges/verts
//   OUTDIR/roots.bin    int64[n]      the roots, in order
//   OUTDIR/atd.bin      int64[n][9]   auto_tuning_data of each timed search
//   OUTDIR/nedge.bin    int64[n]      validate_bfs_result's traversed edges
//   OUTDIR/valid.bin    int8[n]       validate_bfs_result's verdict
//   OUTDIR/pred_NN.bin  int64[pred]   pred after search NN (reference encoding)
//
// usage: ref_dump SCALE OUTDIR [-e ef] [-a alpha] [-b beta] [-r seed] [-n roots] [-A] [-C]
// Test infrastructure (fixtures under tests/golden/); built by oracle/ref/Makefile.
#define main graph500_reference_main
#include "main.cc"
#undef main

#include <sys/stat.h>

#include <cstdio>
#include <string>
#include <vector>

static void write_file(const std::string& path, const void* data, size_t bytes) {
  FILE* f = fopen(path.c_str(), "wb");
  if (f == NULL || fwrite(data, 1, bytes, f) != bytes) {
    fprintf(stderr, "ref_dump: cannot write %s\n", path.c_str());
    exit(1);
  }
  fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s SCALE OUTDIR [-e ef] [-a alpha] [-b beta] [-r seed] [-n roots] [-A] [-C]\n",
            argv[0]);
    return 2;
  }
  const int SCALE = atoi(argv[1]);
  const std::string out = argv[2];
  int edgefactor = DEFAULT_EDGE_FACTOR, root_seed = 0, num_bfs_roots = TEST_BFS_ROOTS;
  double alpha = DEFAULT_ALPHA, beta = DEFAULT_BETA;
  bool auto_tune = false, corebfs_enabled = false;
  for (int i = 3; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "-e" && i + 1 < argc) edgefactor = atoi(argv[++i]);
    else if (a == "-a" && i + 1 < argc) alpha = atof(argv[++i]);
    else if (a == "-b" && i + 1 < argc) beta = atof(argv[++i]);
    else if (a == "-r" && i + 1 < argc) root_seed = atoi(argv[++i]);
    else if (a == "-n" && i + 1 < argc) num_bfs_roots = atoi(argv[++i]);
    else if (a == "-A") auto_tune = true;
    else if (a == "-C") corebfs_enabled = true;
    else {
      fprintf(stderr, "ref_dump: unknown argument %s\n", a.c_str());
      return 2;
    }
  }
  mkdir(out.c_str(), 0755);

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

    std::vector<int64_t> bfs_roots(num_bfs_roots);
    const int64_t max_used_vertex = find_max_used_vertex(benchmark->graph_);
    const int64_t nlocalverts = benchmark->graph_.pred_size();
    int64_t* pred = static_cast<int64_t*>(cache_aligned_xmalloc(nlocalverts * sizeof(pred[0])));
    benchmark->prepare_bfs(2, false, false, edgefactor, alpha, beta, pred);

    if (!auto_tune) {
      std::vector<int64_t[AUTO_NUM]> atd(num_bfs_roots);
      std::vector<double> perf(num_bfs_roots);
      find_roots_in_large_graph(0, num_bfs_roots, benchmark, bfs_roots.data(), pred, SCALE,
                                edgefactor, atd.data(), alpha, beta, perf.data(), root_seed);
    } else {
      auto_tuning(0, num_bfs_roots, benchmark, root_seed, bfs_roots.data(), pred, SCALE,
                  edgefactor, &alpha, &beta);
    }

    std::vector<int64_t> atd((size_t)num_bfs_roots * AUTO_NUM, AUTO_NOT_DEFINED);
    std::vector<int64_t> nedge(num_bfs_roots, 0);
    std::vector<int8_t> valid(num_bfs_roots, 0);
    for (int i = 0; i < num_bfs_roots; ++i) {
      benchmark->run_bfs(bfs_roots[i], pred, edgefactor, alpha, beta, &atd[(size_t)i * AUTO_NUM]);
      benchmark->get_pred(pred);
      char name[64];
      snprintf(name, sizeof(name), "/pred_%02d.bin", i);
      write_file(out + name, pred, (size_t)nlocalverts * sizeof(int64_t));
      int64_t count = 0;
      valid[i] = validate_bfs_result(&edge_list, max_used_vertex + 1, nlocalverts, corebfs_enabled,
                                     bfs_roots[i], pred, &count)
                     ? 1
                     : 0;
      nedge[i] = count;
    }
    write_file(out + "/roots.bin", bfs_roots.data(), bfs_roots.size() * sizeof(int64_t));
    write_file(out + "/atd.bin", atd.data(), atd.size() * sizeof(int64_t));
    write_file(out + "/nedge.bin", nedge.data(), nedge.size() * sizeof(int64_t));
    write_file(out + "/valid.bin", valid.data(), valid.size());

    FILE* m = fopen((out + "/meta.txt").c_str(), "w");
    fprintf(m, "scale %d\nedgefactor %d\nalpha %.17g\nbeta %.17g\ncorebfs %d\nauto_tune %d\n", SCALE,
            edgefactor, alpha, beta, (int)corebfs_enabled, (int)auto_tune);
#ifdef SMALL_REORDER_BIT
    fprintf(m, "reorder_bits %d\n", benchmark->graph_.reorder_bits_);
#else
    fprintf(m, "reorder_bits 0\n");
#endif
    fprintf(m, "pred_size %" PRId64 "\nnum_global_edges %" PRId64 "\nnum_global_verts %" PRId64
               "\nmax_used_vertex %" PRId64 "\nroots %d\n",
            nlocalverts, benchmark->graph_.num_global_edges_, benchmark->graph_.num_global_verts_,
            max_used_vertex, num_bfs_roots);
    fclose(m);

    benchmark->end_bfs();
    delete benchmark;
    free(pred);
  }
  cleanup_globals();
  return 0;
}
