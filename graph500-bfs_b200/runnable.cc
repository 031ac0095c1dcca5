// runnable -- the Graph500 BFS benchmark driver on the B200 engine.
//
// Same command line and the same flow as the reference driver
// (mpi/main.cc:393-714, 749-870), through the BfsOnB200 adapter:
// generate + construct -> find roots (re-picked while a root reaches no more
// than 3 levels, main.cc:334-359) -> optional -A alpha/beta tuning ->
// timed run_bfs per root -> get_pred -> validation -> the result block of
// print_bfs_result (mpi/logfile.h:54-133).
//
//   runnable SCALE [-e edgefactor] [-a alpha] [-b beta] [-r root_seed]
//            [-n roots] [-s skip] [-v 0|1|2] [-A] [-C] [-G] [-R]
//
// -G selects degree ordering within groups of 2^16 vertices (the
// SMALL_REORDER_BIT build of the reference).  Validation runs on the device
// (b200bfs_validate, the rules of mpi/validate.hpp:607-976); its traversed-edge
// count is the TEPS numerator, as in main.cc:643-664.
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "bfs_on_b200.hpp"

namespace {

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Order statistics of get_statistics (mpi/logfile.h:26-53).
struct Stats {
  double min, q1, median, q3, max, mean, sd;
};

Stats statistics(std::vector<double> x) {
  Stats s{};
  const size_t n = x.size();
  double m = 0;
  for (double v : x) m += v;
  m /= n;
  double var = 0;
  for (double v : x) var += (v - m) * (v - m);
  var = n > 1 ? var / (n - 1) : 0;
  std::sort(x.begin(), x.end());
  s.mean = m;
  s.sd = std::sqrt(var);
  s.min = x[0];
  s.q1 = (x[(n - 1) / 4] + x[n / 4]) * .5;
  s.median = (x[(n - 1) / 2] + x[n / 2]) * .5;
  s.q3 = (x[n - 1 - (n - 1) / 4] + x[n - 1 - n / 4]) * .5;
  s.max = x[n - 1];
  return s;
}

void print_result(const std::vector<double>& t, const std::vector<double>& v,
                  const std::vector<double>& e) {
  Stats s = statistics(t);
  printf("min_time:                       %.12g\n", s.min);
  printf("firstquartile_time:             %.12g\n", s.q1);
  printf("median_time:                    %.12g\n", s.median);
  printf("thirdquartile_time:             %.12g\n", s.q3);
  printf("max_time:                       %.12g\n", s.max);
  printf("mean_time:                      %.12g\n", s.mean);
  printf("stddev_time:                    %.12g\n", s.sd);
  s = statistics(e);
  printf("min_nedge:                      %.11g\n", s.min);
  printf("firstquartile_nedge:            %.11g\n", s.q1);
  printf("median_nedge:                   %.11g\n", s.median);
  printf("thirdquartile_nedge:            %.11g\n", s.q3);
  printf("max_nedge:                      %.11g\n", s.max);
  printf("mean_nedge:                     %.11g\n", s.mean);
  printf("stddev_nedge:                   %.11g\n", s.sd);
  std::vector<double> spe(t.size());
  for (size_t i = 0; i < t.size(); ++i) spe[i] = t[i] / e[i];
  s = statistics(spe);
  printf("min_TEPS:                       %.12g\n", 1. / s.max);
  printf("firstquartile_TEPS:             %.12g\n", 1. / s.q3);
  printf("median_TEPS:                    %.12g\n", 1. / s.median);
  printf("thirdquartile_TEPS:             %.12g\n", 1. / s.q1);
  printf("max_TEPS:                       %.12g\n", 1. / s.min);
  printf("harmonic_mean_TEPS:             %.12g\n", 1. / s.mean);
  printf("harmonic_stddev_TEPS:           %.12g\n",
         t.size() > 1 ? s.sd / (s.mean * s.mean * std::sqrt((double)t.size() - 1)) : 0.0);
  s = statistics(v);
  printf("min_validate:                   %.12g\n", s.min);
  printf("firstquartile_validate:         %.12g\n", s.q1);
  printf("median_validate:                %.12g\n", s.median);
  printf("thirdquartile_validate:         %.12g\n", s.q3);
  printf("max_validate:                   %.12g\n", s.max);
  printf("mean_validate:                  %.12g\n", s.mean);
  printf("stddev_validate:                %.12g\n", s.sd);
}

[[noreturn]] void usage(const char* prog) {
  fprintf(stderr,
          "Usage: %s SCALE [-e edgefactor] [-a alpha] [-b beta] [-r root_seed] [-n roots]\n"
          "       [-s skip] [-v 0|1|2] [-A] [-C] [-G] [-R]\n",
          prog);
  exit(1);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc <= 1 || atoi(argv[1]) <= 0) usage(argv[0]);
  const int scale = atoi(argv[1]);
  int edgefactor = 16, root_seed = 0, num_roots = 16, root_start = 0, validation = 2;
  double alpha = 10.0, beta = 14.0;
  bool tune = false, corebfs = false, group = false;
  optind = 2;
  int c;
  while ((c = getopt(argc, argv, "e:a:b:r:n:s:v:ACGR")) != -1) {
    switch (c) {
      case 'e': edgefactor = atoi(optarg); break;
      case 'a': alpha = atof(optarg); break;
      case 'b': beta = atof(optarg); break;
      case 'r': root_seed = atoi(optarg); break;
      case 'n': num_roots = atoi(optarg); break;
      case 's': root_start = atoi(optarg); break;
      case 'v': validation = atoi(optarg); break;
      case 'A': tune = true; break;
      case 'C': corebfs = true; break;
      case 'G': group = true; break;
      case 'R': num_roots = 64; validation = 2; break;
      default: usage(argv[0]);
    }
  }
  if (edgefactor <= 0 || alpha <= 0 || beta <= 0 || num_roots <= 0 || validation < 0 ||
      validation > 2 || root_start < 0 || root_start >= num_roots)
    usage(argv[0]);
  if (root_start != 0 && tune) {
    fprintf(stderr, "-s and -A are not available at the same time.\n");
    return 1;
  }
  try {
    BfsOnB200::printInformation(validation, false, false);
    BfsOnB200 bfs;
    double t0 = now();
    bfs.construct_generated(scale, edgefactor, corebfs, group);
    const double construction_time = now() - t0;
    std::vector<int64_t> pred((size_t)bfs.graph_.pred_size());
    bfs.prepare_bfs(validation, false, false, edgefactor, alpha, beta, pred.data());

    // find_roots_in_large_graph (main.cc:334-359)
    std::vector<int64_t> roots((size_t)num_roots);
    std::vector<double> nedge((size_t)num_roots);
    for (int r = root_seed;; ++r) {
      if (b200bfs_find_roots(bfs.handle(), num_roots, r, 0, roots.data()) != B200BFS_OK)
        throw std::runtime_error(b200bfs_last_error(bfs.handle()));
      bool ok = true;
      for (int i = 0; i < num_roots && ok; ++i) {
        int64_t at[9];
        bfs.run_bfs(roots[i], pred.data(), edgefactor, alpha, beta, at);
        if (scale > 6 && at[8] <= 3) ok = false;
        int64_t err = 0, cnt = 0;
        if (ok && b200bfs_validate(bfs.handle(), roots[i], &err, &cnt) == B200BFS_OK)
          nedge[i] = (double)cnt;
      }
      if (ok) break;
      fprintf(stderr, "Pick roots again\n");
    }
    if (tune) {
      double teps = 0;
      const double t = now();
      if (b200bfs_auto_tune(bfs.handle(), roots.data(), num_roots, nedge.data(), edgefactor,
                            &alpha, &beta, &teps) != B200BFS_OK)
        throw std::runtime_error(b200bfs_last_error(bfs.handle()));
      fprintf(stderr, "Estimated Performance = %.0f MTEPS with Alpha = %f and Beta = %f\n",
              teps / 1e6, alpha, beta);
      fprintf(stderr, "Elapsed Time for auto tuning = %f sec.\n", now() - t);
    }

    std::vector<double> bfs_times, validate_times, edge_counts;
    bool ok = true;
    for (int i = root_start; i < num_roots; ++i) {
      fprintf(stderr, "========== Running BFS %02d ==========\n", i);
      int64_t at[9];
      const double t = now();
      bfs.run_bfs(roots[i], pred.data(), edgefactor, alpha, beta, at);
      const double bt = now() - t;
      bfs.get_pred(pred.data());
      const double vt0 = now();
      int64_t err = 0, cnt = (int64_t)nedge[i];
      if (validation == 2 || (validation == 1 && i == root_start)) {
        if (b200bfs_validate(bfs.handle(), roots[i], &err, &cnt) != B200BFS_OK)
          throw std::runtime_error(b200bfs_last_error(bfs.handle()));
      }
      const double vt = now() - vt0;
      fprintf(stderr, "Time for BFS %02d is %f\n", i, bt);
      fprintf(stderr, "Number of traversed edges is %lld\n", (long long)cnt);
      fprintf(stderr, "TEPS for BFS %02d is %g\n", i, cnt / bt);
      bfs_times.push_back(bt);
      validate_times.push_back(vt);
      edge_counts.push_back((double)cnt);
      if (err != 0) {
        ok = false;
        break;
      }
    }
    bfs.end_bfs();
    printf("============= Result ==============\n");
    printf("SCALE:                          %d\n", scale);
    printf("edgefactor:                     %d\n", edgefactor);
    printf("alpha:                          %f\n", alpha);
    printf("beta:                           %f\n", beta);
    printf("NBFS:                           %d\n", num_roots);
    if (group) printf("Reorder bits:                   %d\n", bfs.graph_.reorder_bits_);
    printf("graph_generation:               %g\n", construction_time);
    printf("num_mpi_processes:              %d\n", 1);
    printf("construction_time:              %g\n", construction_time);
    printf("redistribution_time:            %g\n", 0.0);
    if (!ok) {
      printf("No results printed for invalid run.\n");
      return 1;
    }
    print_result(bfs_times, validate_times, edge_counts);
  } catch (const std::exception& ex) {
    fprintf(stderr, "error: %s\n", ex.what());
    return 1;
  }
  return 0;
}
