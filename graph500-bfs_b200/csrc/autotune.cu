// Alpha/beta auto-tuning (the driver's -A mode) on the device-resident graph.
//
// Restates auto_tuning / auto_tuning_each / measure_performance of
// mpi/main.cc:45-391.  Every root is searched once with the current
// (alpha, beta); auto_tuning_data records where each search switched
// direction.  Alpha is then moved so that the top-down -> bottom-up switch of
// one root happens one level earlier (smaller alpha) or later (larger alpha):
// the direction comes from comparing the slowest root that switched with the
// fastest root that did not (main.cc:106-127); the new value is the
// threshold of that root times 0.99 or 1.01, nudged until the switch level
// really moves (:145-167, :245-258).  A move is kept while it does not slow
// the moved root down; the first move that does is undone and tuning of that
// parameter stops.  Beta follows with the bottom-up -> top-down switch.
// Search times are CUDA-event times of the engine's run.
#include <algorithm>
#include <cmath>
#include <vector>
#include "bfs_internal.h"
#include "autotune.h"

namespace b200bfs {
namespace {

enum {
  kGlobalNqEdges = 0,
  kNumGlobalEdges = 1,
  kT2BLevel = 2,
  kGlobalNqSize = 3,
  kNumGlobalVerts = 4,
  kB2TLevel = 5,
  kPreGlobalNqEdges = 6,
  kPreGlobalNqSize = 7,
  kLevel = 8,
  kAutoNum = 9
};
constexpr int64_t kNotDefined = -1;

struct Entry {
  int64_t val;
  int idx;
  bool operator<(const Entry& o) const { return val < o.val; }
};

double harmonic(const std::vector<double>& perf) {
  double s = 0;
  for (double p : perf) s += 1.0 / p;
  return perf.size() / s;
}

class Tuner {
 public:
  Tuner(const SearchFn& search, const std::vector<int64_t>& roots,
        const std::vector<double>& nedge, int edgefactor)
      : search_(search), roots_(roots), nedge_(nedge), ef_(edgefactor),
        at_(roots.size(), std::vector<int64_t>(kAutoNum, kNotDefined)), perf_(roots.size()) {}

  void measure(double alpha, double beta) {
    for (auto& a : at_) std::fill(a.begin(), a.end(), kNotDefined);
    for (size_t i = 0; i < roots_.size(); ++i) {
      const double t = search_(roots_[i], alpha, beta, at_[i].data());
      perf_[i] = nedge_[i] / t;
    }
  }

  // One tuning pass of alpha (is_alpha) or beta; returns false when tuning
  // of that parameter has ended.
  bool step(bool is_alpha, double* alpha, double* beta, int* tries) {
    std::vector<Entry> s, l;
    for (size_t i = 0; i < roots_.size(); ++i) {
      const int64_t a = is_alpha ? at_[i][kGlobalNqEdges] : at_[i][kPreGlobalNqSize];
      if (a != kNotDefined) s.push_back({a, (int)i});
      const int64_t b = is_alpha ? at_[i][kPreGlobalNqEdges] : at_[i][kGlobalNqSize];
      if (b != kNotDefined) l.push_back({b, (int)i});
    }
    std::sort(s.begin(), s.end());
    std::sort(l.begin(), l.end());
    bool smaller;
    if (s.empty()) return false;
    if (l.empty()) smaller = true;
    else smaller = perf_[s.front().idx] < perf_[l.back().idx];

    auto level_of = [&](int idx) {
      return (int)(is_alpha ? at_[idx][kT2BLevel] : at_[idx][kB2TLevel]);
    };
    const int n = smaller ? (int)s.size() : (int)l.size();
    for (int k = 0; k < n; ++k) {
      const Entry e = smaller ? s[k] : l[n - 1 - k];
      const int idx = e.idx;
      const double pre_param = is_alpha ? *alpha : *beta;
      const int pre_level = level_of(idx);
      if (pre_level == kNotDefined) return false;
      if (smaller) {
        if (is_alpha && pre_level + 1 == at_[idx][kLevel]) return false;
        if (!is_alpha && pre_level == 1) return false;
      } else {
        if (is_alpha && pre_level == 1) return false;
        if (!is_alpha && pre_level + 1 == at_[idx][kLevel]) return false;
      }
      const double edges = (double)at_[idx][kNumGlobalEdges];
      const double verts = (double)at_[idx][kNumGlobalVerts];
      if (is_alpha) {
        if (smaller) {
          *alpha = edges / e.val * 0.99;
          while (e.val > (int64_t)(at_[idx][kNumGlobalEdges] / *alpha)) *alpha *= 0.99;
        } else {
          *alpha = edges / e.val * 1.01;
          while (e.val <= (int64_t)(at_[idx][kNumGlobalEdges] / *alpha)) *alpha *= 1.01;
        }
      } else {
        if (smaller) {
          *beta = verts / (e.val * ef_ * 2.0) * 0.99;
          while (e.val >= (int64_t)(at_[idx][kNumGlobalVerts] / (*beta * ef_ * 2.0))) *beta *= 0.99;
        } else {
          *beta = verts / (e.val * ef_ * 2.0) * 1.01;
          while (e.val < (int64_t)(at_[idx][kNumGlobalVerts] / (*beta * ef_ * 2.0))) *beta *= 1.01;
        }
      }
      std::fill(at_[idx].begin(), at_[idx].end(), kNotDefined);
      const double t = search_(roots_[idx], *alpha, *beta, at_[idx].data());
      ++*tries;
      const double new_perf = nedge_[idx] / t;
      if (level_of(idx) == pre_level)
        throw Error{B200BFS_ERR_STATE, "auto-tuning: the switch level did not move"};
      const double pre_perf = perf_[idx];
      perf_[idx] = new_perf;
      if (pre_perf > new_perf) {
        perf_[idx] = pre_perf;
        (is_alpha ? *alpha : *beta) = pre_param;
        return false;
      }
    }
    return true;
  }

  double teps() const { return harmonic(perf_); }

 private:
  const SearchFn& search_;
  const std::vector<int64_t>& roots_;
  const std::vector<double>& nedge_;
  int ef_;
  std::vector<std::vector<int64_t>> at_;
  std::vector<double> perf_;
};

}  // namespace

double auto_tune(const SearchFn& search, const std::vector<int64_t>& roots,
                 const std::vector<double>& nedge, int edgefactor, double* alpha, double* beta,
                 int* tries) {
  Tuner t(search, roots, nedge, edgefactor);
  *tries = 0;
  t.measure(*alpha, *beta);
  while (t.step(true, alpha, beta, tries)) t.measure(*alpha, *beta);
  while (t.step(false, alpha, beta, tries)) t.measure(*alpha, *beta);
  return t.teps();
}

}  // namespace b200bfs
