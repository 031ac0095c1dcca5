// Engine autotuner: picks the kernel forms of the single-source search and
// the alpha of the batched search for the resident graph by timing them.
//
// The reference has no counterpart (its equivalents are compile-time
// constants of parameters.h, and -A tunes only the switch thresholds).
// Candidates are measured with CUDA events on the engine's stream, each after
// one warm-up use; the fastest is kept in the engine's options.  None of the
// choices changes levels or the validity of parents.
#include <algorithm>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "engine_state.h"

namespace b200bfs {
namespace {

struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  EventPair() {
    check_cuda(cudaEventCreate(&a), "event");
    check_cuda(cudaEventCreate(&b), "event");
  }
  ~EventPair() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

// Total CUDA-event time (ms) of one search from every root.
double time_searches(Engine& e, const std::vector<int64_t>& roots, int edgefactor, double alpha,
                     double beta, EventPair& ev) {
  b200bfs_run_stats rs;
  int64_t at[9];
  auto one = [&](int64_t root) {
    if (e.g.core.enabled)
      core_run_bfs(e.g, e.st, e.stream, e.sms, root, edgefactor, alpha, beta, at, e.opt, &rs);
    else
      run_bfs_core(e.g, e.st, e.stream, e.sms, root, 0, edgefactor, alpha, beta, at, e.opt, &rs);
  };
  one(roots[0]);  // warm-up with this configuration
  check_cuda(cudaEventRecord(ev.a, e.stream), "event");
  for (int64_t r : roots) one(r);
  check_cuda(cudaEventRecord(ev.b, e.stream), "event");
  check_cuda(cudaEventSynchronize(ev.b), "tune");
  float ms = 0;
  check_cuda(cudaEventElapsedTime(&ms, ev.a, ev.b), "elapsed");
  return ms;
}

}  // namespace
}  // namespace b200bfs

using b200bfs::Engine;

extern "C" int b200bfs_tune_engine(b200bfs_handle* h, const int64_t* roots, int num_roots,
                                   int edgefactor, double alpha, double beta, int what,
                                   b200bfs_tune_report* out) {
  if (!h) return B200BFS_ERR_INVALID;
  try {
    Engine& e = h->e;
    b200bfs::check_cuda(cudaSetDevice(e.device), "device");
    if (!roots || num_roots < 1 || alpha <= 0 || beta <= 0 || edgefactor <= 0)
      throw b200bfs::Error{B200BFS_ERR_INVALID, "bad arguments"};
    if (!e.prepared) throw b200bfs::Error{B200BFS_ERR_STATE, "prepare_bfs not called"};
    for (int i = 0; i < num_roots; ++i)
      if (roots[i] < 0 || roots[i] >= e.g.nverts)
        throw b200bfs::Error{B200BFS_ERR_INVALID, "root out of range"};
    b200bfs_tune_report rep;
    memset(&rep, 0, sizeof(rep));
    std::vector<int64_t> rs(roots, roots + std::min(num_roots, 16));
    b200bfs::EventPair ev;
    if (what & B200BFS_TUNE_FORMS) {
      double best = 1e30;
      int best_bu = e.opt.bu_kernel;
      for (int bu = 1; bu <= 4; ++bu) {
        e.opt.bu_kernel = bu;
        const double t = b200bfs::time_searches(e, rs, edgefactor, alpha, beta, ev);
        rep.searches += (int)rs.size() + 1;
        if (t < best) {
          best = t;
          best_bu = bu;
        }
      }
      e.opt.bu_kernel = best_bu;
      best = 1e30;
      int best_td = e.opt.td_kernel;
      for (int td : {1, 3, 4, 5, 6, 7}) {
        e.opt.td_kernel = td;
        const double t = b200bfs::time_searches(e, rs, edgefactor, alpha, beta, ev);
        rep.searches += (int)rs.size() + 1;
        if (t < best) {
          best = t;
          best_td = td;
        }
      }
      e.opt.td_kernel = best_td;
      rep.single_ms = best / (double)rs.size();
    }
    rep.alpha = alpha;
    rep.beta = beta;
    if (what & B200BFS_TUNE_SWITCH) {
      // coordinate search: alpha, then beta, each scaled by a few factors
      double best = b200bfs::time_searches(e, rs, edgefactor, alpha, beta, ev);
      rep.searches += (int)rs.size() + 1;
      for (int param = 0; param < 2; ++param) {
        const double base = param == 0 ? rep.alpha : rep.beta;
        double pick = base;
        for (double f : {0.5, 0.7, 1.4, 2.0}) {
          const double a = param == 0 ? base * f : rep.alpha;
          const double b = param == 1 ? base * f : rep.beta;
          const double t = b200bfs::time_searches(e, rs, edgefactor, a, b, ev);
          rep.searches += (int)rs.size() + 1;
          if (t < 0.99 * best) {
            best = t;
            pick = base * f;
          }
        }
        (param == 0 ? rep.alpha : rep.beta) = pick;
      }
      rep.single_ms = best / (double)rs.size();
    }
    if (what & B200BFS_TUNE_BATCH_ALPHA) {
      b200bfs::ensure_batch_view(e.arena, e.g, e.stream, e.sms);
      const int k = std::min(num_roots, B200BFS_BATCH_MAX);
      double best = 1e30, best_a = e.opt.batch_alpha;
      for (double a : {10.0, 20.0, 30.0, 50.0, 100.0, 200.0, 400.0}) {
        b200bfs_batch_stats st;
        b200bfs::run_batch(e.arena, e.g, e.bs, e.stream, e.sms, roots, k, edgefactor, a, beta,
                           e.opt.batch_graph != 0, &st);  // warm-up
        b200bfs::run_batch(e.arena, e.g, e.bs, e.stream, e.sms, roots, k, edgefactor, a, beta,
                           e.opt.batch_graph != 0, &st);
        rep.batches += 2;
        if (st.ms < best) {
          best = st.ms;
          best_a = a;
        }
      }
      e.opt.batch_alpha = best_a;
      rep.batch_ms = best;
    }
    rep.bu_kernel = e.opt.bu_kernel;
    rep.td_kernel = e.opt.td_kernel;
    rep.batch_alpha = e.opt.batch_alpha;
    e.have_run = false;
    if (out) *out = rep;
    return B200BFS_OK;
  } catch (const b200bfs::Error& err) {
    h->e.last_error = err.msg;
    return err.code;
  }
}
