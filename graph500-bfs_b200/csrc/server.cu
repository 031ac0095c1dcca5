// BFS server: graphs resident on one GPU, (graph, root) queries answered with
// continuous batching over batched multi-source searches.
//
// Every graph has `slots_per_graph` batch slots.  A slot is one BatchState
// (its own level planes, queue and CUDA graph of the level loop), one CUDA
// stream and one worker thread.  A worker waits until its graph has queued
// requests and its slot holds no unreleased results, takes up to max_batch
// of the oldest queued roots, runs them as one batched search on its stream
// and marks them done.  While it runs, the other slots of the same graph and
// the slots of other graphs take the requests that arrive meanwhile, so the
// device always has the batches of several slots in flight.  Graphs and
// slots are allocated against one shared HBM budget.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include "common.cuh"
#include "engine_state.h"

namespace b200bfs {
namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Request {
  int graph = 0;
  int64_t root = 0;
  int state = B200BFS_REQ_QUEUED;
  int slot = -1;
  int index = -1;      // position in its batch
  int depth = 0;
  int batch = 0;
  bool holds = false;  // keeps its slot's results
  double t_submit = 0, t_start = 0, t_done = 0;
};

struct Slot {
  BatchState bs;
  cudaStream_t stream = nullptr;
  int users = 0;  // finished requests that still hold this slot's results
  bool busy = false;
};

struct GraphEntry {
  b200bfs_handle* h = nullptr;
  int edgefactor = 16;
  std::deque<int64_t> pending;
  std::vector<std::unique_ptr<Slot>> slots;
  std::vector<std::thread> workers;
  std::mutex decode_mu;  // the engine's single-source buffers used to decode levels
};

}  // namespace

struct Server {
  b200bfs_server_config cfg{};
  SharedBudget budget;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stopping = false;
  std::vector<std::unique_ptr<GraphEntry>> graphs;
  std::unordered_map<int64_t, Request> reqs;
  int64_t next_id = 1;
  // statistics since the last reset
  std::vector<double> lat_ms;
  int64_t submitted = 0, completed = 0, failed = 0, batches = 0, batched_roots = 0;
  double t_first = -1, t_last = -1;
  std::string last_error = "no error";

  void worker(GraphEntry* ge, Slot* slot, int slot_id);
};

void Server::worker(GraphEntry* ge, Slot* slot, int slot_id) {
  Engine& e = ge->h->e;
  cudaSetDevice(e.device);
  const int max_batch = cfg.max_batch;
  std::vector<int64_t> ids, roots;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stopping || (!ge->pending.empty() && slot->users == 0); });
      if (stopping) return;
      ids.clear();
      roots.clear();
      const double t = now_s();
      while (!ge->pending.empty() && (int)ids.size() < max_batch) {
        const int64_t id = ge->pending.front();
        ge->pending.pop_front();
        auto it = reqs.find(id);
        if (it == reqs.end() || it->second.state != B200BFS_REQ_QUEUED) continue;
        Request& r = it->second;
        r.state = B200BFS_REQ_RUNNING;
        r.slot = slot_id;
        r.index = (int)ids.size();
        r.t_start = t;
        ids.push_back(id);
        roots.push_back(r.root);
      }
      if (ids.empty()) continue;
      slot->busy = true;
    }
    std::string err;
    std::vector<int> depth(ids.size(), 0);
    try {
      b200bfs_batch_stats st;
      run_batch(e.arena, e.g, slot->bs, slot->stream, e.sms, roots.data(), (int)roots.size(),
                ge->edgefactor, cfg.alpha, cfg.beta, true, &st);
      const BatchCtl& h = *slot->bs.hctl;
      for (size_t i = 0; i < ids.size(); ++i) {
        int d = slot->bs.entry_level[i];
        for (long long L = 1; L < h.level && L < kBatchHist; ++L)
          if ((h.hist[L].active >> i) & 1ull) d = std::max<int>(d, (int)L);
        depth[i] = d;
      }
    } catch (const Error& x) {
      err = x.msg;
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      const double t = now_s();
      slot->busy = false;
      ++batches;
      batched_roots += (int64_t)ids.size();
      int holders = 0;
      for (size_t i = 0; i < ids.size(); ++i) {
        auto it = reqs.find(ids[i]);
        if (it == reqs.end()) continue;  // released while running
        Request& r = it->second;
        r.t_done = t;
        r.batch = (int)ids.size();
        if (!err.empty()) {
          r.state = B200BFS_REQ_FAILED;
          ++failed;
          continue;
        }
        r.state = B200BFS_REQ_DONE;
        r.depth = depth[i];
        r.holds = cfg.keep_results != 0;
        holders += r.holds ? 1 : 0;
        ++completed;
        lat_ms.push_back(1e3 * (t - r.t_submit));
        t_last = t;
      }
      slot->users = holders;
      if (!err.empty()) last_error = err;
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
}

}  // namespace b200bfs

using b200bfs::Server;

struct b200bfs_server {
  Server s;
};

namespace {

template <typename F>
int srv_guarded(b200bfs_server* p, F&& f) {
  if (!p) return B200BFS_ERR_INVALID;
  try {
    f(p->s);
    return B200BFS_OK;
  } catch (const b200bfs::Error& err) {
    std::lock_guard<std::mutex> lk(p->s.mu);
    p->s.last_error = err.msg;
    return err.code;
  } catch (const std::bad_alloc&) {
    return B200BFS_ERR_OOM;
  }
}

void srv_require(bool cond, int code, const char* msg) {
  if (!cond) throw b200bfs::Error{code, msg};
}

b200bfs::GraphEntry* graph_of(Server& s, int id) {
  srv_require(id >= 0 && id < (int)s.graphs.size() && s.graphs[(size_t)id],
              B200BFS_ERR_NOT_FOUND, "unknown graph id");
  return s.graphs[(size_t)id].get();
}

void fill_info(const b200bfs::Request& r, b200bfs_request_info* info) {
  if (!info) return;
  info->state = r.state;
  info->graph_id = r.graph;
  info->root = r.root;
  info->depth = r.depth;
  info->batch_size = r.batch;
  info->latency_ms = r.state == B200BFS_REQ_DONE || r.state == B200BFS_REQ_FAILED
                         ? 1e3 * (r.t_done - r.t_submit) : 0.0;
  info->queue_ms = r.t_start > 0 ? 1e3 * (r.t_start - r.t_submit) : 0.0;
}

}  // namespace

extern "C" {

int b200bfs_server_start(const b200bfs_server_config* cfg, b200bfs_server** out) {
  if (!out) return B200BFS_ERR_INVALID;
  *out = nullptr;
  b200bfs_server_config c{};
  if (cfg) c = *cfg;
  if (c.max_batch == 0) c.max_batch = B200BFS_BATCH_MAX;
  if (c.slots_per_graph == 0) c.slots_per_graph = 2;
  if (c.alpha <= 0) c.alpha = b200bfs::kBatchAlpha;
  if (c.beta <= 0) c.beta = 14.0;
  if (c.max_batch < 1 || c.max_batch > B200BFS_BATCH_MAX || c.slots_per_graph < 1 ||
      c.slots_per_graph > 16)
    return B200BFS_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return B200BFS_ERR_CUDA;
  }
  if (c.device < 0 || c.device >= ndev) return B200BFS_ERR_INVALID;
  b200bfs_server* p = new (std::nothrow) b200bfs_server();
  if (!p) return B200BFS_ERR_OOM;
  p->s.cfg = c;
  p->s.budget.limit = c.hbm_budget_bytes;
  *out = p;
  return B200BFS_OK;
}

int b200bfs_server_add_graph(b200bfs_server* p, int scale, int edgefactor, uint64_t seed1,
                             uint64_t seed2, int flags, int* graph_id) {
  return srv_guarded(p, [&](Server& s) {
    srv_require(graph_id != nullptr, B200BFS_ERR_INVALID, "null output");
    b200bfs_config hc{};
    hc.device = s.cfg.device;
    b200bfs_handle* h = nullptr;
    int rc = b200bfs_create(&hc, &h);
    if (rc != B200BFS_OK) throw b200bfs::Error{rc, "engine creation failed"};
    std::unique_ptr<b200bfs::GraphEntry> ge(new b200bfs::GraphEntry());
    ge->h = h;
    ge->edgefactor = edgefactor;
    h->e.arena.set_shared(&s.budget);
    auto fail = [&](int code) {
      std::string msg = b200bfs_last_error(h);
      for (auto& sl : ge->slots) {
        sl->bs.release(h->e.arena);
        if (sl->stream) cudaStreamDestroy(sl->stream);
      }
      b200bfs_destroy(h);
      throw b200bfs::Error{code, msg};
    };
    rc = b200bfs_generate_graph(h, scale, edgefactor, seed1, seed2, flags);
    if (rc != B200BFS_OK) fail(rc);
    rc = b200bfs_prepare(h, edgefactor, 10.0, s.cfg.beta);
    if (rc != B200BFS_OK) fail(rc);
    // Slots: as many as the budget admits, at least one.
    cudaSetDevice(h->e.device);
    try {
      b200bfs::ensure_batch_view(h->e.arena, h->e.g, h->e.stream, h->e.sms);
    } catch (const b200bfs::Error& x) {
      h->e.last_error = x.msg;
      fail(x.code);
    }
    for (int i = 0; i < s.cfg.slots_per_graph; ++i) {
      std::unique_ptr<b200bfs::Slot> sl(new b200bfs::Slot());
      try {
        b200bfs::check_cuda(cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking),
                            "stream");
        b200bfs::batch_reserve(h->e.arena, h->e.g, sl->bs);
      } catch (const b200bfs::Error& x) {
        if (sl->stream) cudaStreamDestroy(sl->stream);
        if (x.code != B200BFS_ERR_OOM || i == 0) {
          h->e.last_error = x.msg;
          fail(x.code);
        }
        break;
      }
      ge->slots.push_back(std::move(sl));
    }
    std::lock_guard<std::mutex> lk(s.mu);
    const int id = (int)s.graphs.size();
    b200bfs::GraphEntry* g = ge.get();
    s.graphs.push_back(std::move(ge));
    for (size_t i = 0; i < g->slots.size(); ++i)
      g->workers.emplace_back(&Server::worker, &s, g, g->slots[i].get(), (int)i);
    *graph_id = id;
  });
}

int b200bfs_server_graph_info(b200bfs_server* p, int graph_id, b200bfs_graph_info* out) {
  return srv_guarded(p, [&](Server& s) {
    b200bfs::GraphEntry* ge;
    {
      std::lock_guard<std::mutex> lk(s.mu);
      ge = graph_of(s, graph_id);
    }
    const int rc = b200bfs_graph_info_get(ge->h, out);
    if (rc != B200BFS_OK) throw b200bfs::Error{rc, b200bfs_last_error(ge->h)};
  });
}

int b200bfs_server_find_roots(b200bfs_server* p, int graph_id, int num_roots, int r1, int r2,
                              int64_t* roots) {
  return srv_guarded(p, [&](Server& s) {
    b200bfs::GraphEntry* ge;
    {
      std::lock_guard<std::mutex> lk(s.mu);
      ge = graph_of(s, graph_id);
    }
    std::lock_guard<std::mutex> dk(ge->decode_mu);
    const int rc = b200bfs_find_roots(ge->h, num_roots, r1, r2, roots);
    if (rc != B200BFS_OK) throw b200bfs::Error{rc, b200bfs_last_error(ge->h)};
  });
}

int b200bfs_server_submit(b200bfs_server* p, int graph_id, int64_t root, int64_t* request_id) {
  return srv_guarded(p, [&](Server& s) {
    srv_require(request_id != nullptr, B200BFS_ERR_INVALID, "null output");
    {
      std::lock_guard<std::mutex> lk(s.mu);
      srv_require(!s.stopping, B200BFS_ERR_STATE, "server stopping");
      b200bfs::GraphEntry* ge = graph_of(s, graph_id);
      srv_require(root >= 0 && root < ge->h->e.g.nverts, B200BFS_ERR_INVALID,
                  "root out of range");
      const int64_t id = s.next_id++;
      b200bfs::Request r;
      r.graph = graph_id;
      r.root = root;
      r.t_submit = b200bfs::now_s();
      if (s.t_first < 0) s.t_first = r.t_submit;
      s.reqs.emplace(id, r);
      ge->pending.push_back(id);
      ++s.submitted;
      *request_id = id;
    }
    s.cv_work.notify_all();
  });
}

int b200bfs_server_poll(b200bfs_server* p, int64_t request_id, b200bfs_request_info* info) {
  return srv_guarded(p, [&](Server& s) {
    std::lock_guard<std::mutex> lk(s.mu);
    auto it = s.reqs.find(request_id);
    srv_require(it != s.reqs.end(), B200BFS_ERR_NOT_FOUND, "unknown request");
    fill_info(it->second, info);
  });
}

int b200bfs_server_wait(b200bfs_server* p, int64_t request_id, double timeout_s,
                        b200bfs_request_info* info) {
  return srv_guarded(p, [&](Server& s) {
    std::unique_lock<std::mutex> lk(s.mu);
    auto finished = [&] {
      auto it = s.reqs.find(request_id);
      return it == s.reqs.end() || it->second.state >= B200BFS_REQ_DONE;
    };
    const auto limit = std::chrono::duration<double>(timeout_s < 0 ? 0 : timeout_s);
    s.cv_done.wait_for(lk, limit, finished);
    auto it = s.reqs.find(request_id);
    srv_require(it != s.reqs.end(), B200BFS_ERR_NOT_FOUND, "unknown request");
    fill_info(it->second, info);
    if (it->second.state < B200BFS_REQ_DONE)
      throw b200bfs::Error{B200BFS_ERR_TIMEOUT, "request not finished"};
  });
}

int b200bfs_server_get_levels(b200bfs_server* p, int64_t request_id, int32_t* levels) {
  return srv_guarded(p, [&](Server& s) {
    srv_require(levels != nullptr, B200BFS_ERR_INVALID, "null output");
    b200bfs::GraphEntry* ge;
    b200bfs::Slot* slot;
    int index;
    {
      std::lock_guard<std::mutex> lk(s.mu);
      auto it = s.reqs.find(request_id);
      srv_require(it != s.reqs.end(), B200BFS_ERR_NOT_FOUND, "unknown request");
      const b200bfs::Request& r = it->second;
      srv_require(r.state == B200BFS_REQ_DONE, B200BFS_ERR_STATE, "request not done");
      srv_require(r.holds, B200BFS_ERR_STATE, "results are not kept (keep_results = 0)");
      ge = graph_of(s, r.graph);
      slot = ge->slots[(size_t)r.slot].get();
      index = r.index;
    }
    // The slot is not reused while this request holds it.
    std::lock_guard<std::mutex> dk(ge->decode_mu);
    b200bfs::Engine& e = ge->h->e;
    cudaSetDevice(e.device);
    b200bfs::batch_select(e.g, e.st, slot->bs, slot->stream, e.sms, index);
    b200bfs::check_cuda(cudaStreamSynchronize(slot->stream), "decode");
    e.have_run = true;
    e.last_root = slot->bs.roots[(size_t)index];
    const int rc = b200bfs_get_levels(ge->h, levels);
    if (rc != B200BFS_OK) throw b200bfs::Error{rc, b200bfs_last_error(ge->h)};
  });
}

int b200bfs_server_release(b200bfs_server* p, int64_t request_id) {
  return srv_guarded(p, [&](Server& s) {
    {
      std::lock_guard<std::mutex> lk(s.mu);
      auto it = s.reqs.find(request_id);
      srv_require(it != s.reqs.end(), B200BFS_ERR_NOT_FOUND, "unknown request");
      b200bfs::Request& r = it->second;
      if (r.holds) {
        b200bfs::GraphEntry* ge = graph_of(s, r.graph);
        b200bfs::Slot* sl = ge->slots[(size_t)r.slot].get();
        if (sl->users > 0) --sl->users;
      }
      if (r.state == B200BFS_REQ_QUEUED) r.state = B200BFS_REQ_CANCELLED;
      s.reqs.erase(it);
    }
    s.cv_work.notify_all();
  });
}

int b200bfs_server_get_stats(b200bfs_server* p, b200bfs_server_stats* out) {
  return srv_guarded(p, [&](Server& s) {
    srv_require(out != nullptr, B200BFS_ERR_INVALID, "null output");
    std::lock_guard<std::mutex> lk(s.mu);
    memset(out, 0, sizeof(*out));
    out->submitted = s.submitted;
    out->completed = s.completed;
    out->failed = s.failed;
    out->batches = s.batches;
    out->mean_batch_size = s.batches ? (double)s.batched_roots / (double)s.batches : 0.0;
    if (!s.lat_ms.empty()) {
      std::vector<double> v = s.lat_ms;
      std::sort(v.begin(), v.end());
      auto pct = [&](double q) {
        const size_t i = (size_t)std::min<double>((double)v.size() - 1, q * (double)(v.size() - 1) + 0.5);
        return v[i];
      };
      out->p50_ms = pct(0.50);
      out->p99_ms = pct(0.99);
      out->max_ms = v.back();
    }
    if (s.t_last > s.t_first && s.t_first >= 0)
      out->bfs_per_s = (double)s.completed / (s.t_last - s.t_first);
    out->device_bytes = s.budget.used.load();
    out->graphs = (int32_t)s.graphs.size();
    for (auto& g : s.graphs) out->slots += (int32_t)g->slots.size();
  });
}

int b200bfs_server_reset_stats(b200bfs_server* p) {
  return srv_guarded(p, [&](Server& s) {
    std::lock_guard<std::mutex> lk(s.mu);
    s.lat_ms.clear();
    s.submitted = s.completed = s.failed = s.batches = s.batched_roots = 0;
    s.t_first = s.t_last = -1;
  });
}

const char* b200bfs_server_last_error(const b200bfs_server* p) {
  return p ? p->s.last_error.c_str() : "null server";
}

int b200bfs_server_stop(b200bfs_server* p) {
  if (!p) return B200BFS_ERR_INVALID;
  Server& s = p->s;
  {
    std::lock_guard<std::mutex> lk(s.mu);
    s.stopping = true;
    for (auto& kv : s.reqs)
      if (kv.second.state == B200BFS_REQ_QUEUED) kv.second.state = B200BFS_REQ_CANCELLED;
  }
  s.cv_work.notify_all();
  s.cv_done.notify_all();
  for (auto& g : s.graphs)
    for (auto& t : g->workers)
      if (t.joinable()) t.join();
  for (auto& g : s.graphs) {
    cudaSetDevice(g->h->e.device);
    for (auto& sl : g->slots) {
      if (sl->stream) cudaStreamSynchronize(sl->stream);
      sl->bs.release(g->h->e.arena);
      if (sl->stream) cudaStreamDestroy(sl->stream);
    }
    b200bfs_destroy(g->h);
  }
  delete p;
  return B200BFS_OK;
}

}  // extern "C"
