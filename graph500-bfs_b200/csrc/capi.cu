// C ABI of the engine (include/b200bfs.h): handle lifetime, graph input,
// the BfsBase-shaped search calls and error reporting.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include "common.cuh"
#include "bfs_internal.h"
#include "corebfs.h"
#include "validate.h"
#include "autotune.h"
#include "msbfs.h"
#include "engine_state.h"

namespace b200bfs {

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    if (e == cudaErrorMemoryAllocation)
      throw Error{B200BFS_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e)};
    throw Error{B200BFS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
  }
}

void* DeviceArena::alloc(size_t bytes, const char* what) {
  if (bytes == 0) bytes = 16;
  std::lock_guard<std::mutex> lock(mu_);
  if (budget_ && in_use_ + bytes > budget_)
    throw Error{B200BFS_ERR_OOM, std::string("HBM budget exceeded allocating ") + what};
  if (shared_) {
    const uint64_t before = shared_->used.fetch_add(bytes);
    if (shared_->limit && before + bytes > shared_->limit) {
      shared_->used.fetch_sub(bytes);
      throw Error{B200BFS_ERR_OOM, std::string("shared HBM budget exceeded allocating ") + what};
    }
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (shared_) shared_->used.fetch_sub(bytes);
    throw Error{B200BFS_ERR_OOM, std::string("cudaMalloc failed for ") + what + " (" +
                                     std::to_string(bytes) + " bytes)"};
  }
  in_use_ += bytes;
  live_.push_back({p, bytes, seq_++});
  return p;
}

void DeviceArena::free(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(mu_);
  for (size_t i = 0; i < live_.size(); ++i)
    if (live_[i].p == p) {
      in_use_ -= live_[i].bytes;
      if (shared_) shared_->used.fetch_sub(live_[i].bytes);
      live_[i] = live_.back();
      live_.pop_back();
      cudaFree(p);
      return;
    }
}

void DeviceArena::rollback(uint64_t m) {
  std::lock_guard<std::mutex> lock(mu_);
  for (size_t i = 0; i < live_.size();) {
    if (live_[i].seq >= m) {
      in_use_ -= live_[i].bytes;
      if (shared_) shared_->used.fetch_sub(live_[i].bytes);
      cudaFree(live_[i].p);
      live_[i] = live_.back();
      live_.pop_back();
    } else {
      ++i;
    }
  }
}

namespace detail_io {

__global__ void pairs_to_uint2_kernel(const int64_t* __restrict__ in, int64_t n,
                                      uint2* __restrict__ out, int* bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = in[2 * i], b = in[2 * i + 1];
    if (a < 0 || b < 0 || a >= (int64_t(1) << 30) || b >= (int64_t(1) << 30)) *bad = 1;
    out[i] = make_uint2((uint32_t)a, (uint32_t)b);
  }
}

// UnweightedPackedEdge (mpi/primitives.hpp:54-86): v0_low, v1_low,
// high = (v0 >> 32) & 0xFFFF | ((v1 >> 32) & 0xFFFF) << 16.
__global__ void packed_to_uint2_kernel(const uint32_t* __restrict__ in, int64_t n,
                                       uint2* __restrict__ out, int* bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t lo0 = in[3 * i], lo1 = in[3 * i + 1], hi = in[3 * i + 2];
    if (hi != 0 || lo0 >= (1u << 30) || lo1 >= (1u << 30)) *bad = 1;
    out[i] = make_uint2(lo0, lo1);
  }
}

}  // namespace detail_io
using detail_io::pairs_to_uint2_kernel;
using detail_io::packed_to_uint2_kernel;

}  // namespace b200bfs

using b200bfs::Engine;
using b200bfs::Error;


namespace {

template <typename F>
int guarded(b200bfs_handle* h, F&& f) {
  if (!h) return B200BFS_ERR_INVALID;
  try {
    cudaError_t e = cudaSetDevice(h->e.device);
    if (e != cudaSuccess) throw Error{B200BFS_ERR_CUDA, cudaGetErrorString(e)};
    f(h->e);
    return B200BFS_OK;
  } catch (const Error& err) {
    h->e.last_error = err.msg;
    return err.code;
  } catch (const std::bad_alloc&) {
    h->e.last_error = "host out of memory";
    return B200BFS_ERR_OOM;
  }
}

void require(bool cond, int code, const char* msg) {
  if (!cond) throw Error{code, msg};
}

}  // namespace

extern "C" {

int b200bfs_create(const b200bfs_config* cfg, b200bfs_handle** out) {
  if (!out) return B200BFS_ERR_INVALID;
  *out = nullptr;
  int dev = cfg ? cfg->device : 0;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return B200BFS_ERR_CUDA;
  }
  if (dev < 0 || dev >= ndev) return B200BFS_ERR_INVALID;
  b200bfs_handle* h = new (std::nothrow) b200bfs_handle();
  if (!h) return B200BFS_ERR_OOM;
  h->e.device = dev;
  if (cfg) h->e.arena.set_budget(cfg->hbm_budget_bytes);
  int rc = guarded(h, [&](Engine& e) {
    cudaDeviceProp prop;
    b200bfs::check_cuda(cudaGetDeviceProperties(&prop, dev), "device properties");
    e.sms = prop.multiProcessorCount;
    b200bfs::check_cuda(cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking), "stream");
    b200bfs::check_cuda(cudaEventCreate(&e.run_ev[0]), "event");
    b200bfs::check_cuda(cudaEventCreate(&e.run_ev[1]), "event");
  });
  if (rc != B200BFS_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return B200BFS_OK;
}

int b200bfs_destroy(b200bfs_handle* h) {
  if (!h) return B200BFS_ERR_INVALID;
  guarded(h, [&](Engine& e) {
    e.free_graph();
    for (cudaEvent_t& ev : e.run_ev)
      if (ev) cudaEventDestroy(ev);
    if (e.stream) cudaStreamDestroy(e.stream);
    e.stream = nullptr;
  });
  delete h;
  return B200BFS_OK;
}

const char* b200bfs_last_error(const b200bfs_handle* h) {
  return h ? h->e.last_error.c_str() : "null handle";
}

int b200bfs_print_information(b200bfs_handle* h, char* buf, size_t len) {
  return guarded(h, [&](Engine& e) {
    require(buf && len > 0, B200BFS_ERR_INVALID, "null buffer");
    cudaDeviceProp prop;
    b200bfs::check_cuda(cudaGetDeviceProperties(&prop, e.device), "device properties");
    snprintf(buf, len,
             "b200bfs: direction-optimizing BFS on %s (sm_%d%d, %d SMs, %.1f GB HBM), "
             "one device-resident CSR, alpha/beta switch of bfs.hpp:3413-3457",
             prop.name, prop.major, prop.minor, prop.multiProcessorCount,
             prop.totalGlobalMem / 1e9);
  });
}

int b200bfs_build_from_edges(b200bfs_handle* h, const int64_t* edges, int64_t n, int scale,
                             int flags) {
  return guarded(h, [&](Engine& e) {
    require(edges != nullptr && n > 0, B200BFS_ERR_INVALID, "empty edge list");
    require(scale >= 0 && scale <= 30, B200BFS_ERR_INVALID, "scale out of range");
    e.build_guarded([&] {
    uint2* d = b200bfs::arena_alloc<uint2>(e.arena, n, "input edges");
    const int64_t chunk = int64_t(1) << 26;
    int64_t* stage = b200bfs::arena_alloc<int64_t>(e.arena, 2 * std::min(n, chunk), "staging");
    int* bad = b200bfs::arena_alloc<int>(e.arena, 1, "flag");
    b200bfs::check_cuda(cudaMemsetAsync(bad, 0, 4, e.stream), "memset");
    for (int64_t off = 0; off < n; off += chunk) {
      const int64_t c = std::min(chunk, n - off);
      b200bfs::check_cuda(cudaMemcpyAsync(stage, edges + 2 * off, c * 16, cudaMemcpyHostToDevice,
                                          e.stream),
                          "copy edges");
      b200bfs::pairs_to_uint2_kernel<<<b200bfs::grid_for(c, 256, e.sms, 8), 256, 0, e.stream>>>(
          stage, c, d + off, bad);
    }
    int hbad = 0;
    b200bfs::check_cuda(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, e.stream), "copy");
    b200bfs::check_cuda(cudaStreamSynchronize(e.stream), "edges");
    e.arena.free(stage);
    e.arena.free(bad);
    if (hbad) {
      e.arena.free(d);
      throw Error{B200BFS_ERR_INVALID, "vertex id negative or >= 2^30"};
    }
    e.finish_build(d, n, scale, flags);
    });
  });
}

int b200bfs_build_from_packed(b200bfs_handle* h, const uint32_t* packed, int64_t n, int scale,
                              int flags) {
  return guarded(h, [&](Engine& e) {
    require(packed != nullptr && n > 0, B200BFS_ERR_INVALID, "empty edge list");
    require(scale >= 0 && scale <= 30, B200BFS_ERR_INVALID, "scale out of range");
    e.build_guarded([&] {
    uint2* d = b200bfs::arena_alloc<uint2>(e.arena, n, "input edges");
    const int64_t chunk = int64_t(1) << 26;
    uint32_t* stage = b200bfs::arena_alloc<uint32_t>(e.arena, 3 * std::min(n, chunk), "staging");
    int* bad = b200bfs::arena_alloc<int>(e.arena, 1, "flag");
    b200bfs::check_cuda(cudaMemsetAsync(bad, 0, 4, e.stream), "memset");
    for (int64_t off = 0; off < n; off += chunk) {
      const int64_t c = std::min(chunk, n - off);
      b200bfs::check_cuda(cudaMemcpyAsync(stage, packed + 3 * off, c * 12,
                                          cudaMemcpyHostToDevice, e.stream),
                          "copy edges");
      b200bfs::packed_to_uint2_kernel<<<b200bfs::grid_for(c, 256, e.sms, 8), 256, 0, e.stream>>>(
          stage, c, d + off, bad);
    }
    int hbad = 0;
    b200bfs::check_cuda(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, e.stream), "copy");
    b200bfs::check_cuda(cudaStreamSynchronize(e.stream), "edges");
    e.arena.free(stage);
    e.arena.free(bad);
    if (hbad) {
      e.arena.free(d);
      throw Error{B200BFS_ERR_INVALID, "vertex id >= 2^30"};
    }
    e.finish_build(d, n, scale, flags);
    });
  });
}

int b200bfs_generate_graph(b200bfs_handle* h, int scale, int edgefactor, uint64_t seed1,
                           uint64_t seed2, int flags) {
  return guarded(h, [&](Engine& e) {
    require(scale >= 1 && scale <= 30, B200BFS_ERR_INVALID, "scale out of range");
    require(edgefactor >= 1 && edgefactor <= 1024, B200BFS_ERR_INVALID, "bad edgefactor");
    require(!(flags & B200BFS_BUILD_INPUT_SYMMETRIC), B200BFS_ERR_INVALID,
            "generated edges are not symmetric");
    e.build_guarded([&] {
      const int64_t m = (int64_t(1) << scale) * edgefactor;
      uint2* d = b200bfs::arena_alloc<uint2>(e.arena, m, "generated edges");
      b200bfs::check_cuda(b200bfs::launch_generate(scale, seed1, seed2, 0, m, d, e.stream),
                          "generate");
      e.finish_build(d, m, scale, flags);
    });
  });
}

int b200bfs_generate_edges(b200bfs_handle* h, int scale, uint64_t seed1, uint64_t seed2,
                           int64_t start, int64_t end, int64_t* out) {
  return guarded(h, [&](Engine& e) {
    require(out != nullptr && end >= start && start >= 0, B200BFS_ERR_INVALID, "bad range");
    require(scale >= 1 && scale <= 30, B200BFS_ERR_INVALID, "scale out of range");
    const int64_t n = end - start;
    if (n == 0) return;
    const int64_t chunk = int64_t(1) << 26;
    uint2* d = b200bfs::arena_alloc<uint2>(e.arena, std::min(n, chunk), "edges");
    std::vector<uint2> host((size_t)std::min(n, chunk));
    for (int64_t off = 0; off < n; off += chunk) {
      const int64_t c = std::min(chunk, n - off);
      b200bfs::check_cuda(
          b200bfs::launch_generate(scale, seed1, seed2, start + off, start + off + c, d, e.stream),
          "generate");
      b200bfs::check_cuda(
          cudaMemcpyAsync(host.data(), d, c * 8, cudaMemcpyDeviceToHost, e.stream), "copy");
      b200bfs::check_cuda(cudaStreamSynchronize(e.stream), "generate");
      for (int64_t i = 0; i < c; ++i) {
        out[2 * (off + i)] = host[i].x;
        out[2 * (off + i) + 1] = host[i].y;
      }
    }
    e.arena.free(d);
  });
}

int b200bfs_graph_info_get(b200bfs_handle* h, b200bfs_graph_info* out) {
  return guarded(h, [&](Engine& e) {
    require(out != nullptr, B200BFS_ERR_INVALID, "null output");
    require(e.g.built, B200BFS_ERR_STATE, "no graph built");
    memset(out, 0, sizeof(*out));
    out->scale = e.g.scale;
    out->reorder_bits = e.g.reorder_bits;
    out->pred_size = e.g.pred_size;
    out->num_global_edges = e.g.csr.nedges;
    out->num_global_verts = e.g.csr.nrows;
    out->num_rows = e.g.csr.nrows;
    out->num_input_edges = e.g.num_input_edges;
    out->device_bytes = e.g.device_bytes;
    out->corebfs = e.g.core.enabled ? 1 : 0;
    out->prune_rounds = e.g.core.rounds;
    out->core_vertices = e.g.core.enabled ? e.g.core.core_vertices : e.g.csr.nrows;
    out->tree_vertices = e.g.core.tree_vertices;
  });
}

int b200bfs_get_csr(b200bfs_handle* h, int64_t* row_ptr, int32_t* col, int32_t* inv,
                    int32_t* mdeg) {
  return guarded(h, [&](Engine& e) {
    require(e.g.built, B200BFS_ERR_STATE, "no graph built");
    const b200bfs::Csr& c = e.g.csr;
    if (row_ptr)
      b200bfs::check_cuda(cudaMemcpyAsync(row_ptr, c.row_ptr, (c.nrows + 1) * 8,
                                          cudaMemcpyDeviceToHost, e.stream),
                          "copy row_ptr");
    if (col)
      b200bfs::check_cuda(
          cudaMemcpyAsync(col, c.col, c.nedges * 4, cudaMemcpyDeviceToHost, e.stream), "copy col");
    if (inv)
      b200bfs::check_cuda(
          cudaMemcpyAsync(inv, c.inv, c.nrows * 4, cudaMemcpyDeviceToHost, e.stream), "copy inv");
    if (mdeg)
      b200bfs::check_cuda(
          cudaMemcpyAsync(mdeg, c.mdeg, c.nrows * 4, cudaMemcpyDeviceToHost, e.stream),
          "copy mdeg");
    b200bfs::check_cuda(cudaStreamSynchronize(e.stream), "get_csr");
  });
}

int b200bfs_has_edge(b200bfs_handle* h, int64_t v, int* out) {
  return guarded(h, [&](Engine& e) {
    require(out != nullptr, B200BFS_ERR_INVALID, "null output");
    require(e.g.built, B200BFS_ERR_STATE, "no graph built");
    *out = 0;
    if (v < 0 || v >= e.g.nverts) return;
    int32_t r = -1, tp = -1;
    b200bfs::check_cuda(cudaMemcpyAsync(&r, e.g.csr.rank + v, 4, cudaMemcpyDeviceToHost, e.stream),
                        "copy");
    if (e.g.core.enabled)
      b200bfs::check_cuda(cudaMemcpyAsync(&tp, e.g.core.tree_parent + v, 4,
                                          cudaMemcpyDeviceToHost, e.stream),
                          "copy");
    b200bfs::check_cuda(cudaStreamSynchronize(e.stream), "has_edge");
    *out = (r >= 0 || tp >= 0) ? 1 : 0;
  });
}

int b200bfs_has_edge_all(b200bfs_handle* h, uint8_t* out) {
  return guarded(h, [&](Engine& e) {
    require(out != nullptr, B200BFS_ERR_INVALID, "null output");
    require(e.g.built, B200BFS_ERR_STATE, "no graph built");
    uint8_t* d = b200bfs::arena_alloc<uint8_t>(e.arena, e.g.pred_size, "has_edge");
    b200bfs::has_edge_all(e.g, e.stream, e.sms, d);
    b200bfs::check_cuda(
        cudaMemcpyAsync(out, d, e.g.pred_size, cudaMemcpyDeviceToHost, e.stream), "copy");
    b200bfs::check_cuda(cudaStreamSynchronize(e.stream), "has_edge_all");
    e.arena.free(d);
  });
}

int b200bfs_find_roots(b200bfs_handle* h, int num_roots, int r1, int r2, int64_t* roots) {
  return guarded(h, [&](Engine& e) {
    require(roots != nullptr && num_roots > 0, B200BFS_ERR_INVALID, "bad root buffer");
    require(e.g.built, B200BFS_ERR_STATE, "no graph built");
    std::vector<uint8_t> has((size_t)e.g.pred_size);
    uint8_t* d = b200bfs::arena_alloc<uint8_t>(e.arena, e.g.pred_size, "has_edge");
    b200bfs::has_edge_all(e.g, e.stream, e.sms, d);
    b200bfs::check_cuda(
        cudaMemcpyAsync(has.data(), d, e.g.pred_size, cudaMemcpyDeviceToHost, e.stream), "copy");
    b200bfs::check_cuda(cudaStreamSynchronize(e.stream), "find_roots");
    e.arena.free(d);
    b200bfs::find_roots_host(has.data(), int64_t(1) << e.g.scale, num_roots, r1, r2, roots);
  });
}

int b200bfs_prepare(b200bfs_handle* h, int edgefactor, double alpha, double beta) {
  return guarded(h, [&](Engine& e) {
    require(e.g.built, B200BFS_ERR_STATE, "no graph built");
    require(alpha > 0 && beta > 0 && edgefactor > 0, B200BFS_ERR_INVALID, "bad parameters");
    e.prepared = false;
    e.st.allocate(e.arena, e.g);
    try {
      if (e.g.core.enabled) {
        // reads reachability from pred as the level kernels leave it
        b200bfs::RunOptions direct = e.opt;
        direct.pred_assemble = 0;
        b200bfs::core_reset_unreachable(e.arena, e.stream, e.sms, e.g, e.st, edgefactor, alpha,
                                        beta, direct);
      }
      if (b200bfs::use_pred_assembly(e.g, e.opt))
        b200bfs::build_pred_assembly(e.arena, e.g, e.st, e.stream, e.sms);
    } catch (...) {
      cudaStreamSynchronize(e.stream);
      e.st.release(e.arena);
      throw;
    }
    e.prepared = true;
  });
}

int b200bfs_run(b200bfs_handle* h, int64_t root, int edgefactor, double alpha, double beta,
                int64_t* at) {
  return guarded(h, [&](Engine& e) {
    require(e.prepared, B200BFS_ERR_STATE, "prepare_bfs not called");
    require(root >= 0 && root < e.g.nverts, B200BFS_ERR_INVALID, "root out of range");
    require(alpha > 0 && beta > 0 && edgefactor > 0, B200BFS_ERR_INVALID, "bad parameters");
    b200bfs::check_cuda(cudaEventRecord(e.run_ev[0], e.stream), "event");
    b200bfs_run_stats rs;
    if (e.g.core.enabled)
      b200bfs::core_run_bfs(e.g, e.st, e.stream, e.sms, root, edgefactor, alpha, beta, at, e.opt,
                            &rs);
    else
      b200bfs::run_bfs_core(e.g, e.st, e.stream, e.sms, root, 0, edgefactor, alpha, beta, at,
                            e.opt, &rs);
    b200bfs::check_cuda(cudaEventRecord(e.run_ev[1], e.stream), "event");
    b200bfs::check_cuda(cudaEventSynchronize(e.run_ev[1]), "run");
    float ms = 0;
    cudaEventElapsedTime(&ms, e.run_ev[0], e.run_ev[1]);
    b200bfs::finish_run_stats(e.st, &rs);
    rs.device_ms = ms;
    e.last_stats = rs;
    e.have_run = true;
    e.last_root = root;
  });
}

int b200bfs_auto_tune(b200bfs_handle* h, const int64_t* roots, int num_roots,
                      const double* nedge, int edgefactor, double* alpha, double* beta,
                      double* teps) {
  return guarded(h, [&](Engine& e) {
    require(roots && nedge && alpha && beta && num_roots > 0, B200BFS_ERR_INVALID,
            "bad arguments");
    require(e.prepared, B200BFS_ERR_STATE, "prepare_bfs not called");
    require(*alpha > 0 && *beta > 0 && edgefactor > 0, B200BFS_ERR_INVALID, "bad parameters");
    std::vector<int64_t> r(roots, roots + num_roots);
    std::vector<double> ne(nedge, nedge + num_roots);
    for (int64_t v : r)
      require(v >= 0 && v < e.g.nverts, B200BFS_ERR_INVALID, "root out of range");
    auto search = [&](int64_t root, double a, double b, int64_t* at) {
      b200bfs_run_stats rs;
      if (e.g.core.enabled)
        b200bfs::core_run_bfs(e.g, e.st, e.stream, e.sms, root, edgefactor, a, b, at, e.opt, &rs);
      else
        b200bfs::run_bfs_core(e.g, e.st, e.stream, e.sms, root, 0, edgefactor, a, b, at, e.opt,
                              &rs);
    };
    // each search is timed with events on the engine stream
    cudaEvent_t t0, t1;
    b200bfs::check_cuda(cudaEventCreate(&t0), "event");
    b200bfs::check_cuda(cudaEventCreate(&t1), "event");
    b200bfs::SearchFn timed = [&](int64_t root, double a, double b, int64_t* at) {
      b200bfs::check_cuda(cudaEventRecord(t0, e.stream), "event");
      search(root, a, b, at);
      b200bfs::check_cuda(cudaEventRecord(t1, e.stream), "event");
      b200bfs::check_cuda(cudaEventSynchronize(t1), "event");
      float ms = 0;
      cudaEventElapsedTime(&ms, t0, t1);
      return ms / 1e3;
    };
    int tries = 0;
    double t = 0;
    try {
      t = b200bfs::auto_tune(timed, r, ne, edgefactor, alpha, beta, &tries);
    } catch (...) {
      cudaEventDestroy(t0);
      cudaEventDestroy(t1);
      throw;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (teps) *teps = t;
    e.have_run = true;
  });
}

int b200bfs_get_pred(b200bfs_handle* h, int64_t* pred) {
  return guarded(h, [&](Engine& e) {
    require(pred != nullptr, B200BFS_ERR_INVALID, "null output");
    require(e.have_run, B200BFS_ERR_STATE, "no search has run");
    b200bfs::check_cuda(cudaMemcpyAsync(pred, e.st.pred, e.g.pred_size * 8,
                                        cudaMemcpyDeviceToHost, e.stream),
                        "copy pred");
    b200bfs::check_cuda(cudaStreamSynchronize(e.stream), "get_pred");
  });
}

int b200bfs_get_levels(b200bfs_handle* h, int32_t* levels) {
  return guarded(h, [&](Engine& e) {
    require(levels != nullptr, B200BFS_ERR_INVALID, "null output");
    require(e.have_run, B200BFS_ERR_STATE, "no search has run");
    int32_t* d = b200bfs::arena_alloc<int32_t>(e.arena, e.g.pred_size, "levels");
    b200bfs::levels_from_pred(e.st, e.stream, e.sms, d);
    if (e.g.core.enabled) b200bfs::core_fill_levels(e.g, e.st, e.stream, e.sms, d);
    b200bfs::check_cuda(
        cudaMemcpyAsync(levels, d, e.g.pred_size * 4, cudaMemcpyDeviceToHost, e.stream), "copy");
    b200bfs::check_cuda(cudaStreamSynchronize(e.stream), "get_levels");
    e.arena.free(d);
  });
}

int b200bfs_set_option(b200bfs_handle* h, const char* name, int64_t value) {
  return guarded(h, [&](Engine& e) {
    require(name != nullptr, B200BFS_ERR_INVALID, "null option name");
    const std::string n(name);
    if (n == "bu_kernel") {
      require(value >= 1 && value <= 4, B200BFS_ERR_INVALID, "bu_kernel must be 1..4");
      e.opt.bu_kernel = (int)value;
    } else if (n == "td_kernel") {
      require(value >= 1 && value <= 7, B200BFS_ERR_INVALID, "td_kernel must be 1..7");
      e.opt.td_kernel = (int)value;
    } else if (n == "bu_first") {
      require(value == 0 || value == 1, B200BFS_ERR_INVALID, "bu_first must be 0 or 1");
      e.opt.bu_first = (int)value;
    } else if (n == "td_unroll") {
      require(value == 1 || value == 2 || value == 4, B200BFS_ERR_INVALID,
              "td_unroll must be 1, 2 or 4");
      e.opt.td_unroll = (int)value;
    } else if (n == "bu_probe") {
      require(value >= 1 && value <= 64, B200BFS_ERR_INVALID, "bu_probe must be 1..64");
      e.opt.bu_probe = (int)value;
    } else if (n == "single_graph") {
      require(value == 0 || value == 1, B200BFS_ERR_INVALID, "single_graph must be 0 or 1");
      e.opt.single_graph = (int)value;
    } else if (n == "batch_graph") {
      require(value == 0 || value == 1, B200BFS_ERR_INVALID, "batch_graph must be 0 or 1");
      e.opt.batch_graph = (int)value;
    } else if (n == "batch_alpha") {
      require(value >= 1 && value <= 1000000, B200BFS_ERR_INVALID, "batch_alpha must be 1..1e6");
      e.opt.batch_alpha = (double)value;
    } else if (n == "bu_sparse") {
      require(value == 0 || value == 1, B200BFS_ERR_INVALID, "bu_sparse must be 0 or 1");
      e.opt.bu_sparse = (int)value;
    } else if (n == "bu_spec") {
      require(value == 0 || value == 1, B200BFS_ERR_INVALID, "bu_spec must be 0 or 1");
      e.opt.bu_spec = (int)value;
    } else if (n == "force_direction") {
      require(value >= 0 && value <= 2, B200BFS_ERR_INVALID, "force_direction must be 0..2");
      e.opt.force_direction = (int)value;
    } else if (n == "batch_probe") {
      require(value == 4 || value == 8 || value == 16 || value == 32 || value == 64 ||
                  value == 128 || value == 256 || value == 1024,
              B200BFS_ERR_INVALID, "batch_probe must be 4, 8, 16, 32, 64, 128, 256 or 1024");
      e.bs.bu_probe = (int)value;
    } else if (n == "batch_round") {
      require(value == 4 || value == 8, B200BFS_ERR_INVALID, "batch_round must be 4 or 8");
      e.bs.bu_round = (int)value;
    } else if (n == "pred_assemble") {
      require(value == 0 || value == 1, B200BFS_ERR_INVALID, "pred_assemble must be 0 or 1");
      e.opt.pred_assemble = (int)value;
      if (e.prepared && !e.st.pmap && b200bfs::use_pred_assembly(e.g, e.opt))
        b200bfs::build_pred_assembly(e.arena, e.g, e.st, e.stream, e.sms);
    } else {
      throw b200bfs::Error{B200BFS_ERR_INVALID, "unknown option " + n};
    }
  });
}

int b200bfs_get_stream(b200bfs_handle* h, void** stream) {
  return guarded(h, [&](Engine& e) {
    require(stream != nullptr, B200BFS_ERR_INVALID, "null output");
    *stream = (void*)e.stream;
  });
}

int b200bfs_get_level_stats(b200bfs_handle* h, b200bfs_level_stats* out, int max, int* count) {
  return guarded(h, [&](Engine& e) {
    require(count != nullptr && (out != nullptr || max == 0), B200BFS_ERR_INVALID, "null output");
    require(e.prepared && !e.st.levels.empty(), B200BFS_ERR_STATE, "no search has run");
    *count = (int)e.st.levels.size();
    for (int i = 0; i < max && i < *count; ++i) out[i] = e.st.levels[(size_t)i];
  });
}

int b200bfs_get_run_stats(b200bfs_handle* h, b200bfs_run_stats* out) {
  return guarded(h, [&](Engine& e) {
    require(out != nullptr, B200BFS_ERR_INVALID, "null output");
    require(e.have_run, B200BFS_ERR_STATE, "no search has run");
    *out = e.last_stats;
  });
}

int b200bfs_end(b200bfs_handle* h) {
  return guarded(h, [&](Engine& e) {
    if (e.st.allocated) e.st.release(e.arena);
    e.bs.release(e.arena);
    e.prepared = false;
    e.have_run = false;
  });
}

int b200bfs_run_batch(b200bfs_handle* h, const int64_t* roots, int num_roots, int edgefactor,
                      double alpha, double beta, b200bfs_batch_stats* stats) {
  return guarded(h, [&](Engine& e) {
    require(e.prepared, B200BFS_ERR_STATE, "prepare_bfs not called");
    require(roots != nullptr && num_roots >= 1 && num_roots <= B200BFS_BATCH_MAX,
            B200BFS_ERR_INVALID, "num_roots must be 1..64");
    require(beta > 0 && edgefactor > 0, B200BFS_ERR_INVALID, "bad parameters");
    for (int i = 0; i < num_roots; ++i)
      require(roots[i] >= 0 && roots[i] < e.g.nverts, B200BFS_ERR_INVALID, "root out of range");
    b200bfs_batch_stats rs;
    b200bfs::ensure_batch_view(e.arena, e.g, e.stream, e.sms);
    b200bfs::run_batch(e.arena, e.g, e.bs, e.stream, e.sms, roots, num_roots, edgefactor,
                       alpha > 0 ? alpha : e.opt.batch_alpha, beta, e.opt.batch_graph != 0, &rs);
    e.st.levels = e.bs.level_records;
    if (stats) *stats = rs;
    e.have_run = false;
  });
}

int b200bfs_batch_root_levels(b200bfs_handle* h, int64_t* auto_level) {
  return guarded(h, [&](Engine& e) {
    require(auto_level != nullptr, B200BFS_ERR_INVALID, "null output");
    require(e.prepared && e.bs.allocated && e.bs.K > 0, B200BFS_ERR_STATE, "no batch has run");
    for (int i = 0; i < e.bs.K; ++i) {
      const long long L = e.bs.hctl->last_level[i];
      auto_level[i] = L < 0 ? 0 : L + 1;
    }
  });
}

int b200bfs_batch_select(b200bfs_handle* h, int index) {
  return guarded(h, [&](Engine& e) {
    require(e.prepared && e.bs.allocated && e.bs.K > 0, B200BFS_ERR_STATE, "no batch has run");
    require(index >= 0 && index < e.bs.K, B200BFS_ERR_INVALID, "index out of range");
    b200bfs::batch_select(e.g, e.st, e.bs, e.stream, e.sms, index);
    e.have_run = true;
    e.last_root = e.bs.roots[(size_t)index];
  });
}

int b200bfs_validate(b200bfs_handle* h, int64_t root, int64_t* errors, int64_t* edge_visit_count) {
  return guarded(h, [&](Engine& e) {
    require(errors && edge_visit_count, B200BFS_ERR_INVALID, "null output");
    require(e.have_run, B200BFS_ERR_STATE, "no search has run");
    b200bfs::validate_device(e.arena, e.stream, e.sms, e.g, e.st.pred, e.g.core.enabled, root,
                             errors, edge_visit_count);
  });
}

int b200bfs_validate_pred(b200bfs_handle* h, int64_t root, const int64_t* pred, int corebfs,
                          int64_t* errors, int64_t* edge_visit_count) {
  return guarded(h, [&](Engine& e) {
    require(pred && errors && edge_visit_count, B200BFS_ERR_INVALID, "null argument");
    require(e.g.built, B200BFS_ERR_STATE, "no graph");
    b200bfs::validate_device(e.arena, e.stream, e.sms, e.g, pred, corebfs != 0, root, errors,
                             edge_visit_count);
  });
}

}  // extern "C"
