// CoreBFS forest pruning on the device.
//
// Restates, for one GPU, the CoreBFS extension of the reference:
//  - prune_trees (external/indexed_bfs/bfs/corebfs/decomposition.hpp:350-572):
//    rounds of leaf peeling.  In a round every vertex with exactly one live
//    neighbour (a leaf) takes that neighbour -- live at the start of the
//    round -- as its tree parent and is removed; the parent loses a
//    neighbour and is removed without a parent once it has none left.  More
//    than 32 rounds abort, like OR_DIE(n_iter <= 32) at :401.
//  - the 2-core left over is the searched graph; it keeps the degree order of
//    the full graph (a monotone renumbering of the live rows), so neighbour
//    lists stay sorted without another sort;
//  - reset_unreachable (mpi/corebfs_adaptor.hpp:228-249,
//    postprocess.hpp:106-154): a search from the highest-degree core vertex
//    marks the giant component; tree vertices whose parent chain does not
//    reach it lose their parent;
//  - run_bfs with CoreBFS (mpi/bfs.hpp:3214-3232): climb from the root to the
//    2-core (bfs_tree_with_callback, corebfs.hpp:125-157), search the core
//    with the climbed distance as level offset, then write the parents of
//    all tree vertices with the unknown level 0xFFFF and the climbed path on
//    top (write_tree_parents, corebfs_adaptor.hpp:285-301).
#include <algorithm>
#include <cstring>
#include <cub/cub.cuh>
#include "common.cuh"
#include "corebfs.h"

namespace b200bfs {
namespace {

__global__ void peel_init_kernel(const int64_t* __restrict__ row_ptr, int64_t R,
                                 int32_t* __restrict__ deg, uint32_t* __restrict__ live,
                                 int64_t W) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < W * 32;
       i += (int64_t)gridDim.x * blockDim.x) {
    const bool ok = i < R;
    if (ok) deg[i] = (int32_t)(row_ptr[i + 1] - row_ptr[i]);
    const unsigned m = __ballot_sync(kFull, ok);
    if (lane_id() == 0) live[i >> 5] = m;
  }
}

__global__ void find_leaves_kernel(const int64_t* __restrict__ row_ptr,
                                   const int32_t* __restrict__ col, const int32_t* __restrict__ deg,
                                   const uint32_t* __restrict__ snap, int64_t R,
                                   int2* __restrict__ leaves, unsigned long long* count) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < R;
       r += (int64_t)gridDim.x * blockDim.x) {
    if (deg[r] != 1) continue;
    int32_t par = -1;
    for (int64_t j = row_ptr[r]; j < row_ptr[r + 1]; ++j) {
      const int32_t u = col[j];
      if ((snap[u >> 5] >> (u & 31)) & 1u) {
        par = u;
        break;
      }
    }
    if (par < 0) continue;  // cannot happen: deg counts live neighbours
    const unsigned long long k = atomicAdd(count, 1ull);
    leaves[k] = make_int2((int32_t)r, par);
  }
}

__global__ void apply_leaves_kernel(const int2* __restrict__ leaves, int64_t n,
                                    const int32_t* __restrict__ inv, int32_t* __restrict__ deg,
                                    uint32_t* __restrict__ live, int32_t* __restrict__ tree_parent) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int2 l = leaves[i];
    deg[l.x] = 0;
    atomicAnd(live + (l.x >> 5), ~(1u << (l.x & 31)));
    tree_parent[inv[l.x]] = inv[l.y];
  }
}

__global__ void apply_parents_kernel(const int2* __restrict__ leaves, int64_t n,
                                     int32_t* __restrict__ deg, uint32_t* __restrict__ live) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t u = leaves[i].y;
    if (deg[u] > 0) {
      if (atomicSub(deg + u, 1) == 1) atomicAnd(live + (u >> 5), ~(1u << (u & 31)));
    }
  }
}

// Live-neighbour count of live rows; 0 for removed rows.
__global__ void core_degree_kernel(const int64_t* __restrict__ row_ptr,
                                   const int32_t* __restrict__ col,
                                   const uint32_t* __restrict__ live, int64_t R,
                                   int32_t* __restrict__ cdeg, int32_t* __restrict__ flag) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = lane_id();
  for (int64_t r = warp; r < R; r += nw) {
    const bool alive = (live[r >> 5] >> (r & 31)) & 1u;
    int64_t cnt = 0;
    if (alive) {
      const int64_t b = row_ptr[r], e = row_ptr[r + 1];
      for (int64_t j = b + lane; j - lane < e; j += 32) {
        bool ok = false;
        if (j < e) {
          const int32_t u = col[j];
          ok = (live[u >> 5] >> (u & 31)) & 1u;
        }
        cnt += __popc(__ballot_sync(kFull, ok));
      }
    }
    if (lane == 0) {
      cdeg[r] = (int32_t)cnt;
      flag[r] = alive ? 1 : 0;
    }
  }
}

__global__ void core_lengths_kernel(const int32_t* __restrict__ cdeg,
                                    const int32_t* __restrict__ flag,
                                    const int32_t* __restrict__ newid, int64_t R,
                                    const int32_t* __restrict__ inv, int64_t* __restrict__ len,
                                    int32_t* __restrict__ cinv, int32_t* __restrict__ cmdeg) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < R;
       r += (int64_t)gridDim.x * blockDim.x) {
    if (!flag[r]) continue;
    const int32_t k = newid[r];
    len[k] = cdeg[r];
    cinv[k] = inv[r];
    cmdeg[k] = cdeg[r];
  }
}

__global__ void core_fill_kernel(const int64_t* __restrict__ row_ptr,
                                 const int32_t* __restrict__ col,
                                 const uint32_t* __restrict__ live,
                                 const int32_t* __restrict__ newid, int64_t R,
                                 const int64_t* __restrict__ crow, int32_t* __restrict__ ccol) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = lane_id();
  for (int64_t r = warp; r < R; r += nw) {
    if (!((live[r >> 5] >> (r & 31)) & 1u)) continue;
    const int64_t b = row_ptr[r], e = row_ptr[r + 1];
    int64_t out = crow[newid[r]];
    for (int64_t j = b + lane; j - lane < e; j += 32) {
      bool ok = false;
      int32_t u = 0;
      if (j < e) {
        u = col[j];
        ok = (live[u >> 5] >> (u & 31)) & 1u;
      }
      const unsigned m = __ballot_sync(kFull, ok);
      if (ok) ccol[out + __popc(m & ((1u << lane) - 1))] = newid[u];
      out += __popc(m);
    }
  }
}

__global__ void core_rank_kernel(const int32_t* __restrict__ old_rank,
                                 const uint32_t* __restrict__ live,
                                 const int32_t* __restrict__ newid, int64_t n,
                                 int32_t* __restrict__ crank) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = old_rank[v];
    crank[v] = (r >= 0 && ((live[r >> 5] >> (r & 31)) & 1u)) ? newid[r] : -1;
  }
}

__global__ void tree_count_kernel(const int32_t* __restrict__ tp, int64_t n, int32_t* __restrict__ f) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x)
    f[v] = tp[v] >= 0 ? 1 : 0;
}

__global__ void tree_list_kernel(const int32_t* __restrict__ tp, const int32_t* __restrict__ pos,
                                 int64_t n, int2* __restrict__ list) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x)
    if (tp[v] >= 0) list[pos[v]] = make_int2((int32_t)v, tp[v]);
}

__global__ void argmax_degree_kernel(const int32_t* __restrict__ mdeg, int64_t R,
                                     unsigned long long* out) {
  unsigned long long best = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < R;
       r += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long k =
        ((unsigned long long)(uint32_t)mdeg[r] << 32) | (0xFFFFFFFFull - (uint64_t)r);
    best = max(best, k);
  }
  for (int o = 16; o; o >>= 1) best = max(best, __shfl_xor_sync(kFull, best, o));
  if (lane_id() == 0) atomicMax(out, best);
}

__global__ void reach_init_kernel(const int64_t* __restrict__ pred, int64_t n,
                                  uint8_t* __restrict__ reach) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x)
    reach[v] = pred[v] != -1;
}

__global__ void reach_step_kernel(const int2* __restrict__ list, int64_t n,
                                  uint8_t* __restrict__ reach, int* changed) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int2 t = list[i];
    if (!reach[t.x] && reach[t.y]) {
      reach[t.x] = 1;
      *changed = 1;
    }
  }
}

__global__ void reach_apply_kernel(const int2* __restrict__ list, int64_t n,
                                   const uint8_t* __restrict__ reach,
                                   int32_t* __restrict__ tree_parent) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int2 t = list[i];
    if (!reach[t.x]) tree_parent[t.x] = -1;
  }
}

__global__ void write_tree_kernel(const int2* __restrict__ list, int64_t n,
                                  int64_t* __restrict__ pred) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int2 t = list[i];
    pred[t.x] = pred_entry(t.y, 0xFFFF);
  }
}

constexpr int kMaxPath = 48;
struct PathArg {
  int n;
  int64_t v[kMaxPath];
  int64_t e[kMaxPath];
};

__global__ void write_path_kernel(PathArg p, int64_t* __restrict__ pred) {
  for (int i = threadIdx.x; i < p.n; i += blockDim.x) pred[p.v[i]] = p.e[i];
}

__global__ void fill_levels_kernel(const int2* __restrict__ list, int64_t n,
                                   int32_t* __restrict__ lv) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int2 t = list[i];
    if (lv[t.x] != 0xFFFF) continue;
    const int32_t lp = lv[t.y];
    if (lp == -1) lv[t.x] = -1;
    else if (lp != 0xFFFF) lv[t.x] = lp + 1;
  }
}

__global__ void has_edge_kernel(const int32_t* __restrict__ rank,
                                const int32_t* __restrict__ tp, int64_t n, int64_t pred_size,
                                uint8_t* __restrict__ out) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < pred_size;
       v += (int64_t)gridDim.x * blockDim.x)
    out[v] = (v < n) && (rank[v] >= 0 || (tp && tp[v] >= 0));
}

void exclusive_scan_i32(DeviceArena& arena, cudaStream_t s, const int32_t* in, int32_t* out,
                        int64_t n) {
  size_t tmp = 0;
  check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, (int)n, s), "scan size");
  void* t = arena.alloc(tmp, "scan temp");
  check_cuda(cub::DeviceScan::ExclusiveSum(t, tmp, in, out, (int)n, s), "scan");
  arena.free(t);
}

int64_t read_i32(const int32_t* p, cudaStream_t s) {
  int32_t v = 0;
  check_cuda(cudaMemcpyAsync(&v, p, 4, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "copy");
  return v;
}

// Rebuilds the tree list (vertex, parent) from tree_parent.
void rebuild_tree_list(DeviceArena& arena, cudaStream_t s, int sms, Graph& g) {
  CoreIndex& k = g.core;
  const int64_t n = g.nverts;
  const int B = 256;
  int32_t* f = arena_alloc<int32_t>(arena, n + 1, "tree flags");
  int32_t* pos = arena_alloc<int32_t>(arena, n + 1, "tree positions");
  tree_count_kernel<<<grid_for(n, B, sms, 16), B, 0, s>>>(k.tree_parent, n, f);
  check_cuda(cudaMemsetAsync(f + n, 0, 4, s), "memset");
  exclusive_scan_i32(arena, s, f, pos, n + 1);
  const int64_t cnt = read_i32(pos + n, s);
  if (k.tree_list) arena.free(k.tree_list);
  k.tree_list = arena_alloc<int2>(arena, cnt, "tree list");
  tree_list_kernel<<<grid_for(n, B, sms, 16), B, 0, s>>>(k.tree_parent, pos, n, k.tree_list);
  k.tree_vertices = cnt;
  k.h_tree_parent.resize(n);
  check_cuda(cudaMemcpyAsync(k.h_tree_parent.data(), k.tree_parent, n * 4,
                             cudaMemcpyDeviceToHost, s),
             "copy tree parents");
  check_cuda(cudaStreamSynchronize(s), "tree list");
  arena.free(f);
  arena.free(pos);
}

}  // namespace

void build_core(DeviceArena& arena, cudaStream_t s, Graph& g, int sms) {
  Csr& c = g.csr;
  CoreIndex& k = g.core;
  const int B = 256;
  const int64_t R = c.nrows, W = (R + 31) / 32, n = g.nverts;
  auto grid = [&](int64_t items) { return grid_for(items, B, sms, 16); };

  k.tree_parent = arena_alloc<int32_t>(arena, n, "tree parents");
  check_cuda(cudaMemsetAsync(k.tree_parent, 0xFF, n * 4, s), "memset");
  int32_t* deg = arena_alloc<int32_t>(arena, R, "peel degree");
  uint32_t* live = arena_alloc<uint32_t>(arena, W, "live bitmap");
  uint32_t* snap = arena_alloc<uint32_t>(arena, W, "live snapshot");
  int2* leaves = arena_alloc<int2>(arena, R, "leaves");
  unsigned long long* cnt = arena_alloc<unsigned long long>(arena, 1, "count");
  peel_init_kernel<<<grid(W * 32), B, 0, s>>>(c.row_ptr, R, deg, live, W);
  int rounds = 0;
  for (int iter = 1;; ++iter) {
    if (iter > 32) throw Error{B200BFS_ERR_OVERFLOW, "CoreBFS needs more than 32 pruning rounds"};
    check_cuda(cudaMemcpyAsync(snap, live, W * 4, cudaMemcpyDeviceToDevice, s), "snapshot");
    check_cuda(cudaMemsetAsync(cnt, 0, 8, s), "memset");
    find_leaves_kernel<<<grid(R), B, 0, s>>>(c.row_ptr, c.col, deg, snap, R, leaves, cnt);
    unsigned long long nl = 0;
    check_cuda(cudaMemcpyAsync(&nl, cnt, 8, cudaMemcpyDeviceToHost, s), "copy");
    check_cuda(cudaStreamSynchronize(s), "leaves");
    if (nl == 0) break;
    rounds = iter;
    apply_leaves_kernel<<<grid(nl), B, 0, s>>>(leaves, (int64_t)nl, c.inv, deg, live,
                                               k.tree_parent);
    apply_parents_kernel<<<grid(nl), B, 0, s>>>(leaves, (int64_t)nl, deg, live);
  }
  k.rounds = rounds;
  arena.free(leaves);
  arena.free(snap);
  arena.free(cnt);

  // The 2-core as a renumbered CSR.
  int32_t* cdeg = deg;  // reuse: live-neighbour counts
  int32_t* flag = arena_alloc<int32_t>(arena, R + 1, "core flags");
  int32_t* newid = arena_alloc<int32_t>(arena, R + 1, "core ids");
  core_degree_kernel<<<grid(R * 32), B, 0, s>>>(c.row_ptr, c.col, live, R, cdeg, flag);
  check_cuda(cudaMemsetAsync(flag + R, 0, 4, s), "memset");
  exclusive_scan_i32(arena, s, flag, newid, R + 1);
  const int64_t Rc = read_i32(newid + R, s);
  if (Rc == 0) throw Error{B200BFS_ERR_INVALID, "the 2-core is empty"};
  Csr k2;
  k2.nrows = Rc;
  int64_t* len = arena_alloc<int64_t>(arena, Rc, "core lengths");
  k2.inv = arena_alloc<int32_t>(arena, Rc, "core inv");
  k2.mdeg = arena_alloc<int32_t>(arena, Rc, "core degree");
  core_lengths_kernel<<<grid(R), B, 0, s>>>(cdeg, flag, newid, R, c.inv, len, k2.inv, k2.mdeg);
  k2.row_ptr = arena_alloc<int64_t>(arena, Rc + 1, "core row ptr");
  check_cuda(cudaMemsetAsync(k2.row_ptr, 0, 8, s), "memset");
  {
    size_t tmp = 0;
    check_cuda(cub::DeviceScan::InclusiveSum(nullptr, tmp, len, k2.row_ptr + 1, (int)Rc, s),
               "scan size");
    void* t = arena.alloc(tmp, "scan temp");
    check_cuda(cub::DeviceScan::InclusiveSum(t, tmp, len, k2.row_ptr + 1, (int)Rc, s), "scan");
    arena.free(t);
  }
  check_cuda(cudaMemcpyAsync(&k2.nedges, k2.row_ptr + Rc, 8, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "core size");
  k2.col = arena_alloc<int32_t>(arena, k2.nedges, "core adjacency");
  core_fill_kernel<<<grid(R * 32), B, 0, s>>>(c.row_ptr, c.col, live, newid, R, k2.row_ptr,
                                              k2.col);
  k2.rank = arena_alloc<int32_t>(arena, n, "core rank");
  core_rank_kernel<<<grid(n), B, 0, s>>>(c.rank, live, newid, n, k2.rank);
  check_cuda(cudaStreamSynchronize(s), "core build");
  k2.max_degree = c.max_degree;
  arena.free(len);
  arena.free(flag);
  arena.free(newid);
  arena.free(deg);
  arena.free(live);
  arena.free(c.row_ptr);
  arena.free(c.col);
  arena.free(c.inv);
  arena.free(c.rank);
  arena.free(c.mdeg);
  arena.free(c.first);
  arena.free(c.first_pair);
  c = k2;
  build_first(arena, s, c, sms);
  k.enabled = true;
  k.core_vertices = Rc;
  rebuild_tree_list(arena, s, sms, g);
}

void free_core(DeviceArena& arena, Graph& g) {
  arena.free(g.core.tree_parent);
  arena.free(g.core.tree_list);
  g.core = CoreIndex();
}

void core_reset_unreachable(DeviceArena& arena, cudaStream_t s, int sms, Graph& g, BfsState& st,
                            int edgefactor, double alpha, double beta, const RunOptions& opt) {
  const int B = 256;
  unsigned long long* best = arena_alloc<unsigned long long>(arena, 1, "argmax");
  check_cuda(cudaMemsetAsync(best, 0, 8, s), "memset");
  argmax_degree_kernel<<<grid_for(g.csr.nrows, B, sms, 8), B, 0, s>>>(g.csr.mdeg, g.csr.nrows,
                                                                      best);
  unsigned long long hb = 0;
  check_cuda(cudaMemcpyAsync(&hb, best, 8, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "argmax");
  arena.free(best);
  const int64_t row = (int64_t)(0xFFFFFFFFull - (hb & 0xFFFFFFFFull));
  int32_t root = 0;
  check_cuda(cudaMemcpyAsync(&root, g.csr.inv + row, 4, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "root");
  int64_t at[9];
  for (auto& x : at) x = -1;
  run_bfs_core(g, st, s, sms, root, 0, edgefactor, alpha, beta, at, opt, nullptr);
  uint8_t* reach = arena_alloc<uint8_t>(arena, g.nverts, "reach");
  int* changed = arena_alloc<int>(arena, 1, "flag");
  reach_init_kernel<<<grid_for(g.nverts, B, sms, 16), B, 0, s>>>(st.pred, g.nverts, reach);
  const int64_t nt = g.core.tree_vertices;
  for (int pass = 0; pass < 64 && nt > 0; ++pass) {
    check_cuda(cudaMemsetAsync(changed, 0, 4, s), "memset");
    reach_step_kernel<<<grid_for(nt, B, sms, 16), B, 0, s>>>(g.core.tree_list, nt, reach, changed);
    int hc = 0;
    check_cuda(cudaMemcpyAsync(&hc, changed, 4, cudaMemcpyDeviceToHost, s), "copy");
    check_cuda(cudaStreamSynchronize(s), "reach");
    if (!hc) break;
  }
  if (nt > 0)
    reach_apply_kernel<<<grid_for(nt, B, sms, 16), B, 0, s>>>(g.core.tree_list, nt, reach,
                                                              g.core.tree_parent);
  arena.free(reach);
  arena.free(changed);
  rebuild_tree_list(arena, s, sms, g);
}

void core_climb(const Graph& g, int64_t root, std::vector<int64_t>& path_v,
                std::vector<int64_t>& path_e, int64_t* entry, int64_t* entry_level) {
  // bfs_tree_with_callback: climb to the 2-core, each vertex taking the
  // previous one as parent at the climbed distance.
  path_v.clear();
  path_e.clear();
  int64_t u = root, p = root, lv = 0;
  const std::vector<int32_t>& tp = g.core.h_tree_parent;
  for (;; ++lv) {
    if ((int)path_v.size() >= kMaxPath) throw Error{B200BFS_ERR_OVERFLOW, "tree climb longer than 48"};
    path_v.push_back(p);
    path_e.push_back(pred_entry(u, lv));
    u = p;
    p = tp[u];
    if (p < 0) break;
  }
  *entry = u;
  *entry_level = lv;
}

int core_write_tree(const Graph& g, int64_t* pred, const std::vector<int64_t>& path_v,
                    const std::vector<int64_t>& path_e, cudaStream_t s, int sms) {
  PathArg path;
  path.n = (int)path_v.size();
  for (int i = 0; i < path.n; ++i) {
    path.v[i] = path_v[(size_t)i];
    path.e[i] = path_e[(size_t)i];
  }
  const int64_t nt = g.core.tree_vertices;
  if (nt > 0)
    write_tree_kernel<<<grid_for(nt, 256, sms, 8), 256, 0, s>>>(g.core.tree_list, nt, pred);
  write_path_kernel<<<1, 64, 0, s>>>(path, pred);
  check_cuda(cudaGetLastError(), "core tree parents");
  return (nt > 0 ? 1 : 0) + 1;
}

constexpr int kMaxRewrite = 2 * kMaxPath;
struct RewriteArg {
  int n;
  int64_t v[kMaxRewrite];
  int64_t e[kMaxRewrite];
};

__global__ void rewrite_kernel(RewriteArg a, int64_t* __restrict__ pred) {
  for (int i = threadIdx.x; i < a.n; i += blockDim.x) pred[a.v[i]] = a.e[i];
}

void core_run_bfs(const Graph& g, BfsState& st, cudaStream_t s, int sms, int64_t root,
                  int edgefactor, double alpha, double beta, int64_t* at, const RunOptions& opt,
                  b200bfs_run_stats* stats) {
  std::vector<int64_t> pv, pe;
  int64_t u = root, lv = 0;
  core_climb(g, root, pv, pe, &u, &lv);
  run_bfs_core(g, st, s, sms, u, lv, edgefactor, alpha, beta, at, opt, stats);
  int launches;
  int64_t bytes;
  if (st.assembled && !st.asm_sparse) {
    // the assembly pass wrote every tree parent with level 0xFFFF: only this
    // climb differs
    RewriteArg a;
    a.n = (int)pv.size();
    for (size_t i = 0; i < pv.size(); ++i) {
      a.v[i] = pv[i];
      a.e[i] = pe[i];
    }
    rewrite_kernel<<<1, 128, 0, s>>>(a, st.pred);
    check_cuda(cudaGetLastError(), "core climb");
    launches = 1;
    bytes = 16 * a.n;
    st.tree_clean = true;
  } else if (!st.assembled && !st.tree_clean) {
    // write_tree_parents (corebfs_adaptor.hpp:285-301): every pruned vertex
    launches = core_write_tree(g, st.pred, pv, pe, s, sms);
    bytes = 16 * g.core.tree_vertices;
    st.tree_clean = true;
  } else {
    // pred already holds every tree parent with level 0xFFFF except on the
    // previous climb (a sparse assembly left the tree parents as they were):
    // put those back (unless on this climb), then this climb
    RewriteArg a;
    a.n = 0;
    const std::vector<int32_t>& tp = g.core.h_tree_parent;
    for (int64_t v : st.prev_path_v) {
      if (tp[(size_t)v] < 0) continue;  // the core entry: handled by the search
      if (std::find(pv.begin(), pv.end(), v) != pv.end()) continue;
      a.v[a.n] = v;
      a.e[a.n] = pred_entry(tp[(size_t)v], 0xFFFF);
      ++a.n;
    }
    for (size_t i = 0; i < pv.size(); ++i) {
      a.v[a.n] = pv[i];
      a.e[a.n] = pe[i];
      ++a.n;
    }
    rewrite_kernel<<<1, 128, 0, s>>>(a, st.pred);
    check_cuda(cudaGetLastError(), "core climb");
    launches = 1;
    bytes = 16 * a.n;
    st.tree_clean = true;
  }
  st.prev_path_v = pv;
  if (stats) {
    stats->algorithmic_bytes += bytes;
    stats->kernel_launches += launches;
  }
}

void core_fill_levels(const Graph& g, const BfsState& st, cudaStream_t s, int sms,
                      int32_t* d_levels) {
  const int64_t nt = g.core.tree_vertices;
  if (nt == 0) return;
  for (int pass = 0; pass <= g.core.rounds + 1; ++pass)
    fill_levels_kernel<<<grid_for(nt, 256, sms, 8), 256, 0, s>>>(g.core.tree_list, nt, d_levels);
}

void has_edge_all(const Graph& g, cudaStream_t s, int sms, uint8_t* d_out) {
  has_edge_kernel<<<grid_for(g.pred_size, 256, sms, 16), 256, 0, s>>>(
      g.csr.rank, g.core.enabled ? g.core.tree_parent : nullptr, g.nverts, g.pred_size, d_out);
}

}  // namespace b200bfs
