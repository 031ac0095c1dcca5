// Graph500 result validation on the device.
//
// Restates BfsValidation::validate (mpi/validate.hpp:607-976) for one GPU,
// stopping at the first group of checks that finds errors, as the reference
// does: value ranges (:994-1016), root is its own parent, no other self-parent,
// the depth map (check_bfs_depth_map_using_predecessors :1145-1254, or
// build_bfs_depth_map :1040-1141 with CoreBFS, which leaves tree levels
// unknown), then one pass over the input edges: endpoint depths must differ
// by at most one or both be unreached, tree edges must match depths
// (check_pred_depth :1018-1034), each reached vertex must have an input edge
// to its parent, and the edges with both endpoints reached are counted
// (edge_visit_count, the TEPS numerator).
#include "common.cuh"
#include "validate.h"
#include "corebfs.h"

namespace b200bfs {
namespace {

__device__ __forceinline__ int64_t parent_of(int64_t x) { return (int64_t)((uint64_t)x << 16) >> 16; }
__device__ __forceinline__ int depth_of(int64_t x) { return (int)(((uint64_t)x >> 48) & 0xFFFF); }
__device__ __forceinline__ int64_t with_depth(int64_t x, int d) {
  return (int64_t)(((uint64_t)x & 0xFFFFFFFFFFFFull) | ((uint64_t)(d & 0xFFFF) << 48));
}

__global__ void max_used_kernel(const uint8_t* __restrict__ has, int64_t n,
                                unsigned long long* out) {
  unsigned long long m = 0;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x)
    if (has[v]) m = max(m, (unsigned long long)v);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
  if (lane_id() == 0 && m) atomicMax(out, m);
}

__global__ void range_kernel(const int64_t* __restrict__ pred, int64_t n, int64_t nglobal,
                             unsigned long long* err) {
  unsigned long long e = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = parent_of(pred[i]);
    if (p < -1 || p >= nglobal) ++e;
  }
  if (e) atomicAdd(err, e);
}

__global__ void self_parent_kernel(const int64_t* __restrict__ pred, int64_t n, int64_t root,
                                   unsigned long long* err) {
  unsigned long long e = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (i != root && parent_of(pred[i]) == i) ++e;
  if (e) atomicAdd(err, e);
}

__global__ void depth_check_kernel(const int64_t* __restrict__ pred, int64_t n, int64_t root,
                                   unsigned long long* err) {
  unsigned long long e = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = pred[i];
    const int64_t p = parent_of(x);
    const int d = depth_of(x);
    if (p == -1 && d != 0xFFFF) ++e;
    else if (p != -1 && d == 0xFFFF) ++e;
    if (i == root) {
      if (d != 0) ++e;
      continue;
    }
    if (p == -1) continue;
    const int dp = depth_of(pred[p]);
    if (dp == 0xFFFF) ++e;
    if (d != dp + 1) ++e;
  }
  if (e) atomicAdd(err, e);
}

__global__ void depth_build_kernel(int64_t* __restrict__ pred, int64_t n, int64_t root,
                                   int* changed) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i == root) continue;
    const int64_t x = pred[i];
    const int64_t p = parent_of(x);
    if (p < 0 || depth_of(x) != 0xFFFF) continue;
    const int dp = depth_of(pred[p]);
    if (dp != 0xFFFF) {
      pred[i] = with_depth(x, dp + 1);
      *changed = 1;
    }
  }
}

__global__ void edge_check_kernel(const uint2* __restrict__ edges, int64_t m, int64_t n,
                                  const int64_t* __restrict__ pred, uint8_t* __restrict__ valid,
                                  unsigned long long* err, unsigned long long* count) {
  unsigned long long e = 0, c = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint2 ed = edges[i];
    const int64_t s = ed.x, t = ed.y;
    if (s >= n || t >= n) {  // endpoint outside pred[]
      ++e;
      continue;
    }
    const int64_t ps = pred[s], pt = pred[t];
    const int sd = depth_of(ps), td = depth_of(pt);
    if (sd != 0xFFFF && td == 0xFFFF) ++e;
    else if (sd == 0xFFFF && td != 0xFFFF) ++e;
    else if (sd - td < -1 || sd - td > 1) ++e;
    else if (sd != 0xFFFF) ++c;
    if (parent_of(ps) == t) {
      if (s != t && td + 1 != sd) ++e;
      valid[s] = 1;
    }
    if (parent_of(pt) == s) {
      if (s != t && sd + 1 != td) ++e;
      valid[t] = 1;
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    e += __shfl_xor_sync(kFull, e, o);
    c += __shfl_xor_sync(kFull, c, o);
  }
  if (lane_id() == 0) {
    if (e) atomicAdd(err, e);
    if (c) atomicAdd(count, c);
  }
}

__global__ void parent_edge_kernel(const int64_t* __restrict__ pred, int64_t n, int64_t root,
                                   const uint8_t* __restrict__ valid, unsigned long long* err) {
  unsigned long long e = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i == root || parent_of(pred[i]) == -1) continue;
    if (!valid[i]) ++e;
  }
  if (e) atomicAdd(err, e);
}

__global__ void set_root_depth_kernel(int64_t* pred, int64_t root) {
  pred[root] = with_depth(pred[root], 0);
}

}  // namespace

void validate_device(DeviceArena& arena, cudaStream_t s, int sms, const Graph& g,
                     const int64_t* pred, bool corebfs, int64_t root, int64_t* errors,
                     int64_t* edge_visit_count) {
  const int B = 256;
  const int64_t n = g.pred_size;
  auto grid = [&](int64_t items) { return grid_for(items, B, sms, 16); };
  if (root < 0 || root >= g.nverts) throw Error{B200BFS_ERR_INVALID, "root out of range"};
  if (!g.input_edges) throw Error{B200BFS_ERR_STATE, "input edges are not resident"};
  unsigned long long* cnt = arena_alloc<unsigned long long>(arena, 4, "validation counters");
  check_cuda(cudaMemsetAsync(cnt, 0, 32, s), "memset");
  // find_max_used_vertex (benchmark_helper.hpp:564-582): nglobalverts = max + 1
  uint8_t* has = arena_alloc<uint8_t>(arena, n, "has_edge");
  has_edge_all(g, s, sms, has);
  max_used_kernel<<<grid(n), B, 0, s>>>(has, n, cnt + 3);
  unsigned long long maxv = 0;
  check_cuda(cudaMemcpyAsync(&maxv, cnt + 3, 8, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "max used");
  arena.free(has);
  const int64_t nglobal = (int64_t)maxv + 1;

  int64_t* p = arena_alloc<int64_t>(arena, n, "pred copy");
  check_cuda(cudaMemcpyAsync(p, pred, n * 8, cudaMemcpyDefault, s), "copy");
  // The checks run in the reference's order and stop at the first that
  // fails (validate.hpp:612-664): value ranges, the root's own parent,
  // other self-parents, the depth map, then the pass over the input edges.
  auto read_errors = [&](const char* what) {
    unsigned long long h = 0;
    check_cuda(cudaMemcpyAsync(&h, cnt, 8, cudaMemcpyDeviceToHost, s), "copy");
    check_cuda(cudaStreamSynchronize(s), what);
    return (int64_t)h;
  };
  *edge_visit_count = 0;
  range_kernel<<<grid(n), B, 0, s>>>(p, n, nglobal, cnt);
  // a root beyond the used vertex range counts as one more range error
  int64_t err = read_errors("validate ranges") + (root >= nglobal ? 1 : 0);
  if (err == 0) {
    int64_t proot = 0;
    check_cuda(cudaMemcpyAsync(&proot, p + root, 8, cudaMemcpyDeviceToHost, s), "copy");
    check_cuda(cudaStreamSynchronize(s), "root entry");
    if (((int64_t)((uint64_t)proot << 16) >> 16) != root) err = 1;
  }
  if (err == 0) {
    self_parent_kernel<<<grid(n), B, 0, s>>>(p, n, root, cnt);
    err = read_errors("validate self parents");
  }
  if (err == 0) {
    if (corebfs) {
      // build_bfs_depth_map (validate.hpp:1040-1141): tree entries take
      // their parent's depth + 1; it reports no errors of its own
      set_root_depth_kernel<<<1, 1, 0, s>>>(p, root);
      int* changed = arena_alloc<int>(arena, 1, "flag");
      for (int pass = 0; pass < 0x10000; ++pass) {
        check_cuda(cudaMemsetAsync(changed, 0, 4, s), "memset");
        depth_build_kernel<<<grid(n), B, 0, s>>>(p, n, root, changed);
        int hc = 0;
        check_cuda(cudaMemcpyAsync(&hc, changed, 4, cudaMemcpyDeviceToHost, s), "copy");
        check_cuda(cudaStreamSynchronize(s), "depth map");
        if (!hc) break;
      }
      arena.free(changed);
    } else {
      depth_check_kernel<<<grid(n), B, 0, s>>>(p, n, root, cnt);
      err = read_errors("validate depth map");
    }
  }
  if (err == 0) {
    uint8_t* valid = arena_alloc<uint8_t>(arena, n, "pred valid");
    check_cuda(cudaMemsetAsync(valid, 0, n, s), "memset");
    edge_check_kernel<<<grid(g.num_input_edges), B, 0, s>>>(g.input_edges, g.num_input_edges, n,
                                                            p, valid, cnt, cnt + 1);
    parent_edge_kernel<<<grid(n), B, 0, s>>>(p, n, root, valid, cnt);
    unsigned long long h2[2] = {0, 0};
    check_cuda(cudaMemcpyAsync(h2, cnt, 16, cudaMemcpyDeviceToHost, s), "copy");
    check_cuda(cudaStreamSynchronize(s), "validate edges");
    arena.free(valid);
    err = (int64_t)h2[0];
    *edge_visit_count = (int64_t)h2[1];
  }
  *errors = err;
  arena.free(p);
  arena.free(cnt);
}

}  // namespace b200bfs
