// BFS entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc: applications whose caching allocator
// owns the device memory (a framework's memory pool that must not be
// bypassed, or that has already reserved nearly all of the GPU), and hosts
// that give a library a fixed device-memory budget at start-up and forbid
// allocations after it.  b200bfs_bfs_noalloc serves them: the caller passes a
// CSR and the output array already on the device, and the search keeps its
// two visited bitmaps and its counter in one file-scope device array of fixed
// size (B200BFS_NOALLOC_MAX_ROWS vertices, 4 MiB of bitmaps), which every GPU
// that loads the library holds until the process exits.
//
// It is the bottom-up step of the engine (bfs.cu, bu_kernel) in a variant
// over caller row ids: every level, each warp owns 32 vertices, each
// unvisited vertex looks for a neighbour visited before the level, and the
// next bitmap word is built with __ballot_sync.  Bottom-up from the first
// level is still a correct BFS on a symmetric CSR (the first level finds the
// root's neighbours), so no frontier queue -- and no more scratch -- is
// needed.  The host reads the level's count after each level, so the call
// synchronises its stream once per level; a stream that is being captured
// into a CUDA graph is refused before anything is enqueued on it.
#include <algorithm>
#include <mutex>
#include "common.cuh"
#include "engine.h"

namespace b200bfs {
namespace {

constexpr int64_t kMaxRows = B200BFS_NOALLOC_MAX_ROWS;
constexpr int64_t kMaxWords = kMaxRows / 32;
// [0, kMaxWords): bitmap A, [kMaxWords, 2 kMaxWords): bitmap B,
// [2 kMaxWords, +2): 64-bit counter of vertices found in the level.
static __device__ __align__(256) uint32_t g_noalloc_scratch[2 * kMaxWords + 64];

struct DeviceScratch {
  bool ready = false;
  uint32_t* ptr = nullptr;
};
std::mutex g_mu;
DeviceScratch g_scratch[256];

__global__ void noalloc_init_kernel(int64_t* __restrict__ pred, int64_t n,
                                    uint32_t* __restrict__ vis0, uint32_t* __restrict__ vis1,
                                    int64_t W) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t i = t0; i < n; i += stride) pred[i] = -1;
  for (int64_t w = t0; w < W; w += stride) {
    const int64_t first = w * 32;
    const uint32_t v = (first + 32 > n) ? ((first >= n) ? kFull : (kFull << (n - first))) : 0u;
    vis0[w] = v;
    vis1[w] = v;
  }
}

__global__ void noalloc_root_kernel(int64_t* pred, uint32_t* vis0, uint32_t* vis1, int64_t root) {
  pred[root] = root;
  vis0[root >> 5] |= 1u << (root & 31);
  vis1[root >> 5] |= 1u << (root & 31);
}

__global__ void __launch_bounds__(256) noalloc_bu_kernel(const uint32_t* __restrict__ cur,
                                                         uint32_t* __restrict__ nxt, int64_t W,
                                                         const int64_t* __restrict__ row_ptr,
                                                         const int32_t* __restrict__ col,
                                                         int64_t* __restrict__ pred, int64_t level,
                                                         int64_t n,
                                                         unsigned long long* __restrict__ found) {
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long total = 0;
  for (int64_t w = gw; w < W; w += nwarps) {
    const uint32_t c = cur[w];
    if (c == kFull) {
      if (lane == 0) nxt[w] = c;
      continue;
    }
    const int64_t v = w * 32 + lane;
    const bool active = ((~c) >> lane) & 1u;
    int64_t b = 0, e = 0;
    int32_t parent = -1;
    if (active) {
      b = row_ptr[v];
      e = row_ptr[v + 1];
      const int64_t lim = min(e, b + (int64_t)8);
      for (; b < lim; ++b) {
        const int32_t u = __ldg(col + b);
        // ids outside [0, n) are ignored rather than read out of the scratch
        if ((uint32_t)u < (uint64_t)n && bit_test(cur, u)) {
          parent = u;
          break;
        }
      }
    }
    unsigned rem = __ballot_sync(kFull, active && parent < 0 && b < e);
    while (rem) {
      const int l = __ffs(rem) - 1;
      rem &= rem - 1;
      const int64_t jb = __shfl_sync(kFull, b, l), je = __shfl_sync(kFull, e, l);
      int32_t p = -1;
      for (int64_t j = jb; j < je; j += 32) {
        const int64_t jj = j + lane;
        int32_t u = 0;
        bool hit = false;
        if (jj < je) {
          u = __ldg(col + jj);
          hit = (uint32_t)u < (uint64_t)n && bit_test(cur, u);
        }
        const unsigned hm = __ballot_sync(kFull, hit);
        if (hm) {
          p = __shfl_sync(kFull, u, __ffs(hm) - 1);
          break;
        }
      }
      if (lane == l) parent = p;
    }
    const unsigned fm = __ballot_sync(kFull, parent >= 0);
    if (lane == 0) {
      nxt[w] = c | fm;
      total += __popc(fm);
    }
    if (parent >= 0) pred[v] = pred_entry(parent, level);
  }
  if (lane == 0 && total) atomicAdd(found, total);
}

}  // namespace
}  // namespace b200bfs

extern "C" int b200bfs_bfs_noalloc(const int64_t* row_ptr, const int32_t* col, int64_t nrows,
                                   int64_t root, int64_t* pred, void* stream,
                                   int32_t* num_levels) {
  using namespace b200bfs;
  if (!row_ptr || !col || !pred) return B200BFS_ERR_INVALID;
  if (nrows < 1 || nrows > kMaxRows) return B200BFS_ERR_INVALID;  // beyond the fixed scratch
  if (root < 0 || root >= nrows) return B200BFS_ERR_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  {
    // The per-level readback and synchronisation are not allowed during
    // stream capture: refuse before enqueuing anything, so that the caller's
    // capture stays intact.
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
      cudaGetLastError();
      return B200BFS_ERR_INVALID;
    }
    if (cs != cudaStreamCaptureStatusNone) return B200BFS_ERR_INVALID;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
    cudaGetLastError();
    return B200BFS_ERR_CUDA;
  }
  uint32_t* scratch = nullptr;
  {
    // Once per device, with that device current: the host-side name of the
    // array is not a device address, so fetch the address the kernels use.
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch[dev].ready) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        return B200BFS_ERR_CUDA;
      }
      g_scratch[dev].ptr = static_cast<uint32_t*>(p);
      g_scratch[dev].ready = true;
    }
    scratch = g_scratch[dev].ptr;
  }
  const int64_t W = (nrows + 31) / 32;
  uint32_t* vis[2] = {scratch, scratch + kMaxWords};
  unsigned long long* found = reinterpret_cast<unsigned long long*>(scratch + 2 * kMaxWords);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int B = 256;
  noalloc_init_kernel<<<grid_for(std::max(nrows, W), B, sms, 8), B, 0, s>>>(pred, nrows, vis[0],
                                                                          vis[1], W);
  noalloc_root_kernel<<<1, 1, 0, s>>>(pred, vis[0], vis[1], root);
  if (cudaGetLastError() != cudaSuccess) return B200BFS_ERR_CUDA;
  int cur = 0;
  int64_t level = 0;
  for (;;) {
    ++level;
    if (level > kMaxLevel) return B200BFS_ERR_OVERFLOW;
    if (cudaMemsetAsync(found, 0, sizeof(unsigned long long), s) != cudaSuccess) break;
    noalloc_bu_kernel<<<grid_for(W * 32, B, sms, 8), B, 0, s>>>(vis[cur], vis[cur ^ 1], W, row_ptr,
                                                                col, pred, level, nrows, found);
    // a launch that failed would leave the count at 0 and end the search
    // early with a partial pred: report it instead
    if (cudaGetLastError() != cudaSuccess) return B200BFS_ERR_CUDA;
    unsigned long long h = 0;
    if (cudaMemcpyAsync(&h, found, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) break;
    if (cudaStreamSynchronize(s) != cudaSuccess) break;
    cur ^= 1;
    if (h == 0) {
      if (num_levels) *num_levels = (int32_t)level;
      return B200BFS_OK;
    }
  }
  cudaGetLastError();
  return B200BFS_ERR_CUDA;
}
