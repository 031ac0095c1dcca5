// Shared device helpers of the B200 BFS engine.
#pragma once

#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <cuda_runtime.h>

namespace b200bfs {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xFFFFFFFFu;
// Levels are stored in the top 16 bits of a pred entry; 0xFFFF is reserved
// for "unknown" (CoreBFS tree vertices), so the deepest searchable level is
// 0xFFFE (mpi/corebfs_adaptor.hpp:51, validate.hpp:982-992).
constexpr int64_t kMaxLevel = 0xFFFE;

__host__ __device__ __forceinline__ int64_t pred_entry(int64_t parent, int64_t level) {
  return (int64_t)(((uint64_t)(level & 0xFFFF) << 48) |
                   ((uint64_t)parent & 0xFFFFFFFFFFFFull));
}

// Blocks of `block` threads of `kernel` resident on one SM (at least 1),
// cached per kernel.  Grid-stride kernels launched with exactly
// blocks_per_sm * SMs blocks run in one wave: a grid larger than what is
// resident leaves the blocks that do not fit for a second, mostly idle
// wave.
template <typename K>
int blocks_per_sm(K kernel, int block) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), block);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, block, 0) != cudaSuccess ||
      n < 1) {
    cudaGetLastError();
    n = 1;
  }
  cache[key] = n;
  return n;
}

// Slot of row v's entry in the buffer a search kernel writes: the row's
// original id (pidx = row -> original id map, the pred array itself), or v
// when pidx is null and the kernel writes the row-order buffer that the
// assembly pass turns into pred.
__device__ __forceinline__ int64_t pred_slot(const int32_t* __restrict__ pidx, int64_t v) {
  return pidx ? (int64_t)__ldg(pidx + v) : v;
}

__device__ __forceinline__ bool bit_test(const uint32_t* bm, int64_t v) {
  return (__ldg(bm + (v >> 5)) >> (v & 31)) & 1u;
}

// Non-returning OR into global memory (compiles to RED.OR).
__device__ __forceinline__ void red_or(uint32_t* p, uint32_t v) { atomicOr(p, v); }

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Largest i in [lo, hi] with qdeg[i] <= t, given qdeg[lo] <= t; every lane
// of the warp gets it.  Each step lets the 32 lanes probe 32 evenly spaced
// entries, so a search over n entries takes log32(n) coalesced rounds.
__device__ __forceinline__ int64_t warp_segment_search(const int64_t* __restrict__ qdeg,
                                                       int64_t lo, int64_t hi, int64_t t) {
  const int lane = lane_id();
  while (hi - lo > 31) {
    const int64_t step = (hi - lo + 31) / 32;
    const int64_t probe = lo + step * lane;
    const unsigned le = __ballot_sync(kFull, probe <= hi && qdeg[probe] <= t);
    const int last = 31 - __clz(le);
    const int64_t next = lo + step * (last + 1);  // first probe known to be > t
    lo += step * last;
    if (last < 31 && next <= hi) hi = next - 1;
  }
  const int64_t probe = lo + lane;
  const unsigned le = __ballot_sync(kFull, probe <= hi && qdeg[probe] <= t);
  return lo + (31 - __clz(le));
}

// Grid size helper: a multiple of the SM count times resident blocks.
inline int grid_for(int64_t work_items, int block, int sms, int per_sm = 8) {
  int64_t need = (work_items + block - 1) / block;
  int64_t cap = (int64_t)sms * per_sm;
  if (need < 1) need = 1;
  return (int)(need < cap ? need : cap);
}

}  // namespace b200bfs
