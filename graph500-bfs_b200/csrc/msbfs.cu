// Batched multi-source direction-optimizing BFS (up to 64 roots).
//
// The reference runs one root per BfsBase::run_bfs call (main.cc:610-640).
// Here up to 64 roots share one traversal.  State per searched row v:
//   seen[2v]       uint64, bit k set once root k has reached v; seen[2v + 1]
//                  holds the bits the top-down push found for v in the current
//                  level until the merge pass moves them (same 16 bytes, so a
//                  push's probe and OR touch one sector);
//   planes[L][v]   uint64, bit k set iff level_k(v) == L (the bit-sliced
//                  level array of the batch; it is also the frontier of
//                  level L).
// Each root keeps its own direction, decided with the reference's switch
// rule (bfs.hpp:3413-3457) on that root's frontier: roots in top-down mode
// are expanded by an edge-balanced push over the rows whose plane has one of
// their bits (batch_td_kernel), roots in bottom-up mode are found by one
// shared pull sweep (batch_bu_kernel) in which every row with unseen
// bottom-up bits reads its neighbours' frontier masks, highest-degree
// neighbours first, until all those bits are found or the row is exhausted.
// One adjacency read serves every root that needs it.
//
// The plan of each level (masks, plane pointers, queue size) lives in a
// device control block written by batch_control_kernel, so the launch
// sequence of a level does not depend on host decisions; the host loop only
// reads back whether to continue.
#include <algorithm>
#include <cstring>
#include <cub/cub.cuh>
#include "common.cuh"
#include "corebfs.h"
#include "msbfs.h"

namespace b200bfs {
namespace {

constexpr int kQThreads = 256;
constexpr int kBTile = 256;                      // adjacency entries per warp tile (top-down)
constexpr int64_t kSampleHead = 32768;           // rows always counted in the per-root statistics
constexpr int kSampleStride = 64;                // then one 32-row chunk in 64

__device__ __forceinline__ unsigned long long warp_or64(unsigned long long x) {
  const unsigned lo = __reduce_or_sync(kFull, (unsigned)x);
  const unsigned hi = __reduce_or_sync(kFull, (unsigned)(x >> 32));
  return ((unsigned long long)hi << 32) | lo;
}

__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}

__device__ __forceinline__ unsigned long long* plane_ptr(const BatchCtl* c, long long L) {
  return c->planes + L * c->R;
}

__device__ __forceinline__ uint32_t* rowbits_of(const BatchCtl* c, long long L) {
  return c->rowbits + L * c->wstride;
}

// Zero-fills p[0, n) with 16-byte stores from thread t0 of a grid of
// `stride` threads (p is 8-byte aligned: a plane starts at L * R words).
__device__ __forceinline__ void zero_u64(unsigned long long* __restrict__ p, int64_t n,
                                         int64_t t0, int64_t stride) {
  const int64_t head = ((uintptr_t)p & 15) ? 1 : 0;
  if (n <= 0) return;
  if (head && t0 == 0) p[0] = 0ull;
  ulonglong2* q = reinterpret_cast<ulonglong2*>(p + head);
  const int64_t n2 = (n - head) >> 1;
  for (int64_t i = t0; i < n2; i += stride) q[i] = make_ulonglong2(0ull, 0ull);
  if (((n - head) & 1) && t0 == 0) p[n - 1] = 0ull;
}

// Level start of a level without a bottom-up sweep: zeroes the rows of the
// level's plane that its bitmap marks (what an earlier batch left there) and
// the bitmap, for the top-down push to OR into.  A bottom-up sweep does the
// same for its own rows.  Each lane reads one bitmap word (a warp reads 32
// consecutive words); the warp then zeroes the 32-row block (256 bytes) of
// each marked word together, one row per lane.
__global__ void batch_clear_kernel(const BatchCtl* __restrict__ ctl) {
  if (ctl->has_bu) return;
  const long long L = ctl->level;
  const int64_t R = ctl->R;
  const int64_t W = (R + 31) >> 5;
  uint32_t* __restrict__ rb = rowbits_of(ctl, L);
  unsigned long long* __restrict__ cur = plane_ptr(ctl, L);
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = gw * 32; base < W; base += nwarps * 32) {
    const int64_t w = base + lane;
    const uint32_t bits = w < W ? rb[w] : 0u;
    unsigned marked = __ballot_sync(kFull, bits != 0);
    if (bits) rb[w] = 0u;
    while (marked) {
      const int l = __ffs(marked) - 1;
      marked &= marked - 1;
      // a marked word may cover rows past R (a pool marked whole)
      const int64_t v = (base + l) * 32 + lane;
      if (v < R) cur[v] = 0ull;
    }
  }
}

// Queue pass 1 (top-down levels): per-block count and degree sum of the rows
// whose previous plane holds a top-down root.  Only rows marked in the
// previous level's touched-row bitmap can, so the pass reads that bitmap
// (one bit per row) and the plane entries of its set bits.  One thread per
// bitmap word; a tile of kQThreads words gives one partial, and a block
// takes tiles blockIdx.x, blockIdx.x + gridDim.x, ... (a one-wave grid: the
// kernel runs at every level and returns at once on bottom-up-only ones).
__global__ void __launch_bounds__(kQThreads) batch_queue_count_kernel(
    const BatchCtl* __restrict__ ctl, const int64_t* __restrict__ row_ptr,
    int64_t* __restrict__ blk_cnt, int64_t* __restrict__ blk_deg, int64_t ntiles) {
  if (!ctl->has_td) return;
  const long long L = ctl->level;
  const int64_t W = (ctl->R + 31) >> 5;
  const unsigned long long T = ctl->td_mask;
  const unsigned long long* __restrict__ prev = plane_ptr(ctl, L - 1);
  const uint32_t* __restrict__ rb = rowbits_of(ctl, L - 1);
  __shared__ int64_t s_c[kQThreads / 32], s_d[kQThreads / 32];
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t w = tile * kQThreads + threadIdx.x;
    int64_t cnt = 0, deg = 0;
    uint32_t bits = w < W ? rb[w] : 0u;
    while (bits) {
      const int64_t v = w * 32 + __ffs(bits) - 1;
      bits &= bits - 1;
      if (prev[v] & T) {
        ++cnt;
        deg += row_ptr[v + 1] - row_ptr[v];
      }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      cnt += __shfl_xor_sync(kFull, cnt, o);
      deg += __shfl_xor_sync(kFull, deg, o);
    }
    if (lane_id() == 0) {
      s_c[threadIdx.x >> 5] = cnt;
      s_d[threadIdx.x >> 5] = deg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t a = 0, b = 0;
      for (int i = 0; i < kQThreads / 32; ++i) {
        a += s_c[i];
        b += s_d[i];
      }
      blk_cnt[tile] = a;
      blk_deg[tile] = b;
    }
    __syncthreads();
  }
}

__device__ __forceinline__ void warp_scan2(int64_t& a, int64_t& b) {
  const int lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t ta = __shfl_up_sync(kFull, a, o);
    const int64_t tb = __shfl_up_sync(kFull, b, o);
    if (lane >= o) {
      a += ta;
      b += tb;
    }
  }
}

// Queue pass 2: exclusive scan of the block partials (one block).
__global__ void __launch_bounds__(1024) batch_queue_scan_kernel(BatchCtl* __restrict__ ctl,
                                                                int64_t* __restrict__ blk_cnt,
                                                                int64_t* __restrict__ blk_deg,
                                                                int64_t nblk,
                                                                int64_t* __restrict__ qdeg) {
  if (!ctl->has_td) return;
  __shared__ int64_t s_a[32], s_b[32];
  const int t = threadIdx.x;
  const int64_t per = (nblk + blockDim.x - 1) / blockDim.x;
  const int64_t lo = min(nblk, t * per), hi = min(nblk, lo + per);
  int64_t a = 0, b = 0;
  for (int64_t i = lo; i < hi; ++i) {
    a += blk_cnt[i];
    b += blk_deg[i];
  }
  int64_t ia = a, ib = b;
  warp_scan2(ia, ib);
  const int wid = t >> 5, lane = lane_id();
  if (lane == 31) {
    s_a[wid] = ia;
    s_b[wid] = ib;
  }
  __syncthreads();
  if (wid == 0) {
    int64_t xa = s_a[lane], xb = s_b[lane];
    warp_scan2(xa, xb);
    s_a[lane] = xa;
    s_b[lane] = xb;
  }
  __syncthreads();
  int64_t ea = ia - a + (wid ? s_a[wid - 1] : 0);
  int64_t eb = ib - b + (wid ? s_b[wid - 1] : 0);
  for (int64_t i = lo; i < hi; ++i) {
    const int64_t ca = blk_cnt[i], cb = blk_deg[i];
    blk_cnt[i] = ea;
    blk_deg[i] = eb;
    ea += ca;
    eb += cb;
  }
  if (t == blockDim.x - 1) {
    ctl->c.qsize = (unsigned long long)s_a[31];
    ctl->c.qedges = (unsigned long long)s_b[31];
    qdeg[s_a[31]] = s_b[31];
  }
}

// Queue pass 3: queue rows (in row order) and their degree prefix; tiles as
// in pass 1.
__global__ void __launch_bounds__(kQThreads) batch_queue_write_kernel(
    const BatchCtl* __restrict__ ctl, const int64_t* __restrict__ row_ptr,
    const int64_t* __restrict__ blk_cnt, const int64_t* __restrict__ blk_deg,
    int32_t* __restrict__ queue, int64_t* __restrict__ qdeg, int64_t ntiles) {
  if (!ctl->has_td) return;
  const long long L = ctl->level;
  const int64_t W = (ctl->R + 31) >> 5;
  const unsigned long long T = ctl->td_mask;
  const unsigned long long* __restrict__ prev = plane_ptr(ctl, L - 1);
  const uint32_t* __restrict__ rb = rowbits_of(ctl, L - 1);
  __shared__ int64_t s_c[kQThreads / 32], s_d[kQThreads / 32];
  const int wid = threadIdx.x >> 5;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t w = tile * kQThreads + threadIdx.x;
    uint32_t take = 0;
    int64_t cnt = 0, deg = 0;
    {
      uint32_t bits = w < W ? rb[w] : 0u;
      while (bits) {
        const int b = __ffs(bits) - 1;
        bits &= bits - 1;
        const int64_t v = w * 32 + b;
        if (prev[v] & T) {
          take |= 1u << b;
          ++cnt;
          deg += row_ptr[v + 1] - row_ptr[v];
        }
      }
    }
    int64_t ic = cnt, id = deg;
    warp_scan2(ic, id);
    if (lane_id() == 31) {
      s_c[wid] = ic;
      s_d[wid] = id;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t a = 0, b = 0;
      for (int i = 0; i < kQThreads / 32; ++i) {
        const int64_t xa = s_c[i], xb = s_d[i];
        s_c[i] = a;
        s_d[i] = b;
        a += xa;
        b += xb;
      }
    }
    __syncthreads();
    int64_t pos = blk_cnt[tile] + s_c[wid] + ic - cnt;
    int64_t dpos = blk_deg[tile] + s_d[wid] + id - deg;
    while (take) {
      const int64_t v = w * 32 + __ffs(take) - 1;
      take &= take - 1;
      const int64_t d = row_ptr[v + 1] - row_ptr[v];
      queue[pos] = (int32_t)v;
      qdeg[pos] = dpos;
      ++pos;
      dpos += d;
    }
    __syncthreads();
  }
}

// Top-down push for the roots in td_mask: edge-balanced over the queue rows
// (each warp takes kBTile adjacency entries of the concatenated rows).  For
// an edge (u, v) the bits m = planes[L-1][u] & td_mask not yet in seen[2v]
// nor in this level's new bits seen[2v + 1] are ORed (non-returning) into
// seen[2v + 1], and v is marked in the touched-row bitmap; batch_merge_kernel
// then moves the new bits into planes[L] and seen.  Both words of v are in
// one 16-byte pair, so the probe and the OR touch one sector.  A stale pair
// (bits set during the level) only costs a redundant OR.  Runs after the
// bottom-up sweep of the level, which only writes bottom-up roots' bits.
__global__ void __launch_bounds__(256) batch_td_kernel(
    BatchCtl* __restrict__ ctl, const int32_t* __restrict__ queue,
    const int64_t* __restrict__ qdeg, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ col) {
  if (!ctl->has_td) return;
  const int64_t qsize = (int64_t)ctl->c.qsize;
  if (qsize == 0) return;
  const long long L = ctl->level;
  const unsigned long long T = ctl->td_mask;
  const unsigned long long* __restrict__ prev = plane_ptr(ctl, L - 1);
  unsigned long long* seen = ctl->seen;
  uint32_t* rb = rowbits_of(ctl, L);
  const int64_t total = qdeg[qsize];
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t ntiles = (total + kBTile - 1) / kBTile;
  unsigned long long found = 0;
  for (int64_t tile = gw; tile < ntiles; tile += nwarps) {
    const int64_t t0 = tile * kBTile;
    int64_t i = warp_segment_search(qdeg, 0, qsize - 1, t0);
    int64_t seg_lo = qdeg[i], seg_hi = qdeg[i + 1];
    int32_t src = queue[i];
    int64_t rbeg = row_ptr[src];
    unsigned long long f = prev[src] & T;
#pragma unroll 1
    for (int k = 0; k < kBTile / 32; ++k) {
      const int64_t e = t0 + k * 32 + lane;
      if (e >= total) break;
      while (e >= seg_hi && i + 1 < qsize) {
        ++i;
        seg_lo = seg_hi;
        seg_hi = qdeg[i + 1];
        src = queue[i];
        rbeg = row_ptr[src];
        f = prev[src] & T;
      }
      const int32_t u = __ldg(col + rbeg + (e - seg_lo));
      // L2 read of the pair: it changes during the kernel
      const ulonglong2 x = __ldcg(reinterpret_cast<const ulonglong2*>(seen) + u);
      const unsigned long long m = f & ~(x.x | x.y);
      if (m) {
        atomicOr(seen + 2 * (int64_t)u + 1, m);
        // the bitmap is L2-resident; most rows are marked by an earlier
        // edge, and a read costs less than an atomic
        const uint32_t bit = 1u << (u & 31);
        if (!(__ldcg(rb + (u >> 5)) & bit)) atomicOr(rb + (u >> 5), bit);
        found |= m;
      }
    }
  }
  found = warp_or64(found);
  if (lane == 0 && found) atomicOr(&ctl->c.active, found);
}

// After the top-down push: for every row of the level's touched-row bitmap,
// the bits the push left in seen[2v + 1] are ORed into planes[L][v] (which
// may hold the bottom-up sweep's bits of other roots) and seen[2v], and
// seen[2v + 1] is cleared.  A warp reads 32 bitmap words and then handles
// the 32 rows of each marked word together, one row per lane.
__global__ void __launch_bounds__(256) batch_merge_kernel(BatchCtl* __restrict__ ctl) {
  if (!ctl->has_td) return;
  const long long L = ctl->level;
  const int64_t R = ctl->R;
  const int64_t W = (R + 31) >> 5;
  const uint32_t* __restrict__ rb = rowbits_of(ctl, L);
  unsigned long long* __restrict__ cur = plane_ptr(ctl, L);
  ulonglong2* __restrict__ pair = reinterpret_cast<ulonglong2*>(ctl->seen);
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = gw * 32; base < W; base += nwarps * 32) {
    const int64_t w = base + lane;
    const uint32_t bits = w < W ? __ldcg(rb + w) : 0u;
    unsigned marked = __ballot_sync(kFull, bits != 0);
    while (marked) {
      const int l = __ffs(marked) - 1;
      marked &= marked - 1;
      const uint32_t word = __shfl_sync(kFull, bits, l);
      const int64_t v = (base + l) * 32 + lane;
      if (v < R && ((word >> lane) & 1u)) {
        const ulonglong2 x = pair[v];
        if (x.y) {
          cur[v] |= x.y;
          pair[v] = make_ulonglong2(x.x | x.y, 0ull);
        }
      }
    }
  }
}

// Bottom-up pull for the roots in bu_mask_active.  A warp owns 32
// consecutive rows (one per lane).  A lane whose row misses some of those
// roots (U = ~seen & mask) ORs the frontier masks planes[L-1][u] of its
// neighbours, up to kProbe of them kPer loads at a time, until every bit of
// U is found; rows still open after that (long lists) are swept by the whole
// warp, 32 neighbours per step, stopping as soon as U is covered.  The warp
// sweep serves one row at a time, so most rows are best finished by their
// own lane (kProbe 128 measured fastest).  Rows are sorted by
// descending degree, so neighbour lists start with the hubs, which most
// roots reach first.  The row's new bits are written to planes[L] and seen
// by the lane that owns it, before the top-down push of the level ORs into
// planes[L]: no atomics.  A warp's 32 rows are one word of the plane's
// bitmap of possibly non-zero rows; the warp writes its rows when it found
// bits or the word marks some (left by an earlier batch), so the plane holds
// exactly this level afterwards, and the word becomes the rows found.
// The frontier masks of level L-1 are only read here, and a bit of U can
// only come from a neighbour at level L-1 of that root, so the OR over
// neighbours is exact.
// first (may be null): the rows' first neighbours; an open row ORs its first
// neighbour's mask (one coalesced read of first[] per warp) before loading
// its row offsets, which it then needs only if that mask does not cover U.
// Launched with 5 blocks per SM, all resident (at most 51 registers): the
// sweep is bound by load latency on the sparser levels, and 5 blocks measured
// faster than 4 (SCALE 28 64-root batch 22.4 against 22.7 ms) and 6 (23.4 ms,
// with spills at 40 registers).
template <int kProbe, int kPer>
__global__ void __launch_bounds__(256, 5) batch_bu_kernel(BatchCtl* __restrict__ ctl,
                                                       const int64_t* __restrict__ row_ptr,
                                                       const int32_t* __restrict__ col,
                                                       const int32_t* __restrict__ first) {
  if (!ctl->has_bu) return;
  const long long L = ctl->level;
  const int64_t R = ctl->R;
  const unsigned long long Bm = ctl->bu_mask_active;
  const unsigned long long* __restrict__ prev = plane_ptr(ctl, L - 1);
  unsigned long long* __restrict__ cur = plane_ptr(ctl, L);
  unsigned long long* __restrict__ seen = ctl->seen;
  uint32_t* __restrict__ rb = rowbits_of(ctl, L);
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t nchunks = (R + 31) >> 5;
  unsigned long long found = 0, scanned = 0, rows = 0;
  // the seen masks and bitmap word of the warp's next chunk are loaded one
  // chunk ahead (only this warp writes them), so a chunk without work costs
  // no exposed load latency
  unsigned long long s_next = ~0ull;
  uint32_t d_next = 0;
  if (gw < nchunks) {
    const int64_t v0 = gw * 32 + lane;
    s_next = v0 < R ? seen[2 * v0] : ~0ull;
    d_next = rb[gw];
  }
  for (int64_t ch = gw; ch < nchunks; ch += nwarps) {
    const int64_t v = ch * 32 + lane;
    const bool valid = v < R;
    const uint32_t dirty = d_next;
    const unsigned long long s = s_next;
    if (ch + nwarps < nchunks) {
      const int64_t vn = v + nwarps * 32;
      s_next = vn < R ? seen[2 * vn] : ~0ull;
      d_next = rb[ch + nwarps];
    }
    const unsigned long long U = ~s & Bm;
    const unsigned work = __ballot_sync(kFull, U != 0);
    if (!work) {
      if (valid && dirty) cur[v] = 0ull;
      if (lane == 0 && dirty) rb[ch] = 0u;
      continue;
    }
    rows += (lane == 0) ? __popc(work) : 0;
    unsigned long long acc = 0;
    int64_t j = 0, e = 0;
    if (first) {
      if (U) {
        acc = __ldg(prev + __ldg(first + v));
        scanned += 1;
        if ((acc & U) != U) {
          j = row_ptr[v] + 1;
          e = row_ptr[v + 1];
        }
      }
    } else if (U) {
      j = row_ptr[v];
      e = row_ptr[v + 1];
    }
#pragma unroll 1
    for (int p = 0; p < kProbe; p += kPer) {
      const bool need = (acc & U) != U && j < e;
      if (!__any_sync(kFull, need)) break;
      if (need) {
        // kPer neighbour ids, then their masks (entries beyond the row
        // repeat the first)
        const int64_t r = e - j;
        int32_t u[kPer];
#pragma unroll
        for (int q = 0; q < kPer; ++q) u[q] = (q == 0 || r > q) ? __ldg(col + j + q) : u[0];
        unsigned long long m = 0;
#pragma unroll
        for (int q = 0; q < kPer; ++q) m |= __ldg(prev + u[q]);
        acc |= m;
        const int64_t t = r < kPer ? r : kPer;
        j += t;
        scanned += t;
      }
    }
    unsigned rem = __ballot_sync(kFull, (acc & U) != U && j < e);
    while (rem) {
      const int l = __ffs(rem) - 1;
      rem &= rem - 1;
      const int64_t jb = __shfl_sync(kFull, j, l), je = __shfl_sync(kFull, e, l);
      const unsigned long long Ul = __shfl_sync(kFull, U, l);
      unsigned long long al = __shfl_sync(kFull, acc, l);
      int64_t jj = jb;
      while (jj < je) {
        const int64_t x = jj + lane;
        unsigned long long m = 0;
        if (x < je) m = __ldg(prev + __ldg(col + x));
        al |= warp_or64(m);
        jj += 32;
        if ((al & Ul) == Ul) break;
      }
      if (lane == l) {
        acc = al;
        scanned += (unsigned long long)(min(jj, je) - jb);
      }
    }
    const unsigned long long n = acc & U;
    const unsigned hit = __ballot_sync(kFull, n != 0);
    // whole 256-byte blocks: partial sector writes cost DRAM reads
    if (valid && (hit || dirty)) cur[v] = n;
    if (valid && hit) seen[2 * v] = s | n;
    if (lane == 0 && (hit || dirty)) rb[ch] = hit;
    found |= n;
  }
  found = warp_or64(found);
  scanned = warp_sum64(scanned);
  if (lane == 0) {
    if (found) atomicOr(&ctl->c.active, found);
    if (scanned) atomicAdd(&ctl->c.scanned_bu, scanned);
    if (rows) atomicAdd(&ctl->c.rows_bu, rows);
  }
}

// Per-root frontier size and pre-dedup degree sum of level L, the inputs of
// the switch rule.  They only steer the direction (levels do not depend on
// them), so they are estimated: the first kSampleHead rows (the hubs, which
// carry most of the degree mass) are counted exactly, the rest through one
// 32-row chunk in kSampleStride, weighted by kSampleStride.
__global__ void __launch_bounds__(256) batch_stats_kernel(BatchCtl* __restrict__ ctl,
                                                          const int32_t* __restrict__ mdeg) {
  __shared__ unsigned long long s_cnt[kBatchMax], s_edg[kBatchMax];
  if (threadIdx.x < kBatchMax) {
    s_cnt[threadIdx.x] = 0;
    s_edg[threadIdx.x] = 0;
  }
  __syncthreads();
  const long long L = ctl->level;
  const int64_t R = ctl->R;
  const unsigned long long* __restrict__ cur = plane_ptr(ctl, L);
  const int64_t head = R < kSampleHead ? R : kSampleHead;
  const int64_t head_w = (head + 31) >> 5;
  const int64_t tail_w =
      R > head ? (R - head + 32 * kSampleStride - 1) / (32 * kSampleStride) : 0;
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  // lane j accumulates roots j and j + 32 in registers
  unsigned long long c_lo = 0, c_hi = 0, e_lo = 0, e_hi = 0;
  for (int64_t w = gw; w < head_w + tail_w; w += nwarps) {
    int64_t v;
    unsigned long long wt;
    if (w < head_w) {
      v = w * 32 + lane;
      wt = 1;
    } else {
      v = head + (w - head_w) * 32 * kSampleStride + lane;
      wt = kSampleStride;
    }
    const unsigned long long n = v < R ? cur[v] : 0ull;
    unsigned long long any = warp_or64(n);
    if (!any) continue;
    const unsigned d = v < R ? (unsigned)min(mdeg[v], 1 << 26) : 0u;
    while (any) {
      const int k = __ffsll((long long)any) - 1;
      any &= any - 1;
      const bool b = (n >> k) & 1ull;
      const unsigned c = __popc(__ballot_sync(kFull, b));
      const unsigned ds = __reduce_add_sync(kFull, b ? d : 0u);
      if (lane == (k & 31)) {
        if (k < 32) {
          c_lo += (unsigned long long)c * wt;
          e_lo += (unsigned long long)ds * wt;
        } else {
          c_hi += (unsigned long long)c * wt;
          e_hi += (unsigned long long)ds * wt;
        }
      }
    }
  }
  if (c_lo) {
    atomicAdd(&s_cnt[lane], c_lo);
    atomicAdd(&s_edg[lane], e_lo);
  }
  if (c_hi) {
    atomicAdd(&s_cnt[lane + 32], c_hi);
    atomicAdd(&s_edg[lane + 32], e_hi);
  }
  __syncthreads();
  if (threadIdx.x < kBatchMax && s_cnt[threadIdx.x]) {
    atomicAdd(&ctl->c.cnt[threadIdx.x], s_cnt[threadIdx.x]);
    atomicAdd(&ctl->c.edg[threadIdx.x], s_edg[threadIdx.x]);
  }
}

// Closes level L = ctl->level and plans level L + 1 (one thread).
//  - roots whose entry level is L (L = 0, or the CoreBFS climb length) are
//    seeded into planes[L] and seen;
//  - the level is recorded;
//  - each root with a frontier applies the reference's switch rule to its
//    own frontier (bfs.hpp:3413-3457): top-down -> bottom-up when its
//    frontier grew and its edge count exceeds num_global_edges / alpha,
//    bottom-up -> top-down when it shrank below
//    num_global_verts / (beta * edgefactor * 2); a root seeded in this
//    level is not tested, as the reference does not test level 0;
//  - done = 1 when no root has a frontier and none is still to enter,
//    2 when planes[L + 1] is not allocated, 3 past level 0xFFFE.
// With a graph conditional handle it also sets the loop condition.
// One thread per root (kBatchMax threads): each seeds and tests its own
// root; the mask updates are gathered in shared memory and thread 0 plans
// the next level.
__global__ void __launch_bounds__(kBatchMax) batch_control_kernel(
    BatchCtl* __restrict__ ctl, const int32_t* __restrict__ mdeg,
    cudaGraphConditionalHandle cond, int use_cond) {
  __shared__ unsigned long long s_seeded, s_entered, s_bu_set, s_bu_clr, s_grow_clr;
  BatchCtl& c = *ctl;
  const int k = threadIdx.x;
  const unsigned long long bit = 1ull << k;
  const long long L = c.level;
  if (k == 0) s_seeded = s_entered = s_bu_set = s_bu_clr = s_grow_clr = 0;
  __syncthreads();
  const unsigned long long pending = c.pending;
  if ((pending & bit) && c.root_lv[k] == L) {
    atomicOr(&s_entered, bit);
    const int r = c.root_row[k];
    if (r >= 0) {
      atomicOr(plane_ptr(ctl, L) + r, bit);
      atomicOr(c.seen + 2 * (int64_t)r, bit);
      atomicOr(rowbits_of(ctl, L) + (r >> 5), 1u << (r & 31));
      atomicOr(&s_seeded, bit);
    }
  }
  __syncthreads();
  const unsigned long long seeded = s_seeded;
  const unsigned long long act = c.c.active | seeded;
  if ((act & ~seeded) & bit) {
    const long long e_thr = (long long)(c.nedges / c.alpha);
    const long long n_thr = (long long)(c.nverts / (c.beta * c.edgefactor * 2.0));
    const long long n = (long long)c.c.cnt[k], e = (long long)c.c.edg[k];
    const unsigned long long bu = c.bu_mask;
    if ((c.growing & bit) && n > c.prev_cnt[k]) {
      if (!(bu & bit) && e > e_thr) atomicOr(&s_bu_set, bit);
    } else if (bu & bit) {
      if (n < n_thr) {
        atomicOr(&s_bu_clr, bit);
        atomicOr(&s_grow_clr, bit);
      }
    }
    c.prev_cnt[k] = n;
  }
  if (seeded & bit) c.prev_cnt[k] = 0;
  if (act & bit) c.last_level[k] = L;
  __syncthreads();
  if (k == 0) {
    c.pending = pending & ~s_entered;
    c.c.active = act;
    if (L < kBatchHist) {
      BatchLevelRec& h = c.hist[L];
      h.td_roots = c.has_td ? c.td_mask : 0ull;
      h.bu_roots = c.has_bu ? c.bu_mask_active : 0ull;
      h.active = act;
      h.scanned_bu = c.c.scanned_bu;
      h.rows_bu = c.c.rows_bu;
      h.qsize = c.has_td ? c.c.qsize : 0ull;
      h.qedges = c.has_td ? c.c.qedges : 0ull;
    }
    const unsigned long long bu_mask = (c.bu_mask | s_bu_set) & ~s_bu_clr;
    c.bu_mask = bu_mask;
    c.growing &= ~s_grow_clr;
    int done = 0;
    if (act == 0 && c.pending == 0) {
      done = 1;
    } else if (L + 1 > kMaxLevel) {
      done = 3;
    } else {
      c.level = L + 1;
      c.td_mask = act & ~bu_mask;
      c.bu_mask_active = act & bu_mask;
      c.has_td = c.td_mask != 0;
      c.has_bu = c.bu_mask_active != 0;
      if (L + 1 >= c.capacity) done = 2;
    }
    c.done = done;
    if (use_cond) cudaGraphSetConditional(cond, done == 0 ? 1u : 0u);
  }
  __syncthreads();
  // the next level's counters start at zero (not when the search stops:
  // the host reads them)
  if (c.done == 0 || c.done == 2) {
    c.c.cnt[k] = 0;
    c.c.edg[k] = 0;
    if (k == 0) {
      c.c.active = 0;
      c.c.scanned_bu = 0;
      c.c.rows_bu = 0;
      c.c.qsize = 0;
      c.c.qedges = 0;
    }
  }
}

struct BatchSetupArg {
  unsigned long long* planes;
  unsigned long long* seen;
  uint32_t* rowbits;
  long long wstride;
  long long R, capacity, nedges, nverts;
  double alpha, beta;
  int edgefactor, K;
  long long v[kBatchMax];  // entry vertex of each root (original id)
  int lv[kBatchMax];       // its level
  // planes[0] is zero except at the rows the previous batch seeded there
  // (clear[0..nclear)); full_clear when that is not known (new pool, failed
  // batch), which also marks every row of the other planes as possibly
  // non-zero
  int full_clear, nclear;
  int clear[kBatchMax];
};

// seen = 0, planes[0] = 0 and the touched-row bitmap of level 0 = 0.  Only
// seeding writes planes[0], so after a batch it holds bits at that batch's
// level-0 root rows alone, and clearing those rows restores it.  With
// full_clear the bitmaps of planes 1 .. capacity-1 are set to all rows.
__global__ void batch_zero_kernel(const BatchSetupArg* __restrict__ a) {
  const int64_t n = a->R;
  unsigned long long* __restrict__ seen = a->seen;
  unsigned long long* __restrict__ p0 = a->planes;
  uint32_t* __restrict__ rb = a->rowbits;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool full = a->full_clear != 0;
  zero_u64(seen, 2 * n, t0, stride);
  if (full) zero_u64(p0, n, t0, stride);
  if (!full && t0 < a->nclear) p0[a->clear[t0]] = 0ull;
  for (int64_t i = t0; i < ((n + 31) >> 5); i += stride) rb[i] = 0u;
  if (full)
    for (int64_t i = a->wstride + t0; i < a->capacity * a->wstride; i += stride) rb[i] = ~0u;
}

// Initialises the control block for a new batch (64 threads).
__global__ void batch_setup_kernel(BatchCtl* __restrict__ ctl, const BatchSetupArg* __restrict__ ap,
                                   const int32_t* __restrict__ rank,
                                   const int32_t* __restrict__ b_of_row, int64_t nverts) {
  const BatchSetupArg& a = *ap;
  const int t = threadIdx.x;
  if (t < kBatchMax) {
    const bool ok = t < a.K && a.v[t] >= 0 && a.v[t] < nverts;
    int row = ok ? rank[a.v[t]] : -1;
    if (row >= 0 && b_of_row) row = b_of_row[row];
    ctl->root_row[t] = row;
    ctl->root_lv[t] = t < a.K ? a.lv[t] : 0;
    ctl->prev_cnt[t] = 0;
    ctl->last_level[t] = -1;
  }
  if (t == 0) {
    ctl->planes = a.planes;
    ctl->seen = a.seen;
    ctl->rowbits = a.rowbits;
    ctl->wstride = a.wstride;
    ctl->R = a.R;
    ctl->capacity = a.capacity;
    ctl->nedges = a.nedges;
    ctl->nverts = a.nverts;
    ctl->alpha = a.alpha;
    ctl->beta = a.beta;
    ctl->edgefactor = a.edgefactor;
    ctl->K = a.K;
    const unsigned long long all = a.K >= 64 ? ~0ull : ((1ull << a.K) - 1);
    ctl->level = 0;
    ctl->td_mask = 0;
    ctl->bu_mask_active = 0;
    ctl->has_td = 0;
    ctl->has_bu = 0;
    ctl->done = 0;
    ctl->bu_mask = 0;
    ctl->growing = all;
    ctl->pending = all;
    memset(&ctl->c, 0, sizeof(BatchCounters));
  }
}

// Points the control block at a larger plane pool and resumes the search.
__global__ void batch_pool_kernel(BatchCtl* ctl, unsigned long long* planes, uint32_t* rowbits,
                                  long long capacity) {
  ctl->planes = planes;
  ctl->rowbits = rowbits;
  ctl->capacity = capacity;
  ctl->done = 0;
}

// Level of root k for every row (-1: not reached), from the planes.
__global__ void batch_row_levels_kernel(const unsigned long long* __restrict__ planes, int64_t R,
                                        int64_t nplanes, int k, int32_t* __restrict__ out) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < R;
       v += (int64_t)gridDim.x * blockDim.x) {
    int32_t lv = -1;
    for (int64_t L = 0; L < nplanes; ++L)
      if ((planes[L * R + v] >> k) & 1ull) {
        lv = (int32_t)L;
        break;
      }
    out[v] = lv;
  }
}

__global__ void fill_minus_one_kernel(int64_t* __restrict__ p, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = -1;
}

// pred of one root from its row levels: the entry row is its own parent,
// every other reached row takes its first neighbour one level nearer.
__global__ void batch_parent_kernel(const int32_t* __restrict__ lv, int64_t R,
                                    const int64_t* __restrict__ row_ptr,
                                    const int32_t* __restrict__ col,
                                    const int32_t* __restrict__ inv, int root_row,
                                    int64_t* __restrict__ pred, int* __restrict__ missing) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < R;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t L = lv[v];
    if (L < 0) continue;
    const int64_t me = inv[v];
    if (v == root_row) {
      pred[me] = pred_entry(me, L);
      continue;
    }
    bool found = false;
    for (int64_t j = row_ptr[v], e = row_ptr[v + 1]; j < e; ++j) {
      const int32_t u = col[j];
      if (lv[u] == L - 1) {
        pred[me] = pred_entry(inv[u], L);
        found = true;
        break;
      }
    }
    if (!found) atomicExch(missing, 1);
  }
}

__global__ void set_entry_kernel(int64_t* p, int64_t i, int64_t value) { p[i] = value; }

}  // namespace

namespace {

// Batch view of a group-reordered graph: rows renumbered in the global
// degree order (the order the neighbour lists already follow).
__global__ void bview_keys_kernel(const int32_t* __restrict__ mdeg, const int32_t* __restrict__ inv,
                                  int64_t R, uint64_t* __restrict__ keys,
                                  int32_t* __restrict__ rows) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < R;
       r += (int64_t)gridDim.x * blockDim.x) {
    keys[r] = ((uint64_t)(0xFFFFFFFFu - (uint32_t)mdeg[r]) << 32) | (uint32_t)inv[r];
    rows[r] = (int32_t)r;
  }
}

__global__ void bview_maps_kernel(const int32_t* __restrict__ order, int64_t R,
                                  const int32_t* __restrict__ inv,
                                  const int32_t* __restrict__ mdeg,
                                  const int64_t* __restrict__ row_ptr,
                                  int32_t* __restrict__ b_of_row, int32_t* __restrict__ binv,
                                  int32_t* __restrict__ bmdeg, int64_t* __restrict__ blen) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < R;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = order[k];
    b_of_row[r] = (int32_t)k;
    binv[k] = inv[r];
    bmdeg[k] = mdeg[r];
    blen[k] = row_ptr[r + 1] - row_ptr[r];
  }
}

// Warp per view row: copies its list with the neighbours renumbered.
__global__ void bview_copy_kernel(const int32_t* __restrict__ order, int64_t R,
                                  const int64_t* __restrict__ row_ptr,
                                  const int32_t* __restrict__ col,
                                  const int32_t* __restrict__ b_of_row,
                                  const int64_t* __restrict__ brow_ptr,
                                  int32_t* __restrict__ bcol) {
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = gw; k < R; k += nwarps) {
    const int32_t r = order[k];
    const int64_t b = row_ptr[r], e = row_ptr[r + 1], o = brow_ptr[k];
    for (int64_t j = b + lane; j < e; j += 32) bcol[o + (j - b)] = b_of_row[col[j]];
  }
}

}  // namespace

void ensure_batch_view(DeviceArena& arena, Graph& g, cudaStream_t s, int sms) {
  if (!g.group_reorder || g.bview_built) return;
  const Csr& c = g.csr;
  const int64_t R = c.nrows;
  const int B = 256;
  uint64_t* k1 = arena_alloc<uint64_t>(arena, R, "view keys");
  uint64_t* k2 = arena_alloc<uint64_t>(arena, R, "view keys");
  int32_t* r1 = arena_alloc<int32_t>(arena, R, "view rows");
  int32_t* order = arena_alloc<int32_t>(arena, R, "view order");
  bview_keys_kernel<<<grid_for(R, B, sms, 8), B, 0, s>>>(c.mdeg, c.inv, R, k1, r1);
  size_t tmp = 0;
  check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k1, k2, r1, order, (int)R, 0, 64, s),
             "view sort size");
  void* t = arena.alloc(tmp, "view sort temp");
  check_cuda(cub::DeviceRadixSort::SortPairs(t, tmp, k1, k2, r1, order, (int)R, 0, 64, s),
             "view sort");
  arena.free(t);
  arena.free(k1);
  arena.free(k2);
  arena.free(r1);
  Csr v;
  v.nrows = R;
  v.nedges = c.nedges;
  v.max_degree = c.max_degree;
  g.b_of_row = arena_alloc<int32_t>(arena, R, "view row map");
  v.inv = arena_alloc<int32_t>(arena, R, "view inv");
  v.mdeg = arena_alloc<int32_t>(arena, R, "view mdeg");
  int64_t* blen = arena_alloc<int64_t>(arena, R, "view row lengths");
  bview_maps_kernel<<<grid_for(R, B, sms, 8), B, 0, s>>>(order, R, c.inv, c.mdeg, c.row_ptr,
                                                        g.b_of_row, v.inv, v.mdeg, blen);
  v.row_ptr = arena_alloc<int64_t>(arena, R + 1, "view row ptr");
  check_cuda(cudaMemsetAsync(v.row_ptr, 0, 8, s), "memset");
  tmp = 0;
  check_cuda(cub::DeviceScan::InclusiveSum(nullptr, tmp, blen, v.row_ptr + 1, (int)R, s),
             "view scan size");
  t = arena.alloc(tmp, "view scan temp");
  check_cuda(cub::DeviceScan::InclusiveSum(t, tmp, blen, v.row_ptr + 1, (int)R, s), "view scan");
  arena.free(t);
  arena.free(blen);
  v.col = arena_alloc<int32_t>(arena, c.nedges, "view adjacency");
  bview_copy_kernel<<<grid_for(R * 32, B, sms, 8), B, 0, s>>>(order, R, c.row_ptr, c.col,
                                                               g.b_of_row, v.row_ptr, v.col);
  build_first(arena, s, v, sms, false);
  check_cuda(cudaStreamSynchronize(s), "batch view");
  arena.free(order);
  g.bview = v;
  g.bview_built = true;
}

void free_batch_view(DeviceArena& arena, Graph& g) {
  if (!g.bview_built) return;
  arena.free(g.bview.row_ptr);
  arena.free(g.bview.col);
  arena.free(g.bview.inv);
  arena.free(g.bview.mdeg);
  arena.free(g.bview.first);
  arena.free(g.b_of_row);
  g.bview = Csr();
  g.b_of_row = nullptr;
  g.bview_built = false;
}

cudaEvent_t BatchState::event(size_t i) {
  while (ev.size() <= i) {
    cudaEvent_t e;
    check_cuda(cudaEventCreate(&e), "event");
    ev.push_back(e);
  }
  return ev[i];
}

void BatchState::release(DeviceArena& arena) {
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  ev.clear();
  plane0_clean = false;
  plane0_rows.clear();
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  if (graph) cudaGraphDestroy(graph);
  graph_exec = nullptr;
  graph = nullptr;
  graph_key.clear();
  if (!allocated) return;
  arena.free(d_arg);
  cudaFreeHost(h_arg);
  d_arg = h_arg = nullptr;
  arena.free(planes);
  arena.free(seen);
  arena.free(rowbits);
  arena.free(queue);
  arena.free(qdeg);
  queue = nullptr;
  qdeg = nullptr;
  arena.free(blk_cnt);
  arena.free(blk_deg);
  arena.free(ctl);
  cudaFreeHost(hctl);
  cudaFreeHost(hdone);
  planes = seen = nullptr;
  rowbits = nullptr;
  blk_cnt = blk_deg = nullptr;
  ctl = nullptr;
  hctl = nullptr;
  hdone = nullptr;
  capacity = 0;
  allocated = false;
  K = 0;
  levels = 0;
}

namespace {

void batch_allocate(DeviceArena& arena, const Graph& g, BatchState& bs) {
  bs.release(arena);
  bs.R = g.csr.nrows;
  const int64_t W = (bs.R + 31) / 32;
  bs.nblk = (W + kQThreads - 1) / kQThreads;
  // (seen, new bits of the level) pairs, see batch_td_kernel
  bs.seen = arena_alloc<unsigned long long>(arena, 2 * bs.R, "batch seen masks");
  bs.wstride = (W + 4) & ~(int64_t)3;
  bs.queue = arena_alloc<int32_t>(arena, bs.R + 1, "batch frontier queue");
  bs.qdeg = arena_alloc<int64_t>(arena, bs.R + 2, "batch frontier degree prefix");
  bs.blk_cnt = arena_alloc<int64_t>(arena, bs.nblk + 1, "batch block counts");
  bs.blk_deg = arena_alloc<int64_t>(arena, bs.nblk + 1, "batch block degrees");
  bs.ctl = arena_alloc<BatchCtl>(arena, 1, "batch control block");
  check_cuda(cudaMallocHost(&bs.hctl, sizeof(BatchCtl)), "pinned batch control");
  check_cuda(cudaMallocHost(&bs.hdone, sizeof(int)), "pinned flag");
  bs.d_arg = arena_alloc<BatchSetupArg>(arena, 1, "batch arguments");
  check_cuda(cudaMallocHost(&bs.h_arg, sizeof(BatchSetupArg)), "pinned batch arguments");
  bs.allocated = true;
  // Level planes: 16 to start with (Kronecker searches need about 10),
  // fewer when memory is short; the search grows the pool when it runs out.
  for (int64_t cap = 16;; cap /= 2) {
    unsigned long long* p = nullptr;
    try {
      p = arena_alloc<unsigned long long>(arena, cap * bs.R, "batch level planes");
      bs.rowbits = arena_alloc<uint32_t>(arena, cap * bs.wstride, "batch touched-row bitmaps");
      bs.planes = p;
      bs.capacity = cap;
      break;
    } catch (const Error& e) {
      arena.free(p);
      if (e.code != B200BFS_ERR_OOM || cap <= 2) throw;
    }
  }
}

// Doubles the plane pool, keeping planes [0, used).
void batch_grow(DeviceArena& arena, BatchState& bs, int64_t used, cudaStream_t s) {
  const int64_t cap = bs.capacity * 2;
  unsigned long long* np = arena_alloc<unsigned long long>(arena, cap * bs.R, "batch level planes");
  uint32_t* nr = nullptr;
  try {
    nr = arena_alloc<uint32_t>(arena, cap * bs.wstride, "batch touched-row bitmaps");
  } catch (...) {
    arena.free(np);
    throw;
  }
  check_cuda(cudaMemcpyAsync(np, bs.planes, (size_t)used * bs.R * 8, cudaMemcpyDeviceToDevice, s),
             "copy planes");
  // the bitmaps of the kept planes come along; the new planes are garbage,
  // so every row of theirs is marked
  check_cuda(cudaMemcpyAsync(nr, bs.rowbits, (size_t)used * bs.wstride * 4,
                             cudaMemcpyDeviceToDevice, s),
             "copy bitmaps");
  check_cuda(cudaMemsetAsync(nr + used * bs.wstride, 0xFF, (size_t)(cap - used) * bs.wstride * 4, s),
             "mark new planes");
  batch_pool_kernel<<<1, 1, 0, s>>>(bs.ctl, np, nr, cap);
  check_cuda(cudaStreamSynchronize(s), "grow planes");
  arena.free(bs.planes);
  arena.free(bs.rowbits);
  bs.planes = np;
  bs.rowbits = nr;
  bs.capacity = cap;
}

}  // namespace

namespace {

// The kernels of one level, in order.  With events, records the level's
// start, end of queue building, end of the bottom-up sweep and end of the
// top-down push at ev[0..3].
void launch_level(const Graph& g, BatchState& bs, cudaStream_t s, int sms,
                  cudaGraphConditionalHandle cond, int use_cond, const cudaEvent_t* ev) {
  const Csr& c = batch_csr(g);
  const int B = 256;
  const int64_t ntiles = std::max<int64_t>(bs.nblk, 1);
  const unsigned qc_grid = (unsigned)std::min<int64_t>(
      ntiles, (int64_t)sms * blocks_per_sm(batch_queue_count_kernel, kQThreads));
  const unsigned qw_grid = (unsigned)std::min<int64_t>(
      ntiles, (int64_t)sms * blocks_per_sm(batch_queue_write_kernel, kQThreads));
  if (ev) check_cuda(cudaEventRecord(ev[0], s), "event");
  batch_clear_kernel<<<grid_for(bs.R, B, sms, 8), B, 0, s>>>(bs.ctl);
  batch_queue_count_kernel<<<qc_grid, kQThreads, 0, s>>>(bs.ctl, c.row_ptr, bs.blk_cnt, bs.blk_deg,
                                                        ntiles);
  batch_queue_scan_kernel<<<1, 1024, 0, s>>>(bs.ctl, bs.blk_cnt, bs.blk_deg, bs.nblk, bs.qdeg);
  batch_queue_write_kernel<<<qw_grid, kQThreads, 0, s>>>(bs.ctl, c.row_ptr, bs.blk_cnt,
                                                        bs.blk_deg, bs.queue, bs.qdeg, ntiles);
  if (ev) check_cuda(cudaEventRecord(ev[1], s), "event");
  auto bu = batch_bu_kernel<128, 4>;
  switch (bs.bu_probe * 16 + bs.bu_round) {
    case 4 * 16 + 4: bu = batch_bu_kernel<4, 4>; break;
    case 8 * 16 + 4: bu = batch_bu_kernel<8, 4>; break;
    case 16 * 16 + 4: bu = batch_bu_kernel<16, 4>; break;
    case 32 * 16 + 4: bu = batch_bu_kernel<32, 4>; break;
    case 64 * 16 + 4: bu = batch_bu_kernel<64, 4>; break;
    case 256 * 16 + 4: bu = batch_bu_kernel<256, 4>; break;
    case 1024 * 16 + 4: bu = batch_bu_kernel<1024, 4>; break;
    case 8 * 16 + 8: bu = batch_bu_kernel<8, 8>; break;
    case 16 * 16 + 8: bu = batch_bu_kernel<16, 8>; break;
    case 32 * 16 + 8: bu = batch_bu_kernel<32, 8>; break;
    case 64 * 16 + 8: bu = batch_bu_kernel<64, 8>; break;
    case 128 * 16 + 8: bu = batch_bu_kernel<128, 8>; break;
    default: break;
  }
  bu<<<sms * 5, B, 0, s>>>(bs.ctl, c.row_ptr, c.col, c.first);
  if (ev) check_cuda(cudaEventRecord(ev[2], s), "event");
  batch_td_kernel<<<sms * blocks_per_sm(batch_td_kernel, B), B, 0, s>>>(bs.ctl, bs.queue, bs.qdeg,
                                                                      c.row_ptr, c.col);
  batch_merge_kernel<<<sms * blocks_per_sm(batch_merge_kernel, B), B, 0, s>>>(bs.ctl);
  if (ev) check_cuda(cudaEventRecord(ev[3], s), "event");
  batch_stats_kernel<<<sms * blocks_per_sm(batch_stats_kernel, B), B, 0, s>>>(bs.ctl, c.mdeg);
  batch_control_kernel<<<1, kBatchMax, 0, s>>>(bs.ctl, c.mdeg, cond, use_cond);
}
constexpr int kLevelLaunches = 9;

void launch_prologue(const Graph& g, BatchState& bs, cudaStream_t s, int sms) {
  batch_zero_kernel<<<grid_for(bs.R, 256, sms, 8), 256, 0, s>>>(
      static_cast<const BatchSetupArg*>(bs.d_arg));
  batch_setup_kernel<<<1, kBatchMax, 0, s>>>(bs.ctl, static_cast<const BatchSetupArg*>(bs.d_arg),
                                             g.csr.rank, g.b_of_row, g.nverts);
}

std::vector<const void*> graph_key_of(const Graph& g, const BatchState& bs, int sms) {
  const Csr& c = batch_csr(g);
  return {bs.ctl, bs.d_arg, bs.blk_cnt, bs.blk_deg, (const void*)(intptr_t)bs.nblk,
          (const void*)(intptr_t)bs.R, c.row_ptr, c.col, c.mdeg, c.first, g.csr.rank, g.b_of_row,
          (const void*)(intptr_t)g.nverts, bs.queue, bs.qdeg, (const void*)(intptr_t)sms,
          (const void*)(intptr_t)bs.bu_probe, (const void*)(intptr_t)bs.bu_round};
}

// Prologue (zero, setup, first control) followed by a WHILE node whose body
// is one level; the control kernel sets the loop condition.
void build_graph(const Graph& g, BatchState& bs, cudaStream_t s, int sms) {
  if (bs.graph_exec) cudaGraphExecDestroy(bs.graph_exec);
  if (bs.graph) cudaGraphDestroy(bs.graph);
  bs.graph_exec = nullptr;
  bs.graph = nullptr;
  // occupancy queries stay outside the capture
  blocks_per_sm(batch_td_kernel, 256);
  blocks_per_sm(batch_stats_kernel, 256);
  blocks_per_sm(batch_queue_count_kernel, kQThreads);
  blocks_per_sm(batch_queue_write_kernel, kQThreads);
  check_cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture");
  cudaGraph_t cg = nullptr;
  cudaGraph_t body = nullptr;
  cudaError_t err = cudaSuccess;
  {
    launch_prologue(g, bs, s, sms);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaGraphConditionalHandle cond = 0;
    err = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd);
    if (err == cudaSuccess)
      err = cudaGraphConditionalHandleCreate(&cond, cg, 0, cudaGraphCondAssignDefault);
    if (err == cudaSuccess) {
      batch_control_kernel<<<1, kBatchMax, 0, s>>>(bs.ctl, batch_csr(g).mdeg, cond, 1);
      err = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd);
    }
    cudaGraphNode_t node = nullptr;
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
    p.conditional.handle = cond;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    if (err == cudaSuccess) err = cudaGraphAddNode(&node, cg, deps, nd, &p);
    if (err == cudaSuccess)
      err = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
    if (err == cudaSuccess) body = p.conditional.phGraph_out[0];
    cudaGraph_t outer = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(s, &outer);
    if (err == cudaSuccess) err = e2;
    bs.graph = outer;
    if (err == cudaSuccess) {
      err = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
      if (err == cudaSuccess) {
        launch_level(g, bs, s, sms, cond, 1, nullptr);
        cudaGraph_t b2 = nullptr;
        err = cudaStreamEndCapture(s, &b2);
      }
    }
  }
  if (err == cudaSuccess) err = cudaGraphInstantiate(&bs.graph_exec, bs.graph, 0);
  if (err != cudaSuccess) {
    if (bs.graph) cudaGraphDestroy(bs.graph);
    bs.graph = nullptr;
    bs.graph_exec = nullptr;
    cudaGetLastError();
    check_cuda(err, "batch level-loop graph");
  }
  bs.graph_key = graph_key_of(g, bs, sms);
}

}  // namespace

void batch_reserve(DeviceArena& arena, const Graph& g, BatchState& bs) {
  batch_allocate(arena, g, bs);
}

void run_batch(DeviceArena& arena, const Graph& g, BatchState& bs, cudaStream_t s,
               int sms, const int64_t* roots, int k, int edgefactor, double alpha, double beta,
               bool use_graph, b200bfs_batch_stats* stats) {
  const Csr& c = batch_csr(g);
  if (!bs.allocated || bs.R != c.nrows) batch_allocate(arena, g, bs);
  BatchSetupArg& a = *static_cast<BatchSetupArg*>(bs.h_arg);
  memset(&a, 0, sizeof(a));
  bs.roots.assign(roots, roots + k);
  bs.entry_vertex.assign((size_t)k, -1);
  bs.entry_level.assign((size_t)k, 0);
  bs.path_v.assign((size_t)k, {});
  bs.path_e.assign((size_t)k, {});
  for (int i = 0; i < k; ++i) {
    int64_t entry = roots[i], lv = 0;
    if (g.core.enabled) core_climb(g, roots[i], bs.path_v[i], bs.path_e[i], &entry, &lv);
    bs.entry_vertex[i] = entry;
    bs.entry_level[i] = (int32_t)lv;
    a.v[i] = entry;
    a.lv[i] = (int)lv;
  }
  a.planes = bs.planes;
  a.seen = bs.seen;
  a.rowbits = bs.rowbits;
  a.wstride = bs.wstride;
  a.R = bs.R;
  a.capacity = bs.capacity;
  a.nedges = c.nedges;
  a.nverts = c.nrows;
  a.alpha = alpha > 0 ? alpha : kBatchAlpha;
  a.beta = beta;
  a.edgefactor = edgefactor;
  a.K = k;
  a.full_clear = bs.plane0_clean ? 0 : 1;
  a.nclear = 0;
  for (int32_t r : bs.plane0_rows) a.clear[a.nclear++] = r;
  bs.plane0_clean = false;  // until this batch completes
  bs.K = k;

  if (use_graph && (!bs.graph_exec || bs.graph_key != graph_key_of(g, bs, sms)))
    build_graph(g, bs, s, sms);

  size_t nev = 0;
  check_cuda(cudaEventRecord(bs.event(nev++), s), "event");
  check_cuda(cudaMemcpyAsync(bs.d_arg, bs.h_arg, sizeof(BatchSetupArg), cudaMemcpyHostToDevice, s),
             "batch arguments");
  int launches;
  bool loop_on_host = !use_graph;
  if (use_graph) {
    check_cuda(cudaGraphLaunch(bs.graph_exec, s), "batch graph");
    launches = 3;  // per level below
  } else {
    launch_prologue(g, bs, s, sms);
    batch_control_kernel<<<1, kBatchMax, 0, s>>>(bs.ctl, c.mdeg, 0, 0);
    launches = 3;
  }
  // per level on the host: start, queue built, bottom-up done, top-down done
  std::vector<size_t> lev_ev;
  for (;;) {
    if (loop_on_host) {
      lev_ev.push_back(nev);
      cudaEvent_t e4[4] = {bs.event(nev), bs.event(nev + 1), bs.event(nev + 2), bs.event(nev + 3)};
      nev += 4;
      launch_level(g, bs, s, sms, 0, 0, e4);
    }
    check_cuda(cudaMemcpyAsync(bs.hdone, &bs.ctl->done, sizeof(int), cudaMemcpyDeviceToHost, s),
               "batch flag");
    check_cuda(cudaStreamSynchronize(s), "batch level");
    const int done = *bs.hdone;
    if (done == 0) {
      loop_on_host = true;
      continue;
    }
    if (done == 1) break;
    if (done == 3) throw Error{B200BFS_ERR_OVERFLOW, "more than 0xFFFE BFS levels"};
    // done == 2: the next level needs another plane; the host loop resumes
    check_cuda(cudaMemcpyAsync(bs.hctl, bs.ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s),
               "batch control");
    check_cuda(cudaStreamSynchronize(s), "batch control");
    batch_grow(arena, bs, bs.hctl->level, s);
    loop_on_host = true;
    ++launches;
  }
  check_cuda(cudaEventRecord(bs.event(nev++), s), "event");
  check_cuda(cudaMemcpyAsync(bs.hctl, bs.ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, s),
             "batch control");
  check_cuda(cudaStreamSynchronize(s), "batch");
  check_cuda(cudaGetLastError(), "batch");
  const BatchCtl& h = *bs.hctl;
  // the last level found nothing: planes [0, level) hold the levels
  bs.levels = h.level;
  bs.plane0_rows.clear();
  for (int i = 0; i < k; ++i)
    if (h.root_lv[i] == 0 && h.root_row[i] >= 0) bs.plane0_rows.push_back(h.root_row[i]);
  bs.plane0_clean = true;
  b200bfs_batch_stats r;
  memset(&r, 0, sizeof(r));
  r.num_roots = k;
  r.levels = (int32_t)std::max<long long>(h.level - 1, 0);
  r.kernel_launches = launches + kLevelLaunches * (int)h.level;
  const int64_t R = bs.R;
  int64_t bytes = 16 * R;  // seen and plane 0
  bs.level_records.clear();
  // host-loop levels carry events; levels run inside the graph do not
  const long long first_host_level = (long long)h.level + 1 - (long long)lev_ev.size();
  for (long long L = 1; L <= h.level && L < kBatchHist; ++L) {
    const BatchLevelRec& x = h.hist[L];
    float td_ms = 0, bu_ms = 0, push_ms = 0;
    if (L >= first_host_level) {
      const size_t ea = lev_ev[(size_t)(L - first_host_level)];
      check_cuda(cudaEventElapsedTime(&td_ms, bs.ev[ea], bs.ev[ea + 1]), "elapsed");
      check_cuda(cudaEventElapsedTime(&bu_ms, bs.ev[ea + 1], bs.ev[ea + 2]), "elapsed");
      check_cuda(cudaEventElapsedTime(&push_ms, bs.ev[ea + 2], bs.ev[ea + 3]), "elapsed");
      td_ms += push_ms;
    }
    if (x.td_roots) {
      ++r.num_td_levels;
      r.edges_scanned_td += (int64_t)x.qedges;
      // rows + entries + seen probes
      const int64_t b = 16 * (int64_t)x.qsize + 12 * (int64_t)x.qedges;
      bytes += b;
      r.td_ms += td_ms;
      bs.level_records.push_back({(int32_t)L, 0, (int64_t)x.qsize, __builtin_popcountll(x.td_roots),
                           (int64_t)x.qedges, b, td_ms});
    }
    if (x.bu_roots) {
      ++r.num_bu_levels;
      r.edges_scanned_bu += (int64_t)x.scanned_bu;
      const int64_t b = 16 * R + 16 * (int64_t)x.rows_bu + 12 * (int64_t)x.scanned_bu;
      r.bu_bytes += b;
      bytes += b;
      r.bu_ms += bu_ms;
      bs.level_records.push_back({(int32_t)L, 1, (int64_t)x.rows_bu, __builtin_popcountll(x.bu_roots),
                           (int64_t)x.scanned_bu, b, bu_ms});
    } else {
      bytes += 8 * R;  // the level's plane
    }
  }
  r.algorithmic_bytes = bytes;
  float ms = 0;
  check_cuda(cudaEventElapsedTime(&ms, bs.ev[0], bs.ev[nev - 1]), "elapsed");
  r.ms = ms;
  if (stats) *stats = r;
}

void batch_select(const Graph& g, BfsState& st, const BatchState& bs, cudaStream_t s, int sms,
                  int index) {
  const Csr& c = batch_csr(g);
  const int B = 256;
  int32_t* lv = st.queue;  // scratch of R + 1 entries (the single-source queue)
  batch_row_levels_kernel<<<grid_for(bs.R, B, sms, 8), B, 0, s>>>(bs.planes, bs.R, bs.levels,
                                                                 index, lv);
  fill_minus_one_kernel<<<grid_for(st.pred_size, B, sms, 8), B, 0, s>>>(st.pred, st.pred_size);
  int* missing = reinterpret_cast<int*>(st.blk_cnt);  // scratch flag
  check_cuda(cudaMemsetAsync(missing, 0, sizeof(int), s), "memset");
  const int root_row = bs.hctl->root_row[index];
  batch_parent_kernel<<<grid_for(bs.R, B, sms, 8), B, 0, s>>>(lv, bs.R, c.row_ptr, c.col, c.inv,
                                                              root_row, st.pred, missing);
  const int64_t root = bs.roots[(size_t)index];
  if (g.core.enabled)
    core_write_tree(g, st.pred, bs.path_v[(size_t)index], bs.path_e[(size_t)index], s, sms);
  else if (root_row < 0 && root >= 0 && root < st.pred_size)
    set_entry_kernel<<<1, 1, 0, s>>>(st.pred, root, pred_entry(root, 0));
  int hmissing = 0;
  check_cuda(cudaMemcpyAsync(&hmissing, missing, sizeof(int), cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "batch select");
  // pred now holds exactly this root's result; its entry vertex is the one
  // entry outside the rows of the searched graph that a later search resets
  st.pred_clean = true;
  st.assembled = false;
  st.prev_root = bs.entry_vertex[(size_t)index];
  if (g.core.enabled) {
    st.tree_clean = true;  // core_write_tree wrote every tree parent
    st.prev_path_v = bs.path_v[(size_t)index];
  }
  if (hmissing) throw Error{B200BFS_ERR_CUDA, "batch levels without a parent one level up"};
}

}  // namespace b200bfs
