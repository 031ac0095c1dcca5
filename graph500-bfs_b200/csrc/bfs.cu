// Direction-optimizing BFS over the device CSR.
//
// One search = BfsBase::run_bfs_core (mpi/bfs.hpp:3238-3609) on one GPU:
//   initialize_memory (:315-349)  -> init_kernel (pred = -1, visited = 0)
//   first_expand (:562-631)        -> root_kernel (pred[root] = root)
//   top_down_search (:1355-1418)   -> td_expand_kernel: edge-balanced
//       expansion of the frontier queue; each warp takes a tile of 256
//       adjacency entries of the concatenated frontier rows, reads them
//       coalesced and claims unvisited neighbours with a race-tolerant pred
//       store plus a non-returning OR into the visited bitmap (any of several
//       same-level parents is a valid BFS parent, as validate.hpp accepts);
//   bottom_up_search_bitmap (:2828-2847, block scan :2184-2414)
//                                  -> bu_kernel: a warp owns 32 vertices (one
//       bitmap word); each unvisited lane probes its first neighbours (highest
//       degree first, so hits come early), the warp then sweeps the remaining
//       long rows cooperatively; the next bitmap word is built with
//       __ballot_sync and written once, so no atomics are needed;
//   expand / frontier bookkeeping (:634-1038)
//                                  -> frontier_count/scan/write kernels that
//       turn the new bitmap bits into the next queue with its degree prefix;
//   direction switch (:3413-3457)  -> host, from the per-level counters.
#include <algorithm>
#include <atomic>
#include <cstring>
#include "common.cuh"
#include "bfs_internal.h"

namespace b200bfs {
namespace {

// frontier kernels: a thread handles kWordsPerThread consecutive bitmap
// words (one 16-byte load), a block kWordsPerBlock
constexpr int kFrontierThreads = 256;
constexpr int kWordsPerThread = 4;
constexpr int kWordsPerBlock = kFrontierThreads * kWordsPerThread;
constexpr int kTdTile = 256;         // adjacency entries per warp tile

__device__ __forceinline__ void warp_inclusive_scan2(int64_t& a, int64_t& b) {
  const int lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int64_t ta = __shfl_up_sync(kFull, a, o);
    int64_t tb = __shfl_up_sync(kFull, b, o);
    if (lane >= o) {
      a += ta;
      b += tb;
    }
  }
}

// initialize_memory (bfs.hpp:315-349).  pred is filled with -1 only when it
// is not already clean (see BfsState::pred_clean); the bitmaps always.
__global__ void init_kernel(int64_t* __restrict__ pred, int64_t pred_size,
                            uint32_t* __restrict__ vis0, uint32_t* __restrict__ vis1, int64_t W,
                            int64_t R, int fill_pred) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (fill_pred) {
    // pred in 16-byte stores
    longlong2* p2 = reinterpret_cast<longlong2*>(pred);
    const int64_t n2 = pred_size >> 1;
    for (int64_t i = t0; i < n2; i += stride) p2[i] = make_longlong2(-1, -1);
    if (t0 == 0 && (pred_size & 1)) pred[pred_size - 1] = -1;
  }
  for (int64_t w = t0; w < W; w += stride) {
    // bits at or beyond R are padding and start "visited"
    int64_t first = w * 32;
    uint32_t v = 0;
    if (first + 32 > R) v = (first >= R) ? kFull : (kFull << (R - first));
    vis0[w] = v;
    vis1[w] = v;
  }
}

// prev_root: the previous search's root entry, cleared first (it is not
// covered by the reset of unvisited rows when it is not a row of the CSR).
// row_mode: pred is the row-order buffer of the assembly pass; the root's
// row gets the root entry there (an edgeless root gets it in the assembly).
__global__ void root_kernel(int64_t root, int64_t prev_root, const int32_t* __restrict__ rank,
                            const int64_t* __restrict__ row_ptr, int64_t* __restrict__ pred,
                            uint32_t* __restrict__ vis0, uint32_t* __restrict__ vis1,
                            int32_t* __restrict__ queue, int64_t* __restrict__ qdeg,
                            Counters* ctr, int row_mode) {
  int32_t r = rank[root];
  if (row_mode) {
    if (r >= 0) pred[r] = root;
  } else {
    if (prev_root >= 0) pred[prev_root] = -1;
    pred[root] = root;  // level 0, first_expand (bfs.hpp:593)
  }
  memset(ctr, 0, sizeof(Counters));
  if (r >= 0) {
    vis0[r >> 5] |= 1u << (r & 31);
    vis1[r >> 5] |= 1u << (r & 31);
    queue[0] = r;
    qdeg[0] = 0;
    qdeg[1] = row_ptr[r + 1] - row_ptr[r];
    ctr->qsize = 1;
    ctr->qedges = qdeg[1];
  } else {
    ctr->qsize = 0;
    qdeg[0] = 0;
  }
}

// End of a search: rows the search did not reach get pred = -1, so pred
// holds exactly this search's result without a full re-initialisation at
// the start of the next one (vertices without edges keep the -1 of the
// first fill; rows reached by an earlier search and not by this one are the
// only stale entries, and they are exactly the rows reset here).
__global__ void reset_unvisited_kernel(const uint32_t* __restrict__ vis, int64_t W,
                                       const int32_t* __restrict__ inv,
                                       int64_t* __restrict__ pred) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < W;
       w += (int64_t)gridDim.x * blockDim.x) {
    uint32_t un = ~vis[w];  // padding bits beyond R are set, so never reset
    while (un) {
      const int b = __ffs(un) - 1;
      un &= un - 1;
      pred[inv[w * 32 + b]] = -1;
    }
  }
}

// Assembly of pred from the row-order buffer rp (engine option
// pred_assemble).  pmap[u] for original id u: its row (>= 0), -1 (no parent:
// no edge, or beyond the graph), or -(p + 2) for a CoreBFS pruned vertex with
// tree parent p.  A reached row gives its rp entry, an unreached row -1, a
// pruned vertex its tree entry (level 0xFFFF, as write_tree_kernel writes),
// the root itself.  The pass runs over u in order, so pred is written in full
// lines; with group reordering the rows of a group of 2^16 ids are
// contiguous, so the rp reads of the ids a wave of warps covers fall in a few
// windows that stay in L2.  Scattering the entries by original id during the
// levels instead costs a random 32-byte sector per entry.
// A row's visited word and rp entry are loaded together (both only for
// rows), so the entry costs one round trip after the map; nearly every row
// is reached in a search of the giant component, so the rp reads of the
// unreached rows are few.
__device__ __forceinline__ int64_t assembled_entry(int32_t m, int64_t u,
                                                   const uint32_t* __restrict__ vis,
                                                   const int64_t* __restrict__ rp, int64_t root) {
  int64_t e = -1;
  if (m >= 0) {
    const uint32_t vw = __ldg(vis + (m >> 5));
    const int64_t r = __ldg(rp + m);
    if ((vw >> (m & 31)) & 1u) e = r;
  } else if (m < -1) {
    e = pred_entry(-(int64_t)m - 2, 0xFFFF);
  }
  return u == root ? root : e;
}

// Four ids per thread: one 16-byte map load, two 16-byte pred stores
// (pred and pmap are 256-byte aligned; n4 = n / 4, the tail done by thread 0).
// sparse: pred already holds the entries of every vertex outside the
// searched rows (-1, or its tree parent at level 0xFFFF), except at
// prev_root (and the previous CoreBFS climb, which the caller restores), so
// a group of four such vertices is not written: a third of the ids are rows
// at SCALE 28, and one group in five has none.
__device__ __forceinline__ void assemble_body(const int32_t* __restrict__ pmap, int64_t n,
                                              const uint32_t* __restrict__ vis,
                                              const int64_t* __restrict__ rp, int64_t root,
                                              int64_t prev_root, int sparse,
                                              int64_t* __restrict__ pred) {
  const int64_t n4 = n >> 2;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int4* m4 = reinterpret_cast<const int4*>(pmap);
  longlong2* p2 = reinterpret_cast<longlong2*>(pred);
  for (int64_t i = t0; i < n4; i += stride) {
    const int4 m = __ldg(m4 + i);
    const int64_t u = 4 * i;
    if (sparse && (m.x & m.y & m.z & m.w) < 0 && (uint64_t)(root - u) >= 4 &&
        (uint64_t)(prev_root - u) >= 4)
      continue;
    p2[2 * i] = make_longlong2(assembled_entry(m.x, u, vis, rp, root),
                               assembled_entry(m.y, u + 1, vis, rp, root));
    p2[2 * i + 1] = make_longlong2(assembled_entry(m.z, u + 2, vis, rp, root),
                                   assembled_entry(m.w, u + 3, vis, rp, root));
  }
  if (t0 == 0)
    for (int64_t u = 4 * n4; u < n; ++u) pred[u] = assembled_entry(pmap[u], u, vis, rp, root);
}

__global__ void assemble_pred_kernel(const int32_t* __restrict__ pmap, int64_t n,
                                     const uint32_t* __restrict__ vis,
                                     const int64_t* __restrict__ rp, int64_t root,
                                     int64_t prev_root, int sparse,
                                     int64_t* __restrict__ pred) {
  assemble_body(pmap, n, vis, rp, root, prev_root, sparse, pred);
}

// Number of 4-id groups of pmap (n4 of them) holding a searched row.
__global__ void core_groups_kernel(const int32_t* __restrict__ pmap, int64_t n4,
                                   unsigned long long* __restrict__ count) {
  const int4* m4 = reinterpret_cast<const int4*>(pmap);
  unsigned long long c = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int4 m = __ldg(m4 + i);
    c += (m.x & m.y & m.z & m.w) >= 0;  // not all four negative
  }
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
  if (lane_id() == 0 && c) atomicAdd(count, c);
}

// pmap from the row map and the CoreBFS tree parents (tp null without CoreBFS).
__global__ void pred_map_kernel(const int32_t* __restrict__ rank, const int32_t* __restrict__ tp,
                                int64_t nverts, int64_t n, int32_t* __restrict__ pmap) {
  for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (int64_t)gridDim.x * blockDim.x) {
    int32_t m = -1;
    if (u < nverts) {
      if (rank[u] >= 0) m = rank[u];
      else if (tp && tp[u] >= 0) m = -tp[u] - 2;
    }
    pmap[u] = m;
  }
}

// Edge-balanced top-down expansion.  Frontier queue[0..qsize) with
// qdeg[i] = sum of degrees of queue[0..i) (qdeg[qsize] = total).
// kWarpSearch: the tile's first row is found by a 32-way warp search
// (log32 rounds of coalesced loads) instead of lane 0's binary search.
// kUnroll: 32-entry steps handled together by a lane (all neighbour ids of
// the steps loaded, then all visited probes, then the claims), so more
// independent loads are in flight.
// Claim of neighbour u by a top-down entry whose probe read the visited
// word `word`: an unvisited u gets the entry's pred entry and its visited
// bit.  Several entries may claim the same u in one level (a probe can read
// a word before another warp's OR reaches it, or a stale L1 line); each
// writes a valid parent of the same level, and the OR has no return.
__device__ __forceinline__ void td_claim(int32_t u, uint32_t word, int64_t entry,
                                         const int32_t* __restrict__ pidx, uint32_t* vis,
                                         int64_t* __restrict__ pred) {
  const uint32_t bit = 1u << (u & 31);
  if ((word & bit) == 0) {
    pred[pred_slot(pidx, u)] = entry;
    red_or(vis + (u >> 5), bit);
  }
}

template <bool kWarpSearch, int kUnroll>
__device__ __forceinline__ void td_expand_body(
    const int32_t* __restrict__ queue, const int64_t* __restrict__ qdeg,
    const Counters* __restrict__ ctr, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ col, const int32_t* __restrict__ inv,
    const int32_t* __restrict__ pidx, uint32_t* vis,
    int64_t* __restrict__ pred, int64_t level) {
  const int64_t qsize = (int64_t)ctr->qsize;
  if (qsize == 0) return;
  const int64_t total = qdeg[qsize];
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t ntiles = (total + kTdTile - 1) / kTdTile;
  for (int64_t tile = gw; tile < ntiles; tile += nwarps) {
    const int64_t t0 = tile * kTdTile;
    int64_t i;
    if (kWarpSearch) {
      i = warp_segment_search(qdeg, 0, qsize - 1, t0);
    } else {
      int64_t i0 = 0;
      if (lane == 0) {
        int64_t lo = 0, hi = qsize - 1;  // largest i with qdeg[i] <= t0
        while (lo < hi) {
          int64_t mid = (lo + hi + 1) >> 1;
          if (qdeg[mid] <= t0) lo = mid;
          else hi = mid - 1;
        }
        i0 = lo;
      }
      i = __shfl_sync(kFull, i0, 0);
    }
    int64_t seg_lo = qdeg[i], seg_hi = qdeg[i + 1];
    int32_t src = queue[i];
    int64_t rbeg = row_ptr[src];
#pragma unroll 1
    for (int k = 0; k < kTdTile / 32; k += kUnroll) {
      int32_t us[kUnroll], srcs[kUnroll];
#pragma unroll
      for (int j = 0; j < kUnroll; ++j) {
        const int64_t e = t0 + (k + j) * 32 + lane;
        us[j] = -1;
        srcs[j] = 0;
        if (e < total) {
          while (e >= seg_hi && i + 1 < qsize) {
            ++i;
            seg_lo = seg_hi;
            seg_hi = qdeg[i + 1];
            src = queue[i];
            rbeg = row_ptr[src];
          }
          us[j] = __ldg(col + rbeg + (e - seg_lo));
          srcs[j] = src;
        }
      }
      // plain loads: vis is being updated by this kernel; a stale word only
      // causes a redundant (still valid) claim
      uint32_t words[kUnroll];
#pragma unroll
      for (int j = 0; j < kUnroll; ++j) words[j] = us[j] >= 0 ? vis[us[j] >> 5] : kFull;
#pragma unroll
      for (int j = 0; j < kUnroll; ++j) {
        if (us[j] < 0) continue;
        const uint32_t bit = 1u << (us[j] & 31);
        if ((words[j] & bit) == 0)
          td_claim(us[j], words[j], pred_entry(__ldg(inv + srcs[j]), level), pidx, vis, pred);
      }
    }
  }
}

// Bottom-up step.  cur is the visited bitmap before this level (read-only
// here); nxt receives cur | newly found bits for every word.
// End of the last kernel of a level (pub null: not the last one).  The
// last block to finish publishes the level: the counters go to host-mapped
// memory, then the level's sequence number (after a system-wide fence, so
// the host that sees the number sees the counters), and the per-level sums
// are cleared for the next level, which runs after this kernel in stream
// order.  Every block's counter atomics come before its ticket (fence); the
// last ticket holder reads the totals after a second fence.
__device__ __forceinline__ void publish_if_last(Counters* __restrict__ ctr,
                                                BfsState::Published* pub,
                                                unsigned long long seq) {
  if (!pub) return;
  __syncthreads();
  if (threadIdx.x != 0) return;
  __threadfence();
  if (atomicAdd(&ctr->blocks_done, 1u) != gridDim.x - 1) return;
  __threadfence();
  volatile Counters* vc = ctr;
  Counters c;
  c.nq = vc->nq;
  c.nq_edges = vc->nq_edges;
  c.scanned = vc->scanned;
  c.qsize = vc->qsize;
  c.qedges = vc->qedges;
  c.error = vc->error;
  c.blocks_done = 0;
  pub->c = c;
  ctr->nq = 0;
  ctr->nq_edges = 0;
  ctr->scanned = 0;
  ctr->blocks_done = 0;
  __threadfence_system();
  *(volatile unsigned long long*)&pub->seq = seq;
}

template <int kProbe>
__global__ void __launch_bounds__(256) bu_kernel(const uint32_t* __restrict__ cur,
                                                 uint32_t* __restrict__ nxt, int64_t W,
                                                 const int64_t* __restrict__ row_ptr,
                                                 const int32_t* __restrict__ col,
                                                 const int32_t* __restrict__ inv,
    const int32_t* __restrict__ pidx,
                                                 int64_t* __restrict__ pred, int64_t level,
                                                 Counters* __restrict__ ctr,
                                                 BfsState::Published* pub,
                                                 unsigned long long seq) {
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long found_total = 0, scanned = 0;
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
      const int64_t lim = min(e, b + (int64_t)kProbe);
      for (; b < lim; ++b) {
        const int32_t u = __ldg(col + b);
        ++scanned;
        if (bit_test(cur, u)) {
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
      int64_t j = jb;
      for (; j < je; j += 32) {
        const int64_t jj = j + lane;
        int32_t u = 0;
        bool hit = false;
        if (jj < je) {
          u = __ldg(col + jj);
          hit = bit_test(cur, u);
        }
        const unsigned hm = __ballot_sync(kFull, hit);
        if (hm) {
          const int fl = __ffs(hm) - 1;
          p = __shfl_sync(kFull, u, fl);
          if (lane == l) scanned += (unsigned long long)(j - jb + fl + 1);
          break;
        }
      }
      if (p < 0 && lane == l) scanned += (unsigned long long)(je - jb);
      if (lane == l) parent = p;
    }
    const unsigned fm = __ballot_sync(kFull, parent >= 0);
    if (lane == 0) {
      nxt[w] = c | fm;
      found_total += __popc(fm);
    }
    if (parent >= 0) pred[pred_slot(pidx, v)] = pred_entry(__ldg(inv + parent), level);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) scanned += __shfl_xor_sync(kFull, scanned, o);
  if (lane == 0) {
    if (found_total) atomicAdd(&ctr->nq, found_total);
    if (scanned) atomicAdd(&ctr->scanned, scanned);
  }
  publish_if_last(ctr, pub, seq);
}

// Bottom-up step, second form: a warp step covers kWords bitmap words, so
// every lane owns kWords vertices and issues their row-offset loads, then
// their neighbour-id loads (two neighbours per round), then the visited
// probes, back to back: kWords * 2 independent loads are in flight per lane
// instead of one dependent chain.  Rows unresolved after 8 probes are swept
// by the whole warp as in bu_kernel.
// kFirst: each open row first probes its first neighbour, read from the
// dense fpair[] array together with that neighbour's original id (one
// coalesced 8-byte read per row), and loads its row offsets only when that
// probe misses; the offset rounds then start at the second neighbour.  A
// parent found by the first probe has its pred entry's id at hand: no
// second load, no gather into inv[].
// kSpec (with kFirst): the fpair[] loads are issued for every row of the
// words, beside the loads of the words themselves, and the visited rows'
// entries are dropped afterwards: one round trip fewer per step, for the
// levels where most rows are still unvisited.
// The row search of the bottom-up forms for kWords bitmap words w[k] (w[k]
// < 0: no word) whose current visited words are c[k]: lane l handles row
// w[k] * 32 + l of each word, and the word's next value c[k] | found is
// written to nxt.
template <int kWords, bool kFirst, bool kSpec = false>
__device__ __forceinline__ void bu_rows(
    const int64_t (&w)[kWords], const uint32_t (&c)[kWords], const uint32_t* __restrict__ cur,
    uint32_t* __restrict__ nxt, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ col, const int2* __restrict__ fpair,
    const int32_t* __restrict__ inv, const int32_t* __restrict__ pidx,
    int64_t* __restrict__ pred, int64_t level, uint32_t& found_total, uint32_t& scanned) {
  const int lane = lane_id();
  // open row w[k] * 32 + lane: its next neighbour is col[b[k]] and
  // rem[k] of them are left (a row has fewer than 2^31 neighbours)
  int64_t b[kWords];
  int32_t rem[kWords];
  // par[k]: the parent's row id, or with pf[k] (found by the first probe)
  // already its original id
  int32_t par[kWords];
  bool pf[kWords];
  if (kFirst) {
    int2 f[kWords];
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
      par[k] = -1;
      pf[k] = false;
      b[k] = 0;
      rem[k] = 0;
      f[k] = make_int2(-1, -1);
      if (kSpec ? w[k] >= 0 : (((~c[k]) >> lane) & 1u) != 0)
        f[k] = __ldg(fpair + w[k] * 32 + lane);
    }
    if (kSpec) {
#pragma unroll
      for (int k = 0; k < kWords; ++k)
        if (((c[k] >> lane) & 1u) != 0) f[k].x = -1;
    }
    uint32_t mf[kWords];
#pragma unroll
    for (int k = 0; k < kWords; ++k) mf[k] = f[k].x >= 0 ? __ldg(cur + (f[k].x >> 5)) : 0u;
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
      if (f[k].x < 0) continue;
      scanned += 1;
      if ((mf[k] >> (f[k].x & 31)) & 1u) {
        par[k] = f[k].y;
        pf[k] = true;
      } else {
        const int64_t v = w[k] * 32 + lane;
        const int64_t rb = row_ptr[v];
        b[k] = rb + 1;
        rem[k] = (int32_t)(row_ptr[v + 1] - rb - 1);
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
      par[k] = -1;
      pf[k] = false;
      b[k] = 0;
      rem[k] = 0;
      if (((~c[k]) >> lane) & 1u) {
        const int64_t v = w[k] * 32 + lane;
        b[k] = row_ptr[v];
        rem[k] = (int32_t)(row_ptr[v + 1] - b[k]);
      }
    }
  }
  // four rounds of two probes per vertex
#pragma unroll
  for (int round = 0; round < 4; ++round) {
    int32_t u0[kWords], u1[kWords];
    bool need = false;
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
      u0[k] = u1[k] = -1;
      if (par[k] < 0 && rem[k] > 0) {
        u0[k] = __ldg(col + b[k]);
        if (rem[k] > 1) u1[k] = __ldg(col + b[k] + 1);
        need = true;
      }
    }
    if (!__any_sync(kFull, need)) break;
    uint32_t m0[kWords], m1[kWords];
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
      m0[k] = u0[k] >= 0 ? __ldg(cur + (u0[k] >> 5)) : 0u;
      m1[k] = u1[k] >= 0 ? __ldg(cur + (u1[k] >> 5)) : 0u;
    }
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
      if (u0[k] < 0) continue;
      if ((m0[k] >> (u0[k] & 31)) & 1u) {
        par[k] = u0[k];
        scanned += 1;
      } else if (u1[k] >= 0 && ((m1[k] >> (u1[k] & 31)) & 1u)) {
        par[k] = u1[k];
        scanned += 2;
      } else {
        const int32_t t = (u1[k] >= 0) ? 2 : 1;
        scanned += t;
        b[k] += t;
        rem[k] -= t;
      }
    }
  }
  // cooperative sweep of the rows still unresolved
#pragma unroll
  for (int k = 0; k < kWords; ++k) {
    unsigned left = __ballot_sync(kFull, par[k] < 0 && rem[k] > 0);
    while (left) {
      const int l = __ffs(left) - 1;
      left &= left - 1;
      const int64_t jb = __shfl_sync(kFull, b[k], l);
      const int64_t je = jb + __shfl_sync(kFull, rem[k], l);
      int32_t p = -1;
      for (int64_t j = jb; j < je; j += 32) {
        const int64_t jj = j + lane;
        int32_t u = 0;
        bool hit = false;
        if (jj < je) {
          u = __ldg(col + jj);
          hit = bit_test(cur, u);
        }
        const unsigned hm = __ballot_sync(kFull, hit);
        if (hm) {
          const int fl = __ffs(hm) - 1;
          p = __shfl_sync(kFull, u, fl);
          if (lane == l) scanned += (uint32_t)(j - jb + fl + 1);
          break;
        }
      }
      if (p < 0 && lane == l) scanned += (uint32_t)(je - jb);
      if (lane == l) par[k] = p;
    }
  }
#pragma unroll
  for (int k = 0; k < kWords; ++k) {
    const unsigned fm = __ballot_sync(kFull, par[k] >= 0);
    if (lane == 0 && w[k] >= 0) {
      nxt[w[k]] = c[k] | fm;
      found_total += __popc(fm);
    }
    if (par[k] >= 0) {
      const int64_t v = w[k] * 32 + lane;
      const int32_t po = pf[k] ? par[k] : __ldg(inv + par[k]);
      pred[pred_slot(pidx, v)] = pred_entry(po, level);
    }
  }
}

template <int kWords, bool kFirst, bool kSparse, bool kSpec = false>
__device__ __forceinline__ void bu_wide_body(
    const uint32_t* __restrict__ cur, uint32_t* __restrict__ nxt, int64_t W,
    const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
    const int2* __restrict__ fpair, const int32_t* __restrict__ inv,
    const int32_t* __restrict__ pidx, int64_t* __restrict__ pred, int64_t level,
    Counters* __restrict__ ctr) {
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  // per-lane counts (a lane scans far fewer than 2^32 entries), added to
  // the 64-bit level counters once at the end
  uint32_t found_total = 0, scanned = 0;
  if (kSparse) {
    // Few unvisited rows left (the last levels): a warp takes blocks of 32
    // bitmap words, one per lane; full words are copied to nxt at once and
    // only the words with unvisited rows go through the row search, kWords
    // at a time.  A block costs one load per lane instead of 32 / kWords
    // dependent word steps.
    const int64_t nblk = (W + 31) >> 5;
    for (int64_t blk = gw; blk < nblk; blk += nwarps) {
      const int64_t wl = (blk << 5) + lane;
      const uint32_t cl = wl < W ? cur[wl] : kFull;
      if (cl == kFull && wl < W) nxt[wl] = kFull;
      unsigned om = __ballot_sync(kFull, cl != kFull);
      while (om) {
        int64_t w[kWords];
        uint32_t c[kWords];
#pragma unroll
        for (int k = 0; k < kWords; ++k) {
          w[k] = -1;
          c[k] = kFull;
          if (om) {
            const int l = __ffs(om) - 1;
            om &= om - 1;
            w[k] = (blk << 5) + l;
            c[k] = __shfl_sync(kFull, cl, l);
          }
        }
        bu_rows<kWords, kFirst>(w, c, cur, nxt, row_ptr, col, fpair, inv, pidx, pred,
                                level, found_total, scanned);
      }
    }
  } else {
    // kWords consecutive words per warp step, strided over the warps
    for (int64_t w0 = gw * kWords; w0 < W; w0 += nwarps * kWords) {
      int64_t w[kWords];
      uint32_t c[kWords];
      bool all_full = true;
#pragma unroll
      for (int k = 0; k < kWords; ++k) {
        w[k] = w0 + k < W ? w0 + k : -1;
        c[k] = w[k] >= 0 ? cur[w0 + k] : kFull;
        all_full &= (c[k] == kFull);
      }
      // (kSpec issues the row loads before the words arrive: no early exit)
      if (!kSpec && all_full) {
        if (lane < kWords && w0 + lane < W) nxt[w0 + lane] = kFull;
        continue;
      }
      bu_rows<kWords, kFirst, kSpec>(w, c, cur, nxt, row_ptr, col, fpair, inv, pidx, pred, level,
                              found_total, scanned);
    }
  }
  unsigned long long sc = scanned;
#pragma unroll
  for (int o = 16; o; o >>= 1) sc += __shfl_xor_sync(kFull, sc, o);
  if (lane == 0) {
    if (found_total) atomicAdd(&ctr->nq, (unsigned long long)found_total);
    if (sc) atomicAdd(&ctr->scanned, sc);
  }
}

// Top-down expansion, second form.  The tile's first frontier row is found
// with a 32-way search (each lane probes one of 32 evenly spaced prefix
// entries per step), and the tile's eight neighbour ids are loaded before its
// eight visited probes.
__global__ void __launch_bounds__(256) td_wide_kernel(
    const int32_t* __restrict__ queue, const int64_t* __restrict__ qdeg,
    const Counters* __restrict__ ctr, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ col, const int32_t* __restrict__ inv,
    const int32_t* __restrict__ pidx, uint32_t* vis,
    int64_t* __restrict__ pred, int64_t level) {
  const int64_t qsize = (int64_t)ctr->qsize;
  if (qsize == 0) return;
  const int64_t total = qdeg[qsize];
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t ntiles = (total + kTdTile - 1) / kTdTile;
  constexpr int kPer = kTdTile / 32;
  for (int64_t tile = gw; tile < ntiles; tile += nwarps) {
    const int64_t t0 = tile * kTdTile;
    // Largest i in [0, qsize) with qdeg[i] <= t0.  Invariant: the answer is
    // in [lo, hi] and qdeg[lo] <= t0 (qdeg[0] = 0), so lane 0 always votes
    // yes; lanes whose probe lies beyond hi never vote and never load.
    int64_t lo = 0, hi = qsize - 1;
    while (hi - lo > 31) {  // more than 32 candidates left
      const int64_t step = (hi - lo + 31) / 32;
      const int64_t probe = lo + step * lane;
      const unsigned le = __ballot_sync(kFull, probe <= hi && qdeg[probe] <= t0);
      const int last = 31 - __clz(le);
      const int64_t next = lo + step * (last + 1);  // first probe known to be > t0
      lo += step * last;
      if (last < 31 && next <= hi) hi = next - 1;
    }
    {
      const int64_t probe = lo + lane;
      const unsigned le = __ballot_sync(kFull, probe <= hi && qdeg[probe] <= t0);
      lo += 31 - __clz(le);
    }
    int64_t i = lo;
    int64_t seg_lo = qdeg[i], seg_hi = qdeg[i + 1];
    int32_t src = queue[i];
    int64_t rbeg = row_ptr[src];
    int32_t srcs[kPer];
    int32_t us[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int64_t e = t0 + k * 32 + lane;
      us[k] = -1;
      srcs[k] = -1;
      if (e < total) {
        while (e >= seg_hi && i + 1 < qsize) {
          ++i;
          seg_lo = seg_hi;
          seg_hi = qdeg[i + 1];
          src = queue[i];
          rbeg = row_ptr[src];
        }
        us[k] = __ldg(col + rbeg + (e - seg_lo));
        srcs[k] = src;
      }
    }
    uint32_t words[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) words[k] = us[k] >= 0 ? vis[us[k] >> 5] : kFull;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      if (us[k] < 0) continue;
      const uint32_t bit = 1u << (us[k] & 31);
      if ((words[k] & bit) == 0) {
        pred[pred_slot(pidx, us[k])] = pred_entry(__ldg(inv + srcs[k]), level);
        red_or(vis + (us[k] >> 5), bit);
      }
    }
  }
}

// Top-down expansion, third form.  Each warp takes a contiguous chunk of
// kTdTile-entry tiles of the concatenated frontier rows and finds the row of
// its first entry with one warp search; from there it steps 32 entries at a
// time, carrying the current row.  When all 32 entries of a step lie in the
// current row (the hub rows of the large levels) they need no lookup at all;
// otherwise the rows starting inside the step (at most 31, since every row
// has an edge) mark their start positions in a 32-slot array and a
// prefix-max over the lanes gives each entry its row, so frontiers of many
// short rows (the tail levels) do not walk the degree prefix row by row.
__device__ __forceinline__ void td_chunk_body(
    const int32_t* __restrict__ queue, const int64_t* __restrict__ qdeg,
    const Counters* __restrict__ ctr, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ col, const int32_t* __restrict__ inv,
    const int32_t* __restrict__ pidx, uint32_t* vis,
    int64_t* __restrict__ pred, int64_t level) {
  __shared__ int s_map[8][32];
  const int64_t qsize = (int64_t)ctr->qsize;
  if (qsize == 0) return;
  const int64_t total = qdeg[qsize];
  const int lane = lane_id();
  const int w = threadIdx.x >> 5;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t ntiles = (total + kTdTile - 1) / kTdTile;
  const int64_t per = (ntiles + nwarps - 1) / nwarps;
  const int64_t e_begin = gw * per * kTdTile;
  const int64_t e_end = min(total, (gw + 1) * per * kTdTile);
  if (e_begin >= e_end) return;
  int64_t base = warp_segment_search(qdeg, 0, qsize - 1, e_begin);
  int64_t b_lo = qdeg[base], b_hi = qdeg[base + 1];
  int32_t b_src = queue[base];
  int64_t b_rb = row_ptr[b_src];
  for (int64_t e0 = e_begin; e0 < e_end; e0 += 32) {
    const int64_t e = e0 + lane;
    const int64_t last = min(e0 + 31, e_end - 1);
    int32_t src = b_src;
    int64_t lo = b_lo, rb = b_rb, seg_last = base;
    if (last >= b_hi) {
      s_map[w][lane] = 0;
      __syncwarp();
      const int64_t j = base + 1 + lane;
      if (j < qsize) {
        const int64_t p = qdeg[j] - e0;
        if (p >= 0 && p < 32) s_map[w][p] = lane + 1;
      }
      __syncwarp();
      int off = s_map[w][lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFull, off, o);
        if (lane >= o) off = max(off, t);
      }
      const int64_t seg = base + off;
      if (off) {
        src = queue[seg];
        lo = qdeg[seg];
        rb = row_ptr[src];
      }
      seg_last = __shfl_sync(kFull, seg, 31);
      __syncwarp();
    }
    if (e < e_end) {
      const int32_t u = __ldg(col + rb + (e - lo));
      const uint32_t bit = 1u << (u & 31);
      if ((vis[u >> 5] & bit) == 0) {
        pred[pred_slot(pidx, u)] = pred_entry(__ldg(inv + src), level);
        red_or(vis + (u >> 5), bit);
      }
    }
    // row of entry e0 + 32: the row of the step's last entry, or the next one
    // when that row ends exactly there
    if (seg_last != base) {
      base = seg_last;
      b_lo = qdeg[base];
      b_hi = qdeg[base + 1];
      b_src = queue[base];
      b_rb = row_ptr[b_src];
    }
    if (b_hi <= e0 + 32 && base + 1 < qsize) {
      ++base;
      b_lo = b_hi;
      b_hi = qdeg[base + 1];
      b_src = queue[base];
      b_rb = row_ptr[b_src];
    }
  }
}

// Top-down expansion, vector form.  Edge-balanced over the concatenated
// frontier rows like td_expand_body, in tiles of kVecTile entries strided
// over the warps, but a warp advances 128 entries per step: when the whole
// step lies inside one row (the hub rows that carry almost all entries of a
// heavy top-down level), each lane takes four consecutive neighbours with one
// 16-byte load (four 4-byte loads when the address is not 16-byte aligned),
// issues their four visited probes together and claims the unvisited ones;
// the row, its column offset and the parent's pred entry are warp-uniform,
// so the step costs no per-entry row lookup.  A step that crosses a row
// boundary runs as four 32-entry sub-steps with the per-lane row walk of
// td_expand_body; its last row, taken from lane 31, becomes the warp's row
// for the next step.
constexpr int kVecTile = 1024;  // entries per warp tile: 8 steps of 128

__device__ __forceinline__ void td_vec_body(
    const int32_t* __restrict__ queue, const int64_t* __restrict__ qdeg,
    const Counters* __restrict__ ctr, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ col, const int32_t* __restrict__ inv,
    const int32_t* __restrict__ pidx, uint32_t* vis,
    int64_t* __restrict__ pred, int64_t level) {
  const int64_t qsize = (int64_t)ctr->qsize;
  if (qsize == 0) return;
  const int64_t total = qdeg[qsize];
  const int lane = lane_id();
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t ntiles = (total + kVecTile - 1) / kVecTile;
  for (int64_t tile = gw; tile < ntiles; tile += nwarps) {
    const int64_t t0 = tile * kVecTile;
    const int64_t t_end = min(total, t0 + kVecTile);
    // warp-uniform row state: row i of the queue holds entries [seg_lo, seg_hi)
    int64_t i = warp_segment_search(qdeg, 0, qsize - 1, t0);
    int64_t seg_lo = qdeg[i], seg_hi = qdeg[i + 1];
    int32_t src = queue[i];
    int64_t rbeg = row_ptr[src];
    int64_t entry = pred_entry(__ldg(inv + src), level);
    for (int64_t e0 = t0; e0 < t_end; e0 += 128) {
      while (e0 >= seg_hi && i + 1 < qsize) {  // rows ending before the step
        ++i;
        seg_lo = seg_hi;
        seg_hi = qdeg[i + 1];
        src = queue[i];
        rbeg = row_ptr[src];
        entry = pred_entry(__ldg(inv + src), level);
      }
      if (e0 + 128 <= seg_hi && e0 + 128 <= t_end) {
        // the whole step is in row i: col[base .. base + 3] for this lane
        const int32_t* p = col + rbeg + (e0 - seg_lo) + 4 * lane;
        int32_t u0, u1, u2, u3;
        if ((reinterpret_cast<uintptr_t>(p) & 15) == 0) {
          const int4 v = __ldg(reinterpret_cast<const int4*>(p));
          u0 = v.x;
          u1 = v.y;
          u2 = v.z;
          u3 = v.w;
        } else {
          u0 = __ldg(p);
          u1 = __ldg(p + 1);
          u2 = __ldg(p + 2);
          u3 = __ldg(p + 3);
        }
        // plain loads: vis is being updated by this kernel; a stale word
        // only causes a redundant (still valid) claim
        const uint32_t w0 = vis[u0 >> 5], w1 = vis[u1 >> 5], w2 = vis[u2 >> 5],
                       w3 = vis[u3 >> 5];
        td_claim(u0, w0, entry, pidx, vis, pred);
        td_claim(u1, w1, entry, pidx, vis, pred);
        td_claim(u2, w2, entry, pidx, vis, pred);
        td_claim(u3, w3, entry, pidx, vis, pred);
        continue;
      }
      // the step crosses a row boundary: per-lane walk over 32-entry sub-steps
      int64_t li = i, l_lo = seg_lo, l_hi = seg_hi, l_rb = rbeg;
      int32_t l_src = src;
      const int64_t step_end = min(e0 + 128, t_end);
#pragma unroll 1
      for (int k = 0; k < 4; ++k) {
        const int64_t e = e0 + k * 32 + lane;
        if (e < step_end) {
          while (e >= l_hi && li + 1 < qsize) {
            ++li;
            l_lo = l_hi;
            l_hi = qdeg[li + 1];
            l_src = queue[li];
            l_rb = row_ptr[l_src];
          }
          const int32_t u = __ldg(col + l_rb + (e - l_lo));
          td_claim(u, vis[u >> 5], pred_entry(__ldg(inv + l_src), level), pidx, vis, pred);
        }
      }
      // lane 31 walked furthest (to the row of entry e0 + 127, when the tile
      // reaches it); the next step starts from there
      const int64_t ni = __shfl_sync(kFull, li, 31);
      if (ni != i) {
        i = ni;
        seg_lo = qdeg[i];
        seg_hi = qdeg[i + 1];
        src = queue[i];
        rbeg = row_ptr[src];
        entry = pred_entry(__ldg(inv + src), level);
      }
    }
  }
}

// Frontier pass 1: fr = nw & ~old, old = nw; per-block counts of frontier
// vertices, their CSR degrees and their pre-dedup degrees.
// kDeg: also the per-block CSR degree sums of the frontier, which only a
// following top-down level needs (its queue's degree prefix); after a
// top-down level they are computed by frontier_deg_body once the next
// direction is known.  The level counters (nq, nq_edges) are added only
// after a top-down level: with kDeg the pass rebuilds the queue of a
// bottom-up level whose counters the bottom-up kernel already reported.
// The kWordsPerThread words of thread t of the block (words at or beyond W
// read as 0; the bitmaps are allocated with 4 words of padding).
__device__ __forceinline__ int64_t frontier_word0() {
  return ((int64_t)blockIdx.x * kFrontierThreads + threadIdx.x) * kWordsPerThread;
}
__device__ __forceinline__ void load_words(const uint32_t* __restrict__ p, int64_t w0, int64_t W,
                                           uint32_t (&x)[kWordsPerThread]) {
  const uint4 v = w0 < W ? *reinterpret_cast<const uint4*>(p + w0) : make_uint4(0, 0, 0, 0);
  x[0] = v.x;
  x[1] = w0 + 1 < W ? v.y : 0u;
  x[2] = w0 + 2 < W ? v.z : 0u;
  x[3] = w0 + 3 < W ? v.w : 0u;
}

template <bool kDeg>
__device__ __forceinline__ void frontier_count_body(
    const uint32_t* __restrict__ nw, uint32_t* __restrict__ old, uint32_t* __restrict__ fr,
    int64_t W, const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ mdeg,
    int64_t* __restrict__ blk_cnt, int64_t* __restrict__ blk_deg, Counters* __restrict__ ctr) {
  __shared__ int64_t s_a[kFrontierThreads / 32], s_b[kFrontierThreads / 32],
      s_c[kFrontierThreads / 32];
  const int64_t w0 = frontier_word0();
  int64_t cnt = 0, dsum = 0, msum = 0;
  if (w0 < W) {
    uint32_t a[kWordsPerThread], o[kWordsPerThread];
    load_words(nw, w0, W, a);
    load_words(old, w0, W, o);
    uint32_t f[kWordsPerThread];
#pragma unroll
    for (int k = 0; k < kWordsPerThread; ++k) f[k] = a[k] & ~o[k];
    *reinterpret_cast<uint4*>(fr + w0) = make_uint4(f[0], f[1], f[2], f[3]);
    *reinterpret_cast<uint4*>(old + w0) = make_uint4(a[0], a[1], a[2], a[3]);
#pragma unroll
    for (int k = 0; k < kWordsPerThread; ++k) {
      cnt += __popc(f[k]);
      uint32_t g = f[k];
      while (g) {
        const int64_t v = (w0 + k) * 32 + __ffs(g) - 1;
        g &= g - 1;
        if (kDeg) dsum += row_ptr[v + 1] - row_ptr[v];
        msum += mdeg[v];
      }
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    cnt += __shfl_xor_sync(kFull, cnt, o);
    dsum += __shfl_xor_sync(kFull, dsum, o);
    msum += __shfl_xor_sync(kFull, msum, o);
  }
  const int wid = threadIdx.x >> 5;
  if (lane_id() == 0) {
    s_a[wid] = cnt;
    s_b[wid] = dsum;
    s_c[wid] = msum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t A = 0, Bs = 0, C = 0;
    for (int i = 0; i < kFrontierThreads / 32; ++i) {
      A += s_a[i];
      Bs += s_b[i];
      C += s_c[i];
    }
    blk_cnt[blockIdx.x] = A;
    if (kDeg) blk_deg[blockIdx.x] = Bs;
    if (A && !kDeg) {
      atomicAdd(&ctr->nq, (unsigned long long)A);
      atomicAdd(&ctr->nq_edges, (unsigned long long)C);
    }
  }
}

// Per-block CSR degree sums of the frontier bitmap fr.
__device__ __forceinline__ void frontier_deg_body(const uint32_t* __restrict__ fr, int64_t W,
                                                  const int64_t* __restrict__ row_ptr,
                                                  int64_t* __restrict__ blk_deg) {
  __shared__ int64_t s_b[kFrontierThreads / 32];
  const int64_t w0 = frontier_word0();
  int64_t dsum = 0;
  if (w0 < W) {
    uint32_t f[kWordsPerThread];
    load_words(fr, w0, W, f);
#pragma unroll
    for (int k = 0; k < kWordsPerThread; ++k) {
      uint32_t g = f[k];
      while (g) {
        const int64_t v = (w0 + k) * 32 + __ffs(g) - 1;
        g &= g - 1;
        dsum += row_ptr[v + 1] - row_ptr[v];
      }
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) dsum += __shfl_xor_sync(kFull, dsum, o);
  if (lane_id() == 0) s_b[threadIdx.x >> 5] = dsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t b = 0;
    for (int i = 0; i < kFrontierThreads / 32; ++i) b += s_b[i];
    blk_deg[blockIdx.x] = b;
  }
}

// Frontier pass 2: exclusive scan of the block partials (single block).
__device__ __forceinline__ void frontier_scan_body(int64_t* __restrict__ blk_cnt,
                                                   int64_t* __restrict__ blk_deg, int64_t nblk,
                                                   int64_t* __restrict__ qdeg,
                                                   Counters* __restrict__ ctr) {
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
  warp_inclusive_scan2(ia, ib);
  const int wid = t >> 5, lane = lane_id();
  if (lane == 31) {
    s_a[wid] = ia;
    s_b[wid] = ib;
  }
  __syncthreads();
  if (wid == 0) {
    int64_t xa = s_a[lane], xb = s_b[lane];
    warp_inclusive_scan2(xa, xb);
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
    const int64_t tot_a = s_a[31], tot_b = s_b[31];
    ctr->qsize = (unsigned long long)tot_a;
    ctr->qedges = (unsigned long long)tot_b;
    qdeg[tot_a] = tot_b;
  }
}

// Frontier pass 3: write the queue in vertex order with its degree prefix.
__device__ __forceinline__ void frontier_write_body(
    const uint32_t* __restrict__ fr, int64_t W, const int64_t* __restrict__ row_ptr,
    const int64_t* __restrict__ blk_cnt, const int64_t* __restrict__ blk_deg,
    int32_t* __restrict__ queue, int64_t* __restrict__ qdeg) {
  __shared__ int64_t s_a[kFrontierThreads / 32], s_b[kFrontierThreads / 32];
  const int64_t w0 = frontier_word0();
  uint32_t f[kWordsPerThread] = {0u, 0u, 0u, 0u};
  if (w0 < W) load_words(fr, w0, W, f);
  int64_t cnt = 0, dsum = 0;
#pragma unroll
  for (int k = 0; k < kWordsPerThread; ++k) {
    cnt += __popc(f[k]);
    uint32_t g = f[k];
    while (g) {
      const int64_t v = (w0 + k) * 32 + __ffs(g) - 1;
      g &= g - 1;
      dsum += row_ptr[v + 1] - row_ptr[v];
    }
  }
  int64_t ic = cnt, id = dsum;
  warp_inclusive_scan2(ic, id);
  const int wid = threadIdx.x >> 5, lane = lane_id();
  if (lane == 31) {
    s_a[wid] = ic;
    s_b[wid] = id;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t ra = 0, rb = 0;
    for (int i = 0; i < kFrontierThreads / 32; ++i) {
      const int64_t xa = s_a[i], xb = s_b[i];
      s_a[i] = ra;
      s_b[i] = rb;
      ra += xa;
      rb += xb;
    }
  }
  __syncthreads();
  int64_t pos = blk_cnt[blockIdx.x] + s_a[wid] + ic - cnt;
  int64_t dpos = blk_deg[blockIdx.x] + s_b[wid] + id - dsum;
#pragma unroll
  for (int k = 0; k < kWordsPerThread; ++k) {
    uint32_t g = f[k];
    while (g) {
      const int64_t v = (w0 + k) * 32 + __ffs(g) - 1;
      g &= g - 1;
      queue[pos] = (int32_t)v;
      qdeg[pos] = dpos;
      ++pos;
      dpos += row_ptr[v + 1] - row_ptr[v];
    }
  }
}

// Kernels of the host-driven level loop: thin wrappers around the bodies
// above, which the device-driven loop (below) shares.
template <bool kWarpSearch, int kUnroll>
__global__ void __launch_bounds__(256) td_expand_kernel(
    const int32_t* __restrict__ queue, const int64_t* __restrict__ qdeg,
    const Counters* __restrict__ ctr, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ col, const int32_t* __restrict__ inv,
    const int32_t* __restrict__ pidx, uint32_t* vis,
    int64_t* __restrict__ pred, int64_t level) {
  td_expand_body<kWarpSearch, kUnroll>(queue, qdeg, ctr, row_ptr, col, inv, pidx, vis, pred, level);
}

template <int kWords, int kMinBlocks, bool kFirst, bool kSparse = false, bool kSpec = false>
__global__ void __launch_bounds__(256, kMinBlocks) bu_wide_kernel(
    const uint32_t* __restrict__ cur, uint32_t* __restrict__ nxt, int64_t W,
    const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
    const int2* __restrict__ fpair, const int32_t* __restrict__ inv,
    const int32_t* __restrict__ pidx, int64_t* __restrict__ pred, int64_t level,
    Counters* __restrict__ ctr, BfsState::Published* pub, unsigned long long seq) {
  bu_wide_body<kWords, kFirst, kSparse, kSpec>(cur, nxt, W, row_ptr, col, fpair, inv, pidx, pred,
                                               level, ctr);
  publish_if_last(ctr, pub, seq);
}

__global__ void __launch_bounds__(256) td_vec_kernel(
    const int32_t* __restrict__ queue, const int64_t* __restrict__ qdeg,
    const Counters* __restrict__ ctr, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ col, const int32_t* __restrict__ inv,
    const int32_t* __restrict__ pidx, uint32_t* vis,
    int64_t* __restrict__ pred, int64_t level) {
  td_vec_body(queue, qdeg, ctr, row_ptr, col, inv, pidx, vis, pred, level);
}

__global__ void __launch_bounds__(256) td_chunk_kernel(
    const int32_t* __restrict__ queue, const int64_t* __restrict__ qdeg,
    const Counters* __restrict__ ctr, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ col, const int32_t* __restrict__ inv,
    const int32_t* __restrict__ pidx, uint32_t* vis,
    int64_t* __restrict__ pred, int64_t level) {
  td_chunk_body(queue, qdeg, ctr, row_ptr, col, inv, pidx, vis, pred, level);
}

template <bool kDeg>
__global__ void __launch_bounds__(kFrontierThreads) frontier_count_kernel(
    const uint32_t* __restrict__ nw, uint32_t* __restrict__ old, uint32_t* __restrict__ fr,
    int64_t W, const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ mdeg,
    int64_t* __restrict__ blk_cnt, int64_t* __restrict__ blk_deg, Counters* __restrict__ ctr,
    BfsState::Published* pub, unsigned long long seq) {
  frontier_count_body<kDeg>(nw, old, fr, W, row_ptr, mdeg, blk_cnt, blk_deg, ctr);
  publish_if_last(ctr, pub, seq);
}

__global__ void __launch_bounds__(kFrontierThreads) frontier_deg_kernel(
    const uint32_t* __restrict__ fr, int64_t W, const int64_t* __restrict__ row_ptr,
    int64_t* __restrict__ blk_deg) {
  frontier_deg_body(fr, W, row_ptr, blk_deg);
}

__global__ void __launch_bounds__(1024) frontier_scan_kernel(int64_t* __restrict__ blk_cnt,
                                                             int64_t* __restrict__ blk_deg,
                                                             int64_t nblk,
                                                             int64_t* __restrict__ qdeg,
                                                             Counters* __restrict__ ctr) {
  frontier_scan_body(blk_cnt, blk_deg, nblk, qdeg, ctr);
}

__global__ void __launch_bounds__(kFrontierThreads) frontier_write_kernel(
    const uint32_t* __restrict__ fr, int64_t W, const int64_t* __restrict__ row_ptr,
    const int64_t* __restrict__ blk_cnt, const int64_t* __restrict__ blk_deg,
    int32_t* __restrict__ queue, int64_t* __restrict__ qdeg) {
  frontier_write_body(fr, W, row_ptr, blk_cnt, blk_deg, queue, qdeg);
}

__global__ void levels_kernel(const int64_t* __restrict__ pred, int64_t n,
                              int32_t* __restrict__ lv) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = pred[i];
    lv[i] = (p == -1) ? -1 : (int32_t)(((uint64_t)p >> 48) & 0xFFFF);
  }
}

// ---------------------------------------------------------------------------
// Device-driven level loop (engine option single_graph): the same kernels,
// with the state that run_bfs_core keeps in host variables (level, direction,
// growing, current bitmap, counts, auto_tuning_data) in a device control
// block.  Every level launches the same sequence; the kernels whose step does
// not apply to the level return at once, and sg_control_kernel applies the
// switch rule of bfs.hpp:3413-3457 exactly as the host loop does (same
// integer and double arithmetic) and sets the WHILE condition of the graph.

__global__ void sg_root_kernel(const SgArg* __restrict__ a, const int32_t* __restrict__ rank,
                               const int64_t* __restrict__ row_ptr, int64_t* __restrict__ pred,
                               uint32_t* __restrict__ vis0, uint32_t* __restrict__ vis1,
                               int32_t* __restrict__ queue, int64_t* __restrict__ qdeg,
                               Counters* ctr, SingleCtl* __restrict__ c, int row_mode) {
  const int64_t root = a->root;
  const int32_t r = rank[root];
  if (row_mode) {  // as root_kernel
    if (r >= 0) pred[r] = root;
  } else {
    if (a->prev_root >= 0) pred[a->prev_root] = -1;
    pred[root] = root;  // level 0, first_expand (bfs.hpp:593)
  }
  memset(ctr, 0, sizeof(Counters));
  if (r >= 0) {
    vis0[r >> 5] |= 1u << (r & 31);
    vis1[r >> 5] |= 1u << (r & 31);
    queue[0] = r;
    qdeg[0] = 0;
    qdeg[1] = row_ptr[r + 1] - row_ptr[r];
    ctr->qsize = 1;
    ctr->qedges = qdeg[1];
  } else {
    ctr->qsize = 0;
    qdeg[0] = 0;
  }
  memset(c, 0, sizeof(SingleCtl));
  c->level = a->root_level;
  c->next_forward = 1;
  c->growing = 1;
  c->visited = 1;
  c->qsize = 1;
  for (int i = 0; i < 9; ++i) c->at[i] = a->at[i];
}

__global__ void sg_reset_unvisited_kernel(const SingleCtl* __restrict__ c,
                                          uint32_t* const* __restrict__ vis_pp, int64_t W,
                                          const int32_t* __restrict__ inv,
                                          int64_t* __restrict__ pred) {
  const uint32_t* vis = vis_pp[c->cur];
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < W;
       w += (int64_t)gridDim.x * blockDim.x) {
    uint32_t un = ~vis[w];
    while (un) {
      const int b = __ffs(un) - 1;
      un &= un - 1;
      pred[inv[w * 32 + b]] = -1;
    }
  }
}

__global__ void sg_assemble_kernel(const SingleCtl* __restrict__ c, const SgArg* __restrict__ a,
                                   uint32_t* const* __restrict__ vis_pp,
                                   const int32_t* __restrict__ pmap, int64_t n,
                                   const int64_t* __restrict__ rp, int64_t* __restrict__ pred) {
  assemble_body(pmap, n, vis_pp[c->cur], rp, a->root, a->sparse ? a->prev_root : -1, a->sparse,
                pred);
}

// Level start (host loop: ++level, at[8], prev_nq, forward, clear counters).
__global__ void sg_begin_kernel(SingleCtl* __restrict__ c, const SgArg* __restrict__ a,
                                Counters* __restrict__ ctr) {
  if (c->done) return;
  ++c->level;
  if (c->level > kMaxLevel) {
    c->done = 3;
    return;
  }
  if (a->want_at) c->at[8] = c->level;  // AUTO_LEVEL
  c->prev_nq = c->global_nq_size;
  c->forward = c->next_forward;
  ctr->nq = 0;
  ctr->nq_edges = 0;
  ctr->scanned = 0;
}

// kForm 1/5: td_expand (lane or warp search); 3: td_chunk.  td_form is the
// engine option (4 = 5 while growing, 3 after).
template <int kForm>
__global__ void __launch_bounds__(256) sg_td_kernel(
    const SingleCtl* __restrict__ c, int td_form, const int32_t* __restrict__ queue,
    const int64_t* __restrict__ qdeg, const Counters* __restrict__ ctr,
    const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
    const int32_t* __restrict__ inv,
    const int32_t* __restrict__ pidx, uint32_t* const* __restrict__ vis_pp,
    int64_t* __restrict__ pred) {
  if (c->done || !c->forward) return;
  const int form = td_form == 4 ? (c->growing ? 5 : 3) : td_form;
  if (form != kForm) return;
  uint32_t* vis = vis_pp[c->cur];
  if (kForm == 3)
    td_chunk_body(queue, qdeg, ctr, row_ptr, col, inv, pidx, vis, pred, c->level);
  else
    td_expand_body<kForm == 5, 1>(queue, qdeg, ctr, row_ptr, col, inv, pidx, vis, pred, c->level);
}

template <bool kFirst>
__global__ void __launch_bounds__(256, 4) sg_bu_kernel(
    const SingleCtl* __restrict__ c, int64_t W, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ col, const int2* __restrict__ fpair,
    const int32_t* __restrict__ inv, const int32_t* __restrict__ pidx,
    uint32_t* const* __restrict__ vis_pp, int64_t* __restrict__ pred,
    Counters* __restrict__ ctr) {
  if (c->done || c->forward) return;
  const int cur = c->cur;
  bu_wide_body<4, kFirst, false>(vis_pp[cur], vis_pp[cur ^ 1], W, row_ptr, col, fpair, inv, pidx,
                                 pred, c->level, ctr);
}

// kAfterBu = false: after a top-down level; true: after a bottom-up level
// whose next level is top-down (the bitmaps have swapped by then).
template <bool kAfterBu>
__global__ void __launch_bounds__(kFrontierThreads) sg_count_kernel(
    const SingleCtl* __restrict__ c, uint32_t* const* __restrict__ vis_pp,
    uint32_t* __restrict__ fr, int64_t W, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ mdeg, int64_t* __restrict__ blk_cnt,
    int64_t* __restrict__ blk_deg, Counters* __restrict__ ctr) {
  if (c->done) return;
  if (kAfterBu ? (c->forward || !c->next_forward) : !c->forward) return;
  const int cur = c->cur;
  frontier_count_body<kAfterBu>(vis_pp[cur], vis_pp[cur ^ 1], fr, W, row_ptr, mdeg, blk_cnt,
                                blk_deg, ctr);
}

// After a top-down level whose next level is top-down: the queue's degree
// sums.
__global__ void __launch_bounds__(kFrontierThreads) sg_deg_kernel(
    const SingleCtl* __restrict__ c, const uint32_t* __restrict__ fr, int64_t W,
    const int64_t* __restrict__ row_ptr, int64_t* __restrict__ blk_deg) {
  if (c->done || !c->forward || !c->next_forward) return;
  frontier_deg_body(fr, W, row_ptr, blk_deg);
}

__global__ void __launch_bounds__(1024) sg_scan_kernel(const SingleCtl* __restrict__ c,
                                                       int64_t* __restrict__ blk_cnt,
                                                       int64_t* __restrict__ blk_deg,
                                                       int64_t nblk, int64_t* __restrict__ qdeg,
                                                       Counters* __restrict__ ctr) {
  if (c->done || !c->next_forward) return;
  frontier_scan_body(blk_cnt, blk_deg, nblk, qdeg, ctr);
}

__global__ void __launch_bounds__(kFrontierThreads) sg_write_kernel(
    const SingleCtl* __restrict__ c, const uint32_t* __restrict__ fr, int64_t W,
    const int64_t* __restrict__ row_ptr, const int64_t* __restrict__ blk_cnt,
    const int64_t* __restrict__ blk_deg, int32_t* __restrict__ queue,
    int64_t* __restrict__ qdeg) {
  if (c->done || !c->next_forward) return;
  frontier_write_body(fr, W, row_ptr, blk_cnt, blk_deg, queue, qdeg);
}

// Level end: the host loop's bookkeeping and switch rule (bfs.hpp:3413-3457).
__global__ void sg_control_kernel(SingleCtl* __restrict__ c, const SgArg* __restrict__ a,
                                  const Counters* __restrict__ ctr, int64_t R, int64_t W,
                                  int64_t nedges, int64_t nrows, int force_direction,
                                  cudaGraphConditionalHandle cond) {
  if (c->done) {
    cudaGraphSetConditional(cond, 0u);
    return;
  }
  const bool forward = c->forward != 0;
  const int64_t nq = (int64_t)ctr->nq;
  c->global_nq_size = nq;
  SgRec rec;
  rec.level = (int32_t)c->level;
  if (forward) {
    c->global_nq_edges = (int64_t)ctr->nq_edges;
    const int64_t e_td = (int64_t)ctr->qedges;
    const int64_t b = 16 * c->qsize + 8 * e_td + 12 * nq;
    c->scanned_td += e_td;
    c->td_bytes += b;
    c->bytes += b;
    ++c->num_td;
    rec.bottom_up = 0;
    rec.input = c->qsize;
    rec.scanned = e_td;
    rec.bytes = b;
  } else {
    const int64_t unvisited = R - c->visited;
    const int64_t sc = (int64_t)ctr->scanned;
    const int64_t b = 3 * (W * 4) + 16 * unvisited + 8 * sc + 12 * nq;
    c->scanned_bu += sc;
    c->bu_bytes += b;
    c->bytes += b;
    ++c->num_bu;
    if (c->level < 64) c->bu_mask |= 1ull << c->level;
    c->cur ^= 1;
    rec.bottom_up = 1;
    rec.input = unvisited;
    rec.scanned = sc;
    rec.bytes = b;
  }
  rec.discovered = nq;
  if (c->nrec < kSgHist) c->rec[c->nrec] = rec;
  ++c->nrec;
  c->visited += nq;
  if (nq == 0) {
    c->done = 1;
    cudaGraphSetConditional(cond, 0u);
    return;
  }
  const double alpha = a->alpha, beta = a->beta;
  const bool at = a->want_at != 0;
  bool next_forward = c->next_forward != 0;
  if (c->growing && nq > c->prev_nq) {
    if (forward) {
      if (c->global_nq_edges > (int64_t)(nedges / alpha)) {
        next_forward = false;
        if (at) {
          c->at[0] = c->global_nq_edges;  // AUTO_GLOBAL_NQ_EDGES
          c->at[1] = nedges;              // AUTO_NUM_GLOBAL_EDGES
          c->at[2] = c->level;            // AUTO_T2B_LEVEL
        }
      } else if (at) {
        c->at[6] = c->global_nq_edges;  // AUTO_PRE_GLOBAL_NQ_EDGES
      }
    }
  } else {
    if (!forward) {
      if (nq < (int64_t)(nrows / (beta * a->edgefactor * 2.0))) {
        next_forward = true;
        c->growing = 0;
        if (at) {
          c->at[3] = nq;        // AUTO_GLOBAL_NQ_SIZE
          c->at[4] = nrows;     // AUTO_NUM_GLOBAL_VERTS
          c->at[5] = c->level;  // AUTO_B2T_LEVEL
        }
      } else if (at) {
        c->at[7] = nq;  // AUTO_PRE_GLOBAL_NQ_SIZE
      }
    }
  }
  if (force_direction == 1) next_forward = true;
  if (force_direction == 2) next_forward = false;
  c->next_forward = next_forward ? 1 : 0;
  if (next_forward) c->qsize = nq;
  cudaGraphSetConditional(cond, 1u);
}

}  // namespace

// Algorithmic bytes of the assembly pass: the map and pred over every id,
// the rp entries of the reached rows, the visited bitmap.
int64_t assembly_bytes(const BfsState& st, int64_t visited, bool sparse) {
  // map read + pred writes + row-order entries of the reached rows + bitmap
  const int64_t written = sparse ? 4 * st.core_groups : st.pred_size;
  return 4 * st.pred_size + 8 * written + 8 * visited + 4 * st.W;
}

void build_pred_assembly(DeviceArena& arena, const Graph& g, BfsState& st, cudaStream_t s,
                         int sms) {
  if (!st.rp) st.rp = arena_alloc<int64_t>(arena, st.R + 1, "row-order pred");
  if (!st.pmap) st.pmap = arena_alloc<int32_t>(arena, st.pred_size + 4, "pred assembly map");
  pred_map_kernel<<<grid_for(st.pred_size, 256, sms, 8), 256, 0, s>>>(
      g.csr.rank, g.core.enabled ? g.core.tree_parent : nullptr, g.nverts, st.pred_size,
      st.pmap);
  // the groups a sparse assembly writes (scratch: the block counts)
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(st.blk_cnt);
  check_cuda(cudaMemsetAsync(cnt, 0, sizeof(*cnt), s), "memset");
  core_groups_kernel<<<grid_for(st.pred_size / 4, 256, sms, 8), 256, 0, s>>>(
      st.pmap, st.pred_size / 4, cnt);
  unsigned long long h = 0;
  check_cuda(cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaGetLastError(), "pred assembly map");
  check_cuda(cudaStreamSynchronize(s), "pred assembly map");
  st.core_groups = (int64_t)h;
}

void BfsState::allocate(DeviceArena& arena, const Graph& g) {
  release(arena);
  R = g.csr.nrows;
  W = (R + 31) / 32;
  pred_size = g.pred_size;
  nblk = (W + kWordsPerBlock - 1) / kWordsPerBlock;
  vis[0] = arena_alloc<uint32_t>(arena, W + 4, "visited bitmap");
  vis[1] = arena_alloc<uint32_t>(arena, W + 4, "visited bitmap");
  fr = arena_alloc<uint32_t>(arena, W + 4, "frontier bitmap");
  queue = arena_alloc<int32_t>(arena, R + 1, "frontier queue");
  qdeg = arena_alloc<int64_t>(arena, R + 2, "frontier degree prefix");
  blk_cnt = arena_alloc<int64_t>(arena, nblk + 1, "block counts");
  blk_deg = arena_alloc<int64_t>(arena, nblk + 1, "block degrees");
  pred = arena_alloc<int64_t>(arena, pred_size + 2, "pred");
  ctr = arena_alloc<Counters>(arena, 1, "counters");
  check_cuda(cudaHostAlloc(&hpub, sizeof(Published), cudaHostAllocMapped), "mapped counters");
  check_cuda(cudaHostGetDevicePointer(&dpub, hpub, 0), "mapped counters");
  hpub->seq = 0;
  pub_seq = 0;
  sctl = arena_alloc<SingleCtl>(arena, 1, "search control block");
  sarg = arena_alloc<SgArg>(arena, 1, "search arguments");
  d_vis = arena_alloc<uint32_t*>(arena, 2, "bitmap pointers");
  pred_clean = false;
  prev_root = -1;
  assembled = false;
  check_cuda(cudaMemcpy(d_vis, vis, sizeof(vis), cudaMemcpyHostToDevice), "bitmap pointers");
  check_cuda(cudaMallocHost(&hsctl, sizeof(SingleCtl)), "pinned control block");
  check_cuda(cudaMallocHost(&hsarg, sizeof(SgArg)), "pinned arguments");
  allocated = true;
}

cudaEvent_t BfsState::event(size_t i) {
  while (ev.size() <= i) {
    cudaEvent_t e;
    check_cuda(cudaEventCreate(&e), "event");
    ev.push_back(e);
  }
  return ev[i];
}

void BfsState::release(DeviceArena& arena) {
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  ev.clear();
  if (sgexec) cudaGraphExecDestroy(sgexec);
  if (sgraph) cudaGraphDestroy(sgraph);
  sgexec = nullptr;
  sgraph = nullptr;
  skey.clear();
  if (!allocated) return;
  arena.free(sctl);
  arena.free(sarg);
  arena.free(d_vis);
  d_vis = nullptr;
  cudaFreeHost(hsctl);
  cudaFreeHost(hsarg);
  sctl = nullptr;
  sarg = nullptr;
  hsctl = nullptr;
  hsarg = nullptr;
  arena.free(vis[0]);
  arena.free(vis[1]);
  arena.free(fr);
  arena.free(queue);
  arena.free(qdeg);
  arena.free(blk_cnt);
  arena.free(blk_deg);
  arena.free(pred);
  arena.free(ctr);
  if (rp) arena.free(rp);
  if (pmap) arena.free(pmap);
  rp = nullptr;
  pmap = nullptr;
  if (hpub) cudaFreeHost(hpub);
  hpub = nullptr;
  dpub = nullptr;
  allocated = false;
}

namespace {


// One level of the device-driven loop (captured into the WHILE body).
void sg_launch_level(const Graph& g, BfsState& st, cudaStream_t s, int sms, int td_form,
                     int force_direction, bool bu_first, bool assemble,
                     cudaGraphConditionalHandle cond) {
  const Csr& c = g.csr;
  const int32_t* pidx = assemble ? nullptr : c.inv;
  int64_t* out = assemble ? st.rp : st.pred;
  const int B = 256;
  const unsigned nblk = (unsigned)st.nblk;
  sg_begin_kernel<<<1, 1, 0, s>>>(st.sctl, st.sarg, st.ctr);
  sg_td_kernel<1><<<sms * 8, B, 0, s>>>(st.sctl, td_form, st.queue, st.qdeg, st.ctr, c.row_ptr,
                                         c.col, c.inv, pidx, st.d_vis, out);
  sg_td_kernel<5><<<sms * 8, B, 0, s>>>(st.sctl, td_form, st.queue, st.qdeg, st.ctr, c.row_ptr,
                                         c.col, c.inv, pidx, st.d_vis, out);
  sg_td_kernel<3><<<sms * blocks_per_sm(td_chunk_kernel, 256), B, 0, s>>>(st.sctl, td_form,
                                                                          st.queue, st.qdeg,
                                                             st.ctr, c.row_ptr, c.col, c.inv, pidx,
                                                             st.d_vis, out);
  (bu_first && c.first_pair ? sg_bu_kernel<true> : sg_bu_kernel<false>)<<<sms * 4, B, 0, s>>>(
      st.sctl, st.W, c.row_ptr, c.col, c.first_pair, c.inv, pidx, st.d_vis, out, st.ctr);
  sg_count_kernel<false><<<nblk, kFrontierThreads, 0, s>>>(st.sctl, st.d_vis, st.fr, st.W,
                                                         c.row_ptr, c.mdeg, st.blk_cnt,
                                                         st.blk_deg, st.ctr);
  sg_control_kernel<<<1, 1, 0, s>>>(st.sctl, st.sarg, st.ctr, st.R, st.W, c.nedges, c.nrows,
                                    force_direction, cond);
  sg_count_kernel<true><<<nblk, kFrontierThreads, 0, s>>>(st.sctl, st.d_vis, st.fr, st.W,
                                                        c.row_ptr, c.mdeg, st.blk_cnt,
                                                        st.blk_deg, st.ctr);
  sg_deg_kernel<<<nblk, kFrontierThreads, 0, s>>>(st.sctl, st.fr, st.W, c.row_ptr, st.blk_deg);
  sg_scan_kernel<<<1, 1024, 0, s>>>(st.sctl, st.blk_cnt, st.blk_deg, st.nblk, st.qdeg, st.ctr);
  sg_write_kernel<<<nblk, kFrontierThreads, 0, s>>>(st.sctl, st.fr, st.W, c.row_ptr, st.blk_cnt,
                                                  st.blk_deg, st.queue, st.qdeg);
}
constexpr int kSgLevelLaunches = 12;

std::vector<const void*> sg_key(const Graph& g, const BfsState& st, int sms, int td_form,
                                int force_direction, bool bu_first, bool assemble) {
  const Csr& c = g.csr;
  return {st.sctl, st.sarg, st.d_vis, st.ctr, st.fr, st.queue, st.qdeg, st.blk_cnt, st.blk_deg,
          st.pred, st.vis[0], st.vis[1], c.row_ptr, c.col, c.inv, c.rank, c.mdeg,
          (const void*)(intptr_t)st.W, (const void*)(intptr_t)st.R,
          (const void*)(intptr_t)st.pred_size, (const void*)(intptr_t)c.nedges,
          (const void*)(intptr_t)sms, (const void*)(intptr_t)td_form,
          (const void*)(intptr_t)force_direction, c.first, c.first_pair,
          (const void*)(intptr_t)bu_first,
          (const void*)(intptr_t)assemble, st.rp, st.pmap};
}

// [init, root] then WHILE(level); the control kernel sets the condition.
void sg_build_graph(const Graph& g, BfsState& st, cudaStream_t s, int sms, int td_form,
                    int force_direction, bool bu_first, bool assemble) {
  if (st.sgexec) cudaGraphExecDestroy(st.sgexec);
  if (st.sgraph) cudaGraphDestroy(st.sgraph);
  st.sgexec = nullptr;
  st.sgraph = nullptr;
  const Csr& c = g.csr;
  blocks_per_sm(td_chunk_kernel, 256);  // occupancy queries stay outside the capture
  check_cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture");
  init_kernel<<<grid_for(st.W, 256, sms, 8), 256, 0, s>>>(st.pred, st.pred_size, st.vis[0],
                                                          st.vis[1], st.W, st.R, 0);
  sg_root_kernel<<<1, 1, 0, s>>>(st.sarg, c.rank, c.row_ptr, assemble ? st.rp : st.pred,
                                 st.vis[0], st.vis[1], st.queue, st.qdeg, st.ctr, st.sctl,
                                 assemble ? 1 : 0);
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  cudaGraph_t cg = nullptr;
  cudaGraphConditionalHandle cond = 0;
  cudaError_t err = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd);
  if (err == cudaSuccess)
    err = cudaGraphConditionalHandleCreate(&cond, cg, 1, cudaGraphCondAssignDefault);
  cudaGraphNode_t node = nullptr;
  cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
  p.conditional.handle = cond;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  if (err == cudaSuccess) err = cudaGraphAddNode(&node, cg, deps, nd, &p);
  if (err == cudaSuccess)
    err = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
  if (err == cudaSuccess && assemble)
    sg_assemble_kernel<<<grid_for(st.pred_size / 4, 256, sms, 8), 256, 0, s>>>(
        st.sctl, st.sarg, st.d_vis, st.pmap, st.pred_size, st.rp, st.pred);
  else if (err == cudaSuccess)
    sg_reset_unvisited_kernel<<<grid_for(st.W, 256, sms, 8), 256, 0, s>>>(st.sctl, st.d_vis, st.W,
                                                                           c.inv, st.pred);
  cudaGraph_t body = err == cudaSuccess ? p.conditional.phGraph_out[0] : nullptr;
  cudaGraph_t outer = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(s, &outer);
  if (err == cudaSuccess) err = e2;
  st.sgraph = outer;
  if (err == cudaSuccess) {
    err = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
      sg_launch_level(g, st, s, sms, td_form, force_direction, bu_first, assemble, cond);
      cudaGraph_t b2 = nullptr;
      err = cudaStreamEndCapture(s, &b2);
    }
  }
  if (err == cudaSuccess) err = cudaGraphInstantiate(&st.sgexec, st.sgraph, 0);
  if (err != cudaSuccess) {
    if (st.sgraph) cudaGraphDestroy(st.sgraph);
    st.sgraph = nullptr;
    st.sgexec = nullptr;
    cudaGetLastError();
    check_cuda(err, "search level-loop graph");
  }
  st.skey = sg_key(g, st, sms, td_form, force_direction, bu_first, assemble);
}

// run_bfs_core with the level loop on the device.
void run_bfs_core_graph(const Graph& g, BfsState& st, cudaStream_t s, int sms, int64_t root,
                        int64_t root_level, int edgefactor, double alpha, double beta,
                        int64_t* at, const RunOptions& opt, b200bfs_run_stats* stats) {
  const bool bu_first = opt.bu_first != 0;
  const bool assemble = use_pred_assembly(g, opt);
  if (assemble && !st.pmap) throw Error{B200BFS_ERR_STATE, "pred assembly map not built"};
  st.asm_ev = -1;  // the graph does not time the assembly pass
  if (!st.sgexec ||
      st.skey != sg_key(g, st, sms, opt.td_kernel, opt.force_direction, bu_first, assemble))
    sg_build_graph(g, st, s, sms, opt.td_kernel, opt.force_direction, bu_first, assemble);
  if (!assemble) st.assembled = false;  // as in run_bfs_core
  if (!st.pred_clean && !assemble) {
    st.tree_clean = false;
    init_kernel<<<grid_for(st.pred_size / 2, 256, sms, 8), 256, 0, s>>>(
        st.pred, st.pred_size, st.vis[0], st.vis[1], st.W, st.R, 1);
    check_cuda(cudaGetLastError(), "pred fill");
  }
  SgArg& a = *st.hsarg;
  a.prev_root = st.pred_clean ? st.prev_root : -1;
  a.root = root;
  a.root_level = root_level;
  a.alpha = alpha;
  a.beta = beta;
  a.edgefactor = edgefactor;
  a.want_at = at != nullptr;
  // as in the host loop: sparse when the last writer of pred was an
  // assembled search
  const bool sparse = assemble && st.assembled && st.pred_clean;
  a.sparse = sparse ? 1 : 0;
  for (int i = 0; i < 9; ++i) a.at[i] = at ? at[i] : -1;
  check_cuda(cudaMemcpyAsync(st.sarg, st.hsarg, sizeof(SgArg), cudaMemcpyHostToDevice, s),
             "search arguments");
  check_cuda(cudaGraphLaunch(st.sgexec, s), "search graph");
  check_cuda(cudaMemcpyAsync(st.hsctl, st.sctl, sizeof(SingleCtl), cudaMemcpyDeviceToHost, s),
             "control block");
  check_cuda(cudaStreamSynchronize(s), "search");
  const SingleCtl& c = *st.hsctl;
  if (c.done == 3) throw Error{B200BFS_ERR_OVERFLOW, "more than 0xFFFE BFS levels"};
  st.pred_clean = true;
  st.prev_root = root;
  st.asm_sparse = sparse;
  st.assembled = assemble;
  if (at)
    for (int i = 0; i < 9; ++i) at[i] = c.at[i];
  st.levels.clear();
  for (int i = 0; i < std::min(c.nrec, kSgHist); ++i) {
    const SgRec& r = c.rec[i];
    st.levels.push_back({r.level, r.bottom_up, r.input, r.discovered, r.scanned, r.bytes, 0.0});
  }
  if (stats) {
    b200bfs_run_stats rs;
    memset(&rs, 0, sizeof(rs));
    rs.levels = (int32_t)c.level;
    rs.num_td_levels = (int32_t)c.num_td;
    rs.num_bu_levels = (int32_t)c.num_bu;
    rs.bu_level_mask = c.bu_mask;
    rs.visited = c.visited;
    rs.edges_scanned_td = c.scanned_td;
    rs.edges_scanned_bu = c.scanned_bu;
    rs.td_bytes = c.td_bytes;
    rs.bu_bytes = c.bu_bytes;
    rs.algorithmic_bytes =
        c.bytes + 4 * st.W +
        (assemble ? assembly_bytes(st, c.visited, sparse)
                  : 8 * std::max<int64_t>(st.R - c.visited, 0));
    rs.kernel_launches = 3 + kSgLevelLaunches * (int)(c.num_td + c.num_bu);
    *stats = rs;
  }
}

}  // namespace

// Waits for the level's counters: polls the host-mapped
// sequence number, checking the stream every few thousand polls so that a
// failed kernel ends the wait with its error instead of a hang.
static Counters wait_level(BfsState& st, cudaStream_t s) {
  // the level's last kernel publishes sequence number pub_seq + 1
  const unsigned long long seq = ++st.pub_seq;
  check_cuda(cudaGetLastError(), "level");
  volatile unsigned long long* flag = &st.hpub->seq;
  for (unsigned long long n = 1; *flag != seq; ++n) {
    if ((n & 4095) == 0) {
      const cudaError_t e = cudaStreamQuery(s);
      if (e == cudaSuccess) {
        if (*flag != seq) throw Error{B200BFS_ERR_CUDA, "level counters not published"};
        break;
      }
      if (e != cudaErrorNotReady) check_cuda(e, "level");
    }
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  Counters h;
  memcpy(&h, (const void*)&st.hpub->c, sizeof(Counters));
  return h;
}

// The level loop with the reference's direction switch.
void run_bfs_core(const Graph& g, BfsState& st, cudaStream_t s, int sms, int64_t root,
                  int64_t root_level, int edgefactor, double alpha, double beta, int64_t* at,
                  const RunOptions& opt, b200bfs_run_stats* stats) {
  // the device-driven loop has top-down forms 1, 3, 4 and 5 and its own
  // bottom-up form (four words per warp step, as form 4)
  if (opt.single_graph && opt.td_kernel != 2 && opt.td_kernel <= 5) {
    run_bfs_core_graph(g, st, s, sms, root, root_level, edgefactor, alpha, beta, at, opt, stats);
    return;
  }
  const Csr& c = g.csr;
  const int B = 256;
  b200bfs_run_stats rs;
  memset(&rs, 0, sizeof(rs));
  int64_t bytes = 0;

  int launches = 2;
  // (level kind, event index) of every timed level kernel
  std::vector<std::pair<bool, size_t>> timed;
  size_t nev = 0;
  // assemble: the levels write the row-order buffer rp and a final pass
  // writes every pred entry; otherwise they write pred by original id
  const bool assemble = use_pred_assembly(g, opt);
  if (assemble && !st.pmap) throw Error{B200BFS_ERR_STATE, "pred assembly map not built"};
  const int32_t* pidx = assemble ? nullptr : c.inv;
  int64_t* out = assemble ? st.rp : st.pred;
  // a direct search writes pred as it goes: from here on, even if it fails,
  // the next assembly must write every group
  if (!assemble) st.assembled = false;
  const bool fill_pred = !st.pred_clean && !assemble;
  if (fill_pred) st.tree_clean = false;
  init_kernel<<<grid_for(std::max(fill_pred ? st.pred_size / 2 : 0, st.W), B, sms, 8), B, 0, s>>>(
      st.pred, st.pred_size, st.vis[0], st.vis[1], st.W, st.R, fill_pred ? 1 : 0);
  root_kernel<<<1, 1, 0, s>>>(root, st.pred_clean ? st.prev_root : -1, c.rank, c.row_ptr, out,
                              st.vis[0], st.vis[1], st.queue, st.qdeg, st.ctr, assemble ? 1 : 0);
  bytes += fill_pred ? 8 * st.pred_size : 4 * st.W;  // pred initialisation / unvisited reset
  int cur = 0;  // vis[cur] is the current visited bitmap

  int64_t level = root_level;
  bool forward = true, next_forward = true, growing = true;
  int64_t global_nq_size = 0, global_nq_edges = 0;
  int64_t visited = 1, qsize = 1;
  st.levels.clear();
  const int bu_grid =
      std::min(grid_for(st.W * 32, B, sms, 8), sms * blocks_per_sm(bu_kernel<8>, B));
  const int bu_wide_grid = sms * 8;
  // the chunked top-down form splits the work evenly over its warps, so its
  // grid is exactly the resident blocks (one wave)
  const int td_chunk_grid = sms * blocks_per_sm(td_chunk_kernel, 256);
  for (;;) {
    ++level;
    if (level > kMaxLevel) throw Error{B200BFS_ERR_OVERFLOW, "more than 0xFFFE BFS levels"};
    if (at) at[8] = level;  // AUTO_LEVEL
    const int64_t prev_nq = global_nq_size;
    forward = next_forward;
    int64_t frontier_in = 0;
    check_cuda(cudaEventRecord(st.event(nev), s), "event");
    timed.push_back({forward, nev});
    nev += 2;
    if (forward) {
      ++rs.num_td_levels;
      // form 4: the strided form while the frontier grows (hub rows), the
      // chunked form once the search has come back from bottom-up (short
      // rows of the tail levels)
      const int td_form = opt.td_kernel == 4   ? (growing ? 5 : 3)
                          : opt.td_kernel == 7 ? (growing ? 6 : 3)
                                               : opt.td_kernel;
      // every top-down form has the same parameters
      // one resident wave of each form (their register counts differ)
      auto launch_td = [&](auto kernel, int grid) {
        if (grid <= 0) grid = sms * blocks_per_sm(kernel, B);
        kernel<<<grid, B, 0, s>>>(st.queue, st.qdeg, st.ctr, c.row_ptr, c.col, c.inv, pidx,
                                  st.vis[cur], out, level);
      };
      if (td_form == 6)
        launch_td(td_vec_kernel, 0);
      else if (td_form == 5 && opt.td_unroll == 4)
        launch_td(td_expand_kernel<true, 4>, 0);
      else if (td_form == 5 && opt.td_unroll == 2)
        launch_td(td_expand_kernel<true, 2>, 0);
      else if (td_form == 5)
        launch_td(td_expand_kernel<true, 1>, 0);
      else if (td_form == 1)
        launch_td(td_expand_kernel<false, 1>, 0);
      else if (td_form == 3)
        launch_td(td_chunk_kernel, td_chunk_grid);
      else
        launch_td(td_wide_kernel, 0);
      check_cuda(cudaEventRecord(st.event(nev - 1), s), "event");
      launches += 2;
      frontier_count_kernel<false><<<(unsigned)st.nblk, kFrontierThreads, 0, s>>>(
          st.vis[cur], st.vis[cur ^ 1], st.fr, st.W, c.row_ptr, c.mdeg, st.blk_cnt, st.blk_deg,
          st.ctr, st.dpub, st.pub_seq + 1);
      frontier_in = qsize;
    } else {
      ++rs.num_bu_levels;
      if (level < 64) rs.bu_level_mask |= 1ull << level;
      const bool first = opt.bu_first && c.first_pair;
      auto launch_wide = [&](auto kernel, int grid) {
        kernel<<<grid, B, 0, s>>>(st.vis[cur], st.vis[cur ^ 1], st.W, c.row_ptr, c.col,
                                  c.first_pair, c.inv, pidx, out, level, st.ctr, st.dpub,
                                  st.pub_seq + 1);
      };
      auto launch_bu = [&](auto kernel) {
        kernel<<<bu_grid, B, 0, s>>>(st.vis[cur], st.vis[cur ^ 1], st.W, c.row_ptr, c.col, c.inv,
                                     pidx, out, level, st.ctr, st.dpub, st.pub_seq + 1);
      };
      // the last levels, with few unvisited rows left, skip full bitmap words
      // 32 at a time (fewer than one unvisited row per four words)
      const bool sparse = opt.bu_sparse && 4 * (st.R - visited) < st.W;
      // the levels where most rows are still unvisited load every row's
      // first-neighbour entry beside its bitmap word
      const bool spec = first && opt.bu_spec && 2 * (st.R - visited) > st.R;
      if (opt.bu_kernel == 2 && sparse)
        launch_wide(first ? bu_wide_kernel<2, 8, true, true> : bu_wide_kernel<2, 8, false, true>,
                    bu_wide_grid);
      else if (opt.bu_kernel == 2 && spec)
        launch_wide(bu_wide_kernel<2, 8, true, false, true>, bu_wide_grid);
      else if (opt.bu_kernel == 2)
        launch_wide(first ? bu_wide_kernel<2, 8, true> : bu_wide_kernel<2, 8, false>,
                    bu_wide_grid);
      else if (opt.bu_kernel == 3 && sparse)
        launch_wide(first ? bu_wide_kernel<2, 6, true, true> : bu_wide_kernel<2, 6, false, true>,
                    sms * 6);
      else if (opt.bu_kernel == 3 && spec)
        launch_wide(bu_wide_kernel<2, 6, true, false, true>, sms * 6);
      else if (opt.bu_kernel == 3)
        launch_wide(first ? bu_wide_kernel<2, 6, true> : bu_wide_kernel<2, 6, false>, sms * 6);
      else if (opt.bu_kernel == 4 && sparse)
        launch_wide(first ? bu_wide_kernel<4, 4, true, true> : bu_wide_kernel<4, 4, false, true>,
                    sms * 4);
      else if (opt.bu_kernel == 4 && spec)
        launch_wide(bu_wide_kernel<4, 4, true, false, true>, sms * 4);
      else if (opt.bu_kernel == 4)
        launch_wide(first ? bu_wide_kernel<4, 4, true> : bu_wide_kernel<4, 4, false>, sms * 4);
      else if (opt.bu_probe <= 4)
        launch_bu(bu_kernel<4>);
      else if (opt.bu_probe <= 8)
        launch_bu(bu_kernel<8>);
      else
        launch_bu(bu_kernel<16>);
      check_cuda(cudaEventRecord(st.event(nev - 1), s), "event");
      launches += 1;
      cur ^= 1;
    }
    const Counters h = wait_level(st, s);
    global_nq_size = (int64_t)h.nq;
    if (forward) {
      global_nq_edges = (int64_t)h.nq_edges;
      const int64_t e_td = (int64_t)h.qedges;  // entries of the frontier rows
      rs.edges_scanned_td += e_td;
      // 16|F| row offsets + 4 E neighbour ids + 4 E visited probes + 12|D|
      const int64_t b = 16 * frontier_in + 8 * e_td + 12 * global_nq_size;
      bytes += b;
      rs.td_bytes += b;
      st.levels.push_back({(int32_t)level, 0, frontier_in, global_nq_size, e_td, b, 0.0});
    } else {
      const int64_t unvisited = st.R - visited;
      rs.edges_scanned_bu += (int64_t)h.scanned;
      // 3 R/8 bitmap sweeps + 16|U| row offsets + 4 E ids + 4 E probes + 12|D|
      const int64_t b =
          3 * (st.W * 4) + 16 * unvisited + 8 * (int64_t)h.scanned + 12 * global_nq_size;
      bytes += b;
      rs.bu_bytes += b;
      st.levels.push_back(
          {(int32_t)level, 1, unvisited, global_nq_size, (int64_t)h.scanned, b, 0.0});
    }
    visited += global_nq_size;
    if (global_nq_size == 0) break;

    if (growing && global_nq_size > prev_nq) {
      if (forward) {
        if (global_nq_edges > (int64_t)(c.nedges / alpha)) {
          next_forward = false;
          if (at) {
            at[0] = global_nq_edges;  // AUTO_GLOBAL_NQ_EDGES
            at[1] = c.nedges;         // AUTO_NUM_GLOBAL_EDGES
            at[2] = level;            // AUTO_T2B_LEVEL
          }
        } else if (at) {
          at[6] = global_nq_edges;  // AUTO_PRE_GLOBAL_NQ_EDGES
        }
      }
    } else {
      if (!forward) {
        if (global_nq_size < (int64_t)(c.nrows / (beta * edgefactor * 2.0))) {
          next_forward = true;
          growing = false;
          if (at) {
            at[3] = global_nq_size;  // AUTO_GLOBAL_NQ_SIZE
            at[4] = c.nrows;         // AUTO_NUM_GLOBAL_VERTS
            at[5] = level;           // AUTO_B2T_LEVEL
          }
        } else if (at) {
          at[7] = global_nq_size;  // AUTO_PRE_GLOBAL_NQ_SIZE
        }
      }
    }
    if (opt.force_direction == 1) next_forward = true;
    if (opt.force_direction == 2) next_forward = false;

    if (next_forward) {
      // Build the next queue from the bits set in this level.
      if (!forward)  // after bottom-up: bits of vis[cur] not in vis[cur^1]
        frontier_count_kernel<true><<<(unsigned)st.nblk, kFrontierThreads, 0, s>>>(
            st.vis[cur], st.vis[cur ^ 1], st.fr, st.W, c.row_ptr, c.mdeg, st.blk_cnt, st.blk_deg,
            st.ctr, nullptr, 0);
      else  // after top-down: the counts are there, the degree sums not yet
        frontier_deg_kernel<<<(unsigned)st.nblk, kFrontierThreads, 0, s>>>(st.fr, st.W, c.row_ptr,
                                                                         st.blk_deg);
      frontier_scan_kernel<<<1, 1024, 0, s>>>(st.blk_cnt, st.blk_deg, st.nblk, st.qdeg, st.ctr);
      frontier_write_kernel<<<(unsigned)st.nblk, kFrontierThreads, 0, s>>>(
          st.fr, st.W, c.row_ptr, st.blk_cnt, st.blk_deg, st.queue, st.qdeg);
      launches += 3;
      qsize = global_nq_size;
    }
  }
  // the last writer of pred was an assembled search: every entry outside
  // the searched rows already holds its value
  const bool sparse = assemble && st.assembled && st.pred_clean;
  st.asm_sparse = sparse;
  if (assemble) {
    check_cuda(cudaEventRecord(st.event(nev), s), "event");
    assemble_pred_kernel<<<grid_for(st.pred_size / 4, B, sms, 8), B, 0, s>>>(
        st.pmap, st.pred_size, st.vis[cur], st.rp, root, sparse ? st.prev_root : -1,
        sparse ? 1 : 0, st.pred);
    check_cuda(cudaEventRecord(st.event(nev + 1), s), "event");
    nev += 2;
    rs.pred_bytes = assembly_bytes(st, visited, sparse);
    bytes += rs.pred_bytes;
  } else {
    reset_unvisited_kernel<<<grid_for(st.W, B, sms, 8), B, 0, s>>>(st.vis[cur], st.W, c.inv,
                                                                   st.pred);
    bytes += 8 * std::max<int64_t>(st.R - visited, 0);
  }
  ++launches;
  st.pred_clean = true;
  st.prev_root = root;
  st.assembled = assemble;
  check_cuda(cudaGetLastError(), "bfs");
  for (size_t k = 0; k < timed.size(); ++k) {
    const auto& t = timed[k];
    float ms = 0;
    check_cuda(cudaEventElapsedTime(&ms, st.ev[t.second], st.ev[t.second + 1]), "elapsed");
    (t.first ? rs.td_ms : rs.bu_ms) += ms;
    if (k < st.levels.size()) st.levels[k].ms = ms;
  }
  st.asm_ev = assemble ? (int)(nev - 2) : -1;  // read by finish_run_stats
  rs.kernel_launches = launches;
  rs.levels = (int32_t)level;
  rs.visited = visited;
  rs.algorithmic_bytes = bytes;
  if (stats) *stats = rs;
}

void finish_run_stats(BfsState& st, b200bfs_run_stats* stats) {
  if (!stats || st.asm_ev < 0) return;
  float ms = 0;
  check_cuda(cudaEventSynchronize(st.ev[st.asm_ev + 1]), "assembly");
  check_cuda(cudaEventElapsedTime(&ms, st.ev[st.asm_ev], st.ev[st.asm_ev + 1]), "elapsed");
  stats->pred_ms = ms;
}

void levels_from_pred(const BfsState& st, cudaStream_t s, int sms, int32_t* d_levels) {
  levels_kernel<<<grid_for(st.pred_size, 256, sms, 8), 256, 0, s>>>(st.pred, st.pred_size,
                                                                   d_levels);
}

}  // namespace b200bfs
