// Edge list -> degree-ordered, de-duplicated CSR on the device.
//
// Replaces make_symmetry_edge_list (mpi/benchmark_helper.hpp:383-497) and
// GraphConstructor2DCSR::construct (mpi/graph_constructor.hpp:1009-1033) for
// one rank:
//   1. estimate SCALE from the OR of all endpoints of non-loop edges
//      (benchmark_helper.hpp:488-494);
//   2. count the pre-dedup symmetric degree of every vertex
//      (DegreeCalculation::calc_degree, graph_constructor.hpp:572-592);
//   3. order vertices by descending degree, dropping degree-0 vertices
//      (VERTEX_REORDERING=2, :632-637; with group reordering the order is
//      taken within groups of 2^16 original ids, SMALL_REORDER_BIT :594-732);
//   4. place every directed entry into its row (two-pass counting placement),
//      sort each row and drop duplicates (sortEdgesInner, :1986-2056) to get
//      num_global_edges_ (:2100) and num_global_verts_ (:2103-2128).  Rows
//      are sorted by the neighbours' global degree rank (highest degree
//      first) even with group reordering, where the reference sorts by the
//      group-ordered id: adjacency order changes neither levels nor the
//      validity of parents, and hub-first lists let the bottom-up searches
//      stop early.
// Self-loops are dropped as in make_symmetry_edge_list (:409, 429, 447).
// All passes are bandwidth-bound integer streams; CUB supplies the radix
// sorts and scans of this (untimed) construction step.
#include <algorithm>
#include <cub/cub.cuh>
#include "common.cuh"
#include "engine.h"

namespace b200bfs {
namespace {

__global__ void or_ids_kernel(const uint2* __restrict__ e, int64_t m, unsigned long long* out) {
  uint32_t acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint2 x = e[i];
    if (x.x != x.y) acc |= x.x | x.y;
  }
  for (int o = 16; o; o >>= 1) acc |= __shfl_xor_sync(kFull, acc, o);
  if (lane_id() == 0 && acc) atomicOr(out, (unsigned long long)acc);
}

__global__ void count_degree_kernel(const uint2* __restrict__ e, int64_t m, bool mirror,
                                    uint32_t* __restrict__ deg) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint2 x = e[i];
    if (x.x == x.y) continue;
    atomicAdd(deg + x.x, 1u);
    if (mirror) atomicAdd(deg + x.y, 1u);
  }
}

// key = (degree==0) << 63 | group << 32 | (2^32-1 - degree): ascending order
// puts degree-0 vertices last and the rest in descending degree per group.
__global__ void make_keys_kernel(const uint32_t* __restrict__ deg, int64_t n, int group_bits,
                                 uint64_t* __restrict__ keys, int32_t* __restrict__ ids) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    uint32_t d = deg[v];
    uint64_t g = group_bits > 0 ? (uint64_t)(v >> group_bits) : 0;
    keys[v] = ((uint64_t)(d == 0) << 63) | (g << 32) | (uint64_t)(0xFFFFFFFFu - d);
    ids[v] = (int32_t)v;
  }
}

__global__ void fill_i32_kernel(int32_t* p, int64_t n, int32_t v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

__global__ void rank_kernel(const int32_t* __restrict__ inv, const uint32_t* __restrict__ deg,
                            int64_t R, int32_t* __restrict__ rank, int32_t* __restrict__ mdeg,
                            int64_t* __restrict__ len64) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < R;
       r += (int64_t)gridDim.x * blockDim.x) {
    int32_t v = inv[r];
    rank[v] = (int32_t)r;
    uint32_t d = deg[v];
    mdeg[r] = (int32_t)d;
    len64[r] = d;
  }
}

// Places every edge in its source row; the stored value is the neighbour's
// sort key nkey[v] (its row id, or its global degree rank when rows follow
// the group order).
__global__ void scatter_kernel(const uint2* __restrict__ e, int64_t m, bool mirror,
                               const int32_t* __restrict__ rank, const int32_t* __restrict__ nkey,
                               const int64_t* __restrict__ raw_ptr,
                               uint32_t* __restrict__ cursor, int32_t* __restrict__ raw) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint2 x = e[i];
    if (x.x == x.y) continue;
    int32_t ra = rank[x.x], rb = rank[x.y];
    raw[raw_ptr[ra] + atomicAdd(cursor + ra, 1u)] = nkey[x.y];
    if (mirror) raw[raw_ptr[rb] + atomicAdd(cursor + rb, 1u)] = nkey[x.x];
  }
}

// Group order: nkey[v] = position of v in the global degree order,
// row_of_key[k] = row of the vertex at global position k.
__global__ void global_rank_kernel(const int32_t* __restrict__ gorder, int64_t R,
                                   const int32_t* __restrict__ rank, int32_t* __restrict__ nkey,
                                   int32_t* __restrict__ row_of_key) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < R;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = gorder[k];
    nkey[v] = (int32_t)k;
    row_of_key[k] = rank[v];
  }
}

__global__ void rel_offsets_kernel(const int64_t* __restrict__ raw_ptr, int64_t r0, int64_t nr,
                                   int32_t* __restrict__ rel) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= nr;
       i += (int64_t)gridDim.x * blockDim.x)
    rel[i] = (int32_t)(raw_ptr[r0 + i] - raw_ptr[r0]);
}

// Largest row index r1 in (r0, R] with raw_ptr[r1] - raw_ptr[r0] <= limit.
__global__ void chunk_end_kernel(const int64_t* __restrict__ raw_ptr, int64_t R, int64_t r0,
                                 int64_t limit, int64_t* out) {
  int64_t lo = r0 + 1, hi = R, base = raw_ptr[r0];
  // invariant: answer in [lo, hi]; at least one row even if it exceeds limit
  while (lo < hi) {
    int64_t mid = lo + (hi - lo + 1) / 2;
    if (raw_ptr[mid] - base <= limit) lo = mid;
    else hi = mid - 1;
  }
  *out = lo;
}

// Distinct values per sorted row (warp per row).
__global__ void count_distinct_kernel(const int32_t* __restrict__ raw,
                                      const int64_t* __restrict__ raw_ptr, int64_t R,
                                      int64_t* __restrict__ dlen) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = lane_id();
  for (int64_t r = warp; r < R; r += nwarps) {
    const int64_t b = raw_ptr[r], e = raw_ptr[r + 1];
    int64_t cnt = 0;
    for (int64_t j = b + lane; j - lane < e; j += 32) {
      bool head = false;
      if (j < e) head = (j == b) || (raw[j] != raw[j - 1]);
      cnt += __popc(__ballot_sync(kFull, head));
    }
    if (lane == 0) dlen[r] = cnt;
  }
}

__global__ void compact_rows_kernel(const int32_t* __restrict__ raw,
                                    const int64_t* __restrict__ raw_ptr, int64_t R,
                                    const int64_t* __restrict__ row_ptr,
                                    const int32_t* __restrict__ row_of_key,
                                    int32_t* __restrict__ col) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = lane_id();
  for (int64_t r = warp; r < R; r += nwarps) {
    const int64_t b = raw_ptr[r], e = raw_ptr[r + 1];
    int64_t out = row_ptr[r];
    for (int64_t j = b + lane; j - lane < e; j += 32) {
      bool head = false;
      int32_t x = 0;
      if (j < e) {
        x = raw[j];
        head = (j == b) || (x != raw[j - 1]);
      }
      unsigned m = __ballot_sync(kFull, head);
      if (head) col[out + __popc(m & ((1u << lane) - 1))] = row_of_key ? row_of_key[x] : x;
      out += __popc(m);
    }
  }
}

__global__ void first_kernel(const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                             const int32_t* __restrict__ inv, int64_t R,
                             int32_t* __restrict__ first, int2* __restrict__ first_pair) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < R;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t f = row_ptr[r + 1] > row_ptr[r] ? col[row_ptr[r]] : -1;
    first[r] = f;
    if (first_pair) first_pair[r] = make_int2(f, f >= 0 ? inv[f] : -1);
  }
}

__global__ void max_degree_kernel(const int64_t* __restrict__ row_ptr, int64_t R,
                                  unsigned long long* out) {
  unsigned long long acc = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < R;
       r += (int64_t)gridDim.x * blockDim.x)
    acc = max(acc, (unsigned long long)(row_ptr[r + 1] - row_ptr[r]));
  for (int o = 16; o; o >>= 1) acc = max(acc, __shfl_xor_sync(kFull, acc, o));
  if (lane_id() == 0) atomicMax(out, acc);
}

int msb_index(uint64_t v) { return v ? 63 - __builtin_clzll(v) : -1; }

}  // namespace

void build_csr(DeviceArena& arena, cudaStream_t s, const uint2* edges, int64_t m, bool mirror,
               bool group_reorder, int scale_hint, Graph& g, int sms) {
  const int B = 256;
  auto grid = [&](int64_t n) { return grid_for(n, B, sms, 16); };

  // 1. SCALE estimate.
  unsigned long long* d_u64 = arena_alloc<unsigned long long>(arena, 2, "scalars");
  check_cuda(cudaMemsetAsync(d_u64, 0, 16, s), "memset");
  or_ids_kernel<<<grid(m), B, 0, s>>>(edges, m, d_u64);
  unsigned long long orv = 0;
  check_cuda(cudaMemcpyAsync(&orv, d_u64, 8, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "scale estimate");
  int est = msb_index(orv) + 1;
  if (est <= 0) est = 1;
  if (scale_hint > 0 && est > scale_hint)
    throw Error{B200BFS_ERR_INVALID, "edge endpoints exceed 2^scale"};
  if (est > 30) throw Error{B200BFS_ERR_INVALID, "SCALE above 30 is not supported"};
  g.scale = est;
  g.nverts = int64_t(1) << est;
  g.pred_size = std::max<int64_t>(g.nverts, int64_t(1) << 16);
  g.group_reorder = group_reorder;
  // Group width of the group order: min(16, 48 - local id bits)
  // (graph_constructor.hpp:704-712), which is 16 for every SCALE <= 30 here.
  // Below SCALE 16 one group holds every id, as with a narrower group.
  const int group_bits = group_reorder ? 16 : 0;
  g.reorder_bits = group_bits;
  const int64_t n = g.nverts;

  // 2. pre-dedup degree
  uint32_t* deg = arena_alloc<uint32_t>(arena, n, "degree");
  check_cuda(cudaMemsetAsync(deg, 0, n * 4, s), "memset");
  count_degree_kernel<<<grid(m), B, 0, s>>>(edges, m, mirror, deg);

  // 3. degree order
  uint64_t* keys = arena_alloc<uint64_t>(arena, n, "sort keys");
  uint64_t* keys2 = arena_alloc<uint64_t>(arena, n, "sort keys");
  int32_t* ids = arena_alloc<int32_t>(arena, n, "sort values");
  int32_t* ids2 = arena_alloc<int32_t>(arena, n, "sort values");
  make_keys_kernel<<<grid(n), B, 0, s>>>(deg, n, group_bits, keys, ids);
  {
    size_t tmp = 0;
    check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, keys2, ids, ids2, (int)n, 0,
                                               64, s),
               "sort size");
    void* t = arena.alloc(tmp, "sort temp");
    check_cuda(cub::DeviceRadixSort::SortPairs(t, tmp, keys, keys2, ids, ids2, (int)n, 0, 64, s),
               "sort");
    arena.free(t);
  }
  arena.free(keys);
  // R = number of keys without the degree-0 bit; find it by a count.
  int64_t R;
  {
    // the sorted keys put degree-0 vertices at the end: count them via a
    // binary search on the host-visible boundary
    uint64_t* probe_keys = keys2;
    int64_t lo = 0, hi = n;  // first index with top bit set
    // small host binary search over device memory (log2(n) 8-byte reads)
    while (lo < hi) {
      int64_t mid = (lo + hi) / 2;
      uint64_t k;
      check_cuda(cudaMemcpyAsync(&k, probe_keys + mid, 8, cudaMemcpyDeviceToHost, s), "probe");
      check_cuda(cudaStreamSynchronize(s), "probe");
      if (k >> 63) hi = mid;
      else lo = mid + 1;
    }
    R = lo;
  }
  arena.free(keys2);
  arena.free(ids);
  if (R == 0) throw Error{B200BFS_ERR_INVALID, "graph has no edges"};
  Csr& c = g.csr;
  c.nrows = R;
  c.inv = arena_alloc<int32_t>(arena, R, "inv map");
  check_cuda(cudaMemcpyAsync(c.inv, ids2, R * 4, cudaMemcpyDeviceToDevice, s), "copy inv");
  arena.free(ids2);
  c.rank = arena_alloc<int32_t>(arena, n, "rank map");
  fill_i32_kernel<<<grid(n), B, 0, s>>>(c.rank, n, -1);
  c.mdeg = arena_alloc<int32_t>(arena, R, "mdeg");
  int64_t* raw_ptr = arena_alloc<int64_t>(arena, R + 1, "raw row ptr");
  int64_t* len64 = arena_alloc<int64_t>(arena, R, "row len");
  rank_kernel<<<grid(R), B, 0, s>>>(c.inv, deg, R, c.rank, c.mdeg, len64);
  // Neighbour lists are sorted by the neighbours' global degree rank, highest
  // degree first, whatever the row numbering: the bottom-up searches stop at
  // the first neighbour found, and the hubs are found first.  With one global
  // degree order the rank is the row id; with the group order it comes from a
  // second sort by degree alone.
  int32_t* nkey = c.rank;
  int32_t* row_of_key = nullptr;
  if (group_bits > 0) {
    uint64_t* k1 = arena_alloc<uint64_t>(arena, n, "sort keys");
    uint64_t* k2 = arena_alloc<uint64_t>(arena, n, "sort keys");
    int32_t* i1 = arena_alloc<int32_t>(arena, n, "sort values");
    int32_t* i2 = arena_alloc<int32_t>(arena, n, "sort values");
    make_keys_kernel<<<grid(n), B, 0, s>>>(deg, n, 0, k1, i1);
    size_t tmp = 0;
    check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k1, k2, i1, i2, (int)n, 0, 64, s),
               "sort size");
    void* t = arena.alloc(tmp, "sort temp");
    check_cuda(cub::DeviceRadixSort::SortPairs(t, tmp, k1, k2, i1, i2, (int)n, 0, 64, s),
               "sort");
    arena.free(t);
    arena.free(k1);
    arena.free(k2);
    arena.free(i1);
    nkey = arena_alloc<int32_t>(arena, n, "neighbour keys");
    row_of_key = arena_alloc<int32_t>(arena, R, "key to row");
    global_rank_kernel<<<grid(R), B, 0, s>>>(i2, R, c.rank, nkey, row_of_key);
    arena.free(i2);
  }
  arena.free(deg);
  check_cuda(cudaMemsetAsync(raw_ptr, 0, 8, s), "memset");
  {
    size_t tmp = 0;
    check_cuda(cub::DeviceScan::InclusiveSum(nullptr, tmp, len64, raw_ptr + 1, (int)R, s),
               "scan size");
    void* t = arena.alloc(tmp, "scan temp");
    check_cuda(cub::DeviceScan::InclusiveSum(t, tmp, len64, raw_ptr + 1, (int)R, s), "scan");
    arena.free(t);
  }
  int64_t total = 0;
  check_cuda(cudaMemcpyAsync(&total, raw_ptr + R, 8, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "total");

  // 4. placement
  int32_t* raw = arena_alloc<int32_t>(arena, total, "raw adjacency");
  uint32_t* cursor = arena_alloc<uint32_t>(arena, R, "cursor");
  check_cuda(cudaMemsetAsync(cursor, 0, R * 4, s), "memset");
  scatter_kernel<<<grid(m), B, 0, s>>>(edges, m, mirror, c.rank, nkey, raw_ptr, cursor, raw);
  if (nkey != c.rank) arena.free(nkey);
  arena.free(cursor);

  // 5. per-row sort in chunks of at most 2^30 entries
  {
    const int64_t kChunk = int64_t(1) << 30;
    int64_t* d_end = reinterpret_cast<int64_t*>(d_u64);
    int32_t* alt = arena_alloc<int32_t>(arena, std::min(total, kChunk) + 1, "sort alt");
    int32_t* rel = nullptr;
    int64_t rel_cap = 0;
    void* tmp = nullptr;
    size_t tmp_cap = 0;
    for (int64_t r0 = 0; r0 < R;) {
      chunk_end_kernel<<<1, 1, 0, s>>>(raw_ptr, R, r0, kChunk, d_end);
      int64_t r1, lo, hi;
      check_cuda(cudaMemcpyAsync(&r1, d_end, 8, cudaMemcpyDeviceToHost, s), "copy");
      check_cuda(cudaMemcpyAsync(&lo, raw_ptr + r0, 8, cudaMemcpyDeviceToHost, s), "copy");
      check_cuda(cudaStreamSynchronize(s), "chunk");
      check_cuda(cudaMemcpyAsync(&hi, raw_ptr + r1, 8, cudaMemcpyDeviceToHost, s), "copy");
      check_cuda(cudaStreamSynchronize(s), "chunk");
      const int64_t nr = r1 - r0, ni = hi - lo;
      if (ni > kChunk) throw Error{B200BFS_ERR_INVALID, "row longer than 2^30 entries"};
      if (nr + 1 > rel_cap) {
        if (rel) arena.free(rel);
        rel_cap = nr + 1;
        rel = arena_alloc<int32_t>(arena, rel_cap, "segment offsets");
      }
      rel_offsets_kernel<<<grid(nr + 1), B, 0, s>>>(raw_ptr, r0, nr, rel);
      if (ni > 1) {
        cub::DoubleBuffer<int32_t> db(raw + lo, alt);
        size_t need = 0;
        check_cuda(cub::DeviceSegmentedSort::SortKeys(nullptr, need, db, (int)ni, (int)nr, rel,
                                                       rel + 1, s),
                   "segsort size");
        if (need > tmp_cap) {
          if (tmp) arena.free(tmp);
          tmp_cap = need;
          tmp = arena.alloc(tmp_cap, "segsort temp");
        }
        check_cuda(cub::DeviceSegmentedSort::SortKeys(tmp, need, db, (int)ni, (int)nr, rel,
                                                       rel + 1, s),
                   "segsort");
        if (db.Current() != raw + lo)
          check_cuda(cudaMemcpyAsync(raw + lo, db.Current(), ni * 4, cudaMemcpyDeviceToDevice, s),
                     "copy back");
      }
      r0 = r1;
    }
    check_cuda(cudaStreamSynchronize(s), "segsort");
    if (tmp) arena.free(tmp);
    if (rel) arena.free(rel);
    arena.free(alt);
  }

  // 6. de-duplicate and compact
  int64_t* dlen = len64;
  count_distinct_kernel<<<grid(R * 32), B, 0, s>>>(raw, raw_ptr, R, dlen);
  c.row_ptr = arena_alloc<int64_t>(arena, R + 1, "row ptr");
  check_cuda(cudaMemsetAsync(c.row_ptr, 0, 8, s), "memset");
  {
    size_t tmp = 0;
    check_cuda(cub::DeviceScan::InclusiveSum(nullptr, tmp, dlen, c.row_ptr + 1, (int)R, s),
               "scan size");
    void* t = arena.alloc(tmp, "scan temp");
    check_cuda(cub::DeviceScan::InclusiveSum(t, tmp, dlen, c.row_ptr + 1, (int)R, s), "scan");
    arena.free(t);
  }
  check_cuda(cudaMemcpyAsync(&c.nedges, c.row_ptr + R, 8, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "dedup count");
  c.col = arena_alloc<int32_t>(arena, c.nedges, "adjacency");
  compact_rows_kernel<<<grid(R * 32), B, 0, s>>>(raw, raw_ptr, R, c.row_ptr, row_of_key, c.col);
  check_cuda(cudaMemsetAsync(d_u64, 0, 8, s), "memset");
  max_degree_kernel<<<grid(R), B, 0, s>>>(c.row_ptr, R, d_u64);
  unsigned long long maxd = 0;
  check_cuda(cudaMemcpyAsync(&maxd, d_u64, 8, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "compact");
  c.max_degree = (int64_t)maxd;
  arena.free(raw);
  arena.free(raw_ptr);
  arena.free(len64);
  arena.free(d_u64);
  if (row_of_key) arena.free(row_of_key);
  build_first(arena, s, c, sms);
  check_cuda(cudaGetLastError(), "build_csr");
}

void build_first(DeviceArena& arena, cudaStream_t s, Csr& c, int sms, bool parent_ids) {
  arena.free(c.first);
  arena.free(c.first_pair);
  c.first_pair = nullptr;
  c.first = arena_alloc<int32_t>(arena, c.nrows, "first neighbours");
  if (parent_ids) {
    // rounded up to whole 32-row bitmap words: the bottom-up sweep's early
    // loads read the entries of all 32 rows of a word, the last word's
    // padding rows included (their entries are discarded); the padding
    // holds (-1, -1)
    const int64_t padded = (c.nrows + 31) / 32 * 32;
    c.first_pair = arena_alloc<int2>(arena, padded, "first neighbour pairs");
    check_cuda(cudaMemsetAsync(c.first_pair, 0xFF, padded * sizeof(int2), s), "memset");
  }
  first_kernel<<<grid_for(c.nrows, 256, sms, 16), 256, 0, s>>>(c.row_ptr, c.col, c.inv, c.nrows,
                                                               c.first, c.first_pair);
  check_cuda(cudaGetLastError(), "first neighbours");
}

}  // namespace b200bfs
