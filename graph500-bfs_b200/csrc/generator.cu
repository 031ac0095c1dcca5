// Device Kronecker (R-MAT) edge generator.
//
// Produces, edge for edge, the edges of RmatGraphGenerator<Edge, 5700, 1900>
// (generator/graph_generator.hpp:781-892), the generator behind
// generate_graph_spec2010 (mpi/benchmark_helper.hpp:234-241):
//  - edge e starts from the user-seeded MRG state advanced by e * 2^64
//    (mrg_skip(&st, 0, e, 0), graph_generator.hpp:803-806);
//  - SCALE quadrant draws with initiator (A, B, C, D) = (.57, .19, .19, .05)
//    and rejection of draws below (2^32-1) mod 10000 (:818-865), with
//    clip-and-flip on the diagonal (:869-891);
//  - both endpoints go through the scramble bijection (:625-637).
// The MRG is L'Ecuyer's order-5 multiple recursive generator mod 2^31-1
// (generator/splittable_mrg.c:15-36).  Skipping ahead multiplies the state by
// a power of its 5x5 companion matrix; this file uses the binary powers
// A^(2^(64+k)), computed on the host by repeated squaring, so each thread
// enters its run of edges with at most 40 matrix-vector products and then
// steps one edge at a time with A^(2^64).  The arithmetic is exact modulo
// 2^31-1, so the states equal the reference's bit for bit.
#include <cstdint>
#include <cstring>
#include "common.cuh"
#include "engine.h"

namespace b200bfs {

namespace {

constexpr uint32_t kP = 0x7FFFFFFFu;
constexpr uint32_t kX = 107374182u;
constexpr uint32_t kY = 104480u;
constexpr int kSkipBits = 40;  // edge indices below 2^40

__constant__ uint32_t c_pow[kSkipBits][25];  // A^(2^(64+k)), row-major
__constant__ uint32_t c_seed[5];
__constant__ uint64_t c_scramble[2];

__device__ __forceinline__ uint32_t fold(uint64_t t) {
  return (uint32_t)((t & kP) + (t >> 31));  // < 2^32
}
__device__ __forceinline__ uint32_t reduce_small(uint64_t s) {
  // s < 2^36: one fold leaves < 2^31 + 32, one conditional subtract finishes.
  uint32_t r = (uint32_t)((s & kP) + (s >> 31));
  return r >= kP ? r - kP : r;
}

struct Mrg {
  uint32_t z0, z1, z2, z3, z4;  // z0 = most recent output (z1 of the reference)

  __device__ __forceinline__ uint32_t next() {
    uint32_t n = reduce_small((uint64_t)fold((uint64_t)kX * z0) + fold((uint64_t)kY * z4));
    z4 = z3;
    z3 = z2;
    z2 = z1;
    z1 = z0;
    z0 = n;
    return n;
  }
  __device__ __forceinline__ void apply(const uint32_t* m) {
    uint32_t in[5] = {z0, z1, z2, z3, z4};
    uint32_t o[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      uint64_t s = 0;
#pragma unroll
      for (int k = 0; k < 5; ++k) s += fold((uint64_t)m[i * 5 + k] * in[k]);
      o[i] = reduce_small(s);
    }
    z0 = o[0]; z1 = o[1]; z2 = o[2]; z3 = o[3]; z4 = o[4];
  }
};

__device__ __forceinline__ int draw_quadrant(Mrg& st) {
  constexpr uint32_t kLimit = 0xFFFFFFFFu % 10000u;
  uint32_t v = st.next();
  while (v < kLimit) v = st.next();
  v %= 10000u;
  if (v < 1900u) return 1;
  v -= 1900u;
  if (v < 1900u) return 2;
  v -= 1900u;
  return v < 5700u ? 0 : 3;
}

__device__ __forceinline__ uint64_t scramble(uint64_t v, int scale) {
  const uint64_t s0 = c_scramble[0], s1 = c_scramble[1];
  v += s0 + s1;
  v *= (s0 | 0x4519840211493211ull);
  v = __brevll(v) >> (64 - scale);
  v *= (s1 | 0x3050852102C843A5ull);
  v = __brevll(v) >> (64 - scale);
  return v;
}

__global__ void __launch_bounds__(256) generate_kernel(int scale, int64_t start, int64_t end,
                                                       int per_thread, uint2* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t e0 = start + t * per_thread;
  if (e0 >= end) return;
  const int64_t e1 = min(e0 + (int64_t)per_thread, end);
  Mrg st{c_seed[0], c_seed[1], c_seed[2], c_seed[3], c_seed[4]};
  for (int k = 0; k < kSkipBits; ++k)
    if ((e0 >> k) & 1) st.apply(c_pow[k]);
  const int64_t nv = int64_t(1) << scale;
  for (int64_t e = e0; e < e1; ++e) {
    Mrg w = st;
    int64_t n = nv, bs = 0, bt = 0;
    while (n > 1) {
      int sq = draw_quadrant(w);
      int so = sq >> 1, to = sq & 1;
      if (bs == bt && so > to) {
        so = 0;
        to = 1;
      }
      n >>= 1;
      bs += n * so;
      bt += n * to;
    }
    out[e - start] = make_uint2((uint32_t)scramble((uint64_t)bs, scale),
                                (uint32_t)scramble((uint64_t)bt, scale));
    st.apply(c_pow[0]);
  }
}

// ----------------------------- host tables ---------------------------------

uint32_t h_mulmod(uint32_t a, uint32_t b) { return (uint32_t)((uint64_t)a * b % kP); }

void mat_mul(const uint32_t* a, const uint32_t* b, uint32_t* c) {
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) {
      uint64_t s = 0;
      for (int k = 0; k < 5; ++k) s += h_mulmod(a[i * 5 + k], b[k * 5 + j]);
      c[i * 5 + j] = (uint32_t)(s % kP);
    }
}

void mat_apply(const uint32_t* m, uint32_t* z) {
  uint32_t o[5];
  for (int i = 0; i < 5; ++i) {
    uint64_t s = 0;
    for (int k = 0; k < 5; ++k) s += h_mulmod(m[i * 5 + k], z[k]);
    o[i] = (uint32_t)(s % kP);
  }
  memcpy(z, o, sizeof(o));
}

struct PowTable {
  uint32_t p[192][25];
  PowTable() {
    uint32_t a[25] = {0};
    a[0] = kX;
    a[4] = kY;
    a[5] = 1;
    a[11] = 1;
    a[17] = 1;
    a[23] = 1;
    memcpy(p[0], a, sizeof(a));
    for (int k = 1; k < 192; ++k) mat_mul(p[k - 1], p[k - 1], p[k]);
  }
};

const PowTable& pow_table() {
  static PowTable t;
  return t;
}

}  // namespace

void host_seed_state(uint64_t s1, uint64_t s2, uint32_t z[5]) {
  z[0] = (uint32_t)(s1 & 0x3FFFFFFF) + 1;
  z[1] = (uint32_t)((s1 >> 30) & 0x3FFFFFFF) + 1;
  z[2] = (uint32_t)(s2 & 0x3FFFFFFF) + 1;
  z[3] = (uint32_t)((s2 >> 30) & 0x3FFFFFFF) + 1;
  z[4] = (uint32_t)((s2 >> 60) << 4) + (uint32_t)(s1 >> 60) + 1;
}

void host_mrg_skip(uint32_t z[5], uint64_t hi, uint64_t mid, uint64_t lo) {
  const PowTable& t = pow_table();
  uint64_t w[3] = {lo, mid, hi};
  for (int q = 0; q < 3; ++q)
    for (int b = 0; b < 64; ++b)
      if ((w[q] >> b) & 1) mat_apply(t.p[q * 64 + b], z);
}

uint32_t host_mrg_next(uint32_t z[5]) {
  uint32_t n = (uint32_t)(((uint64_t)h_mulmod(kX, z[0]) + h_mulmod(kY, z[4])) % kP);
  z[4] = z[3];
  z[3] = z[2];
  z[2] = z[1];
  z[1] = z[0];
  z[0] = n;
  return n;
}

void host_scramble_values(uint64_t s1, uint64_t s2, uint64_t* v0, uint64_t* v1) {
  uint32_t z[5];
  host_seed_state(s1, s2, z);
  host_mrg_skip(z, 50, 7, 0);  // GraphGeneratorBase, graph_generator.hpp:541-551
  uint64_t a = host_mrg_next(z);
  a *= 0xFFFFFFFFull;
  a += host_mrg_next(z);
  uint64_t b = host_mrg_next(z);
  b *= 0xFFFFFFFFull;
  b += host_mrg_next(z);
  *v0 = a;
  *v1 = b;
}

// make_random_numbers (graph_generator.hpp:506-520): two MRG outputs per
// double, (2^31-1)^-1 and (2^31-1)^-2 weights (splittable_mrg.c:330-337).
double host_random_double(uint64_t s1, uint64_t s2, int64_t position) {
  uint32_t z[5];
  host_seed_state(s1, s2, z);
  host_mrg_skip(z, 2, 0, 2 * (uint64_t)position);
  const double a = (double)host_mrg_next(z) * 4.656612875245796924105750827e-10;
  const double b = (double)host_mrg_next(z) * 2.168404346990492787e-19;
  return a + b;
}

// find_roots (mpi/benchmark_helper.hpp:527-562) with USERSEED1/2 = 2/3: the
// counter advances by two doubles per candidate; duplicates and vertices
// without edges are skipped; after 2*nglobalverts candidates the last one is
// taken as is.
void find_roots_host(const uint8_t* has_edge, int64_t nglobal, int num_roots, int r1, int r2,
                     int64_t* roots) {
  int64_t counter = 0;
  for (int idx = 0; idx < num_roots; ++idx) {
    int64_t root = 0;
    for (;;) {
      uint32_t z[5];
      host_seed_state(2 + (uint64_t)r1, 3 + (uint64_t)r2, z);
      host_mrg_skip(z, 2, 0, 2 * (uint64_t)counter);
      const double d0a = (double)host_mrg_next(z) * 4.656612875245796924105750827e-10;
      const double d0b = (double)host_mrg_next(z) * 2.168404346990492787e-19;
      const double d1a = (double)host_mrg_next(z) * 4.656612875245796924105750827e-10;
      const double d1b = (double)host_mrg_next(z) * 2.168404346990492787e-19;
      const double d0 = d0a + d0b, d1 = d1a + d1b;
      root = (int64_t)((d0 + d1) * (double)nglobal) % nglobal;
      counter += 2;
      if (counter > 2 * nglobal) break;
      bool dup = false;
      for (int i = 0; i < idx; ++i)
        if (roots[i] == root) {
          dup = true;
          break;
        }
      if (dup) continue;
      if (has_edge[root]) break;
    }
    roots[idx] = root;
  }
}

cudaError_t launch_generate(int scale, uint64_t seed1, uint64_t seed2, int64_t start, int64_t end,
                            uint2* out, cudaStream_t stream) {
  // The tables are re-sent on every call: constant memory is per device and
  // the copy is a few kilobytes.
  {
    cudaError_t err;
    const PowTable& t = pow_table();
    uint32_t z[5];
    host_seed_state(seed1, seed2, z);
    uint64_t sc[2];
    host_scramble_values(seed1, seed2, &sc[0], &sc[1]);
    if ((err = cudaMemcpyToSymbolAsync(c_pow, t.p[64], sizeof(uint32_t) * 25 * kSkipBits, 0,
                                       cudaMemcpyHostToDevice, stream)) != cudaSuccess)
      return err;
    if ((err = cudaMemcpyToSymbolAsync(c_seed, z, sizeof(z), 0, cudaMemcpyHostToDevice, stream)) !=
        cudaSuccess)
      return err;
    if ((err = cudaMemcpyToSymbolAsync(c_scramble, sc, sizeof(sc), 0, cudaMemcpyHostToDevice,
                                       stream)) != cudaSuccess)
      return err;
    // The host arrays above are stack temporaries: wait for the copies.
    if ((err = cudaStreamSynchronize(stream)) != cudaSuccess) return err;
  }
  if (end <= start) return cudaSuccess;
  if (end > (int64_t(1) << kSkipBits)) return cudaErrorInvalidValue;
  const int per_thread = 32;
  const int64_t threads = (end - start + per_thread - 1) / per_thread;
  const int block = 256;
  const int64_t grid = (threads + block - 1) / block;
  generate_kernel<<<(unsigned)grid, block, 0, stream>>>(scale, start, end, per_thread, out);
  return cudaGetLastError();
}

}  // namespace b200bfs
