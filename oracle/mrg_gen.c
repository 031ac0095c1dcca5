/*
 * Oracle: multiple recursive generator, skip-ahead and the Kronecker edge
 * generator.  TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The generator is the one main.cc uses: generate_graph_spec2010
 * (mpi/benchmark_helper.hpp:234-241) -> RmatGraphGenerator<Edge, 5700, 1900>
 * (generator/graph_generator.hpp:781-892) with user seeds (2, 3)
 * (mpi/parameters.h:204-205).
 *
 * The MRG is L'Ecuyer's order-5 generator modulo 2^31-1 with multipliers
 * x = 107374182 (lag 1) and y = 104480 (lag 5)
 * (generator/splittable_mrg.c:15-36).  Skip-ahead multiplies the state by a
 * power of the 5x5 companion matrix; the powers A^(2^k) are built here by
 * repeated squaring, which is exact modular arithmetic, so any evaluation
 * order gives the reference's state bit for bit.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include "oracle.h"

#define MRG_P 0x7FFFFFFFu
#define MRG_X 107374182u
#define MRG_Y 104480u

/* a*b mod (2^31-1) for a, b < 2^31 (Mersenne fold). */
static inline uint32_t mmul(uint32_t a, uint32_t b) {
  uint64_t t = (uint64_t)a * b;
  uint64_t r = (t & MRG_P) + (t >> 31);
  r = (r & MRG_P) + (r >> 31);
  return (uint32_t)(r >= MRG_P ? r - MRG_P : r);
}

static inline uint32_t mred64(uint64_t t) {
  uint64_t r = (t & MRG_P) + (t >> 31);
  r = (r & MRG_P) + (r >> 31);
  r = (r & MRG_P) + (r >> 31);
  return (uint32_t)(r >= MRG_P ? r - MRG_P : r);
}

/* Row-major 5x5 product c = a * b mod p (c may alias neither). */
static void mat_mul(const uint32_t* a, const uint32_t* b, uint32_t* c) {
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) {
      uint64_t s = 0;
      for (int k = 0; k < 5; ++k) s += (uint64_t)mmul(a[i * 5 + k], b[k * 5 + j]);
      c[i * 5 + j] = mred64(s);
    }
}

/* state z <- M z */
static void mat_apply(const uint32_t* m, orc_mrg_state* st) {
  uint32_t o[5];
  for (int i = 0; i < 5; ++i) {
    uint64_t s = 0;
    for (int k = 0; k < 5; ++k) s += (uint64_t)mmul(m[i * 5 + k], st->z[k]);
    o[i] = mred64(s);
  }
  memcpy(st->z, o, sizeof(o));
}

static uint32_t g_pow2[192][25];
static pthread_once_t g_pow2_once = PTHREAD_ONCE_INIT;

static void build_pow2(void) {
  /* Companion matrix of z1' = x z1 + y z5, zi' = z(i-1). */
  uint32_t a[25] = {0};
  a[0 * 5 + 0] = MRG_X;
  a[0 * 5 + 4] = MRG_Y;
  a[1 * 5 + 0] = 1;
  a[2 * 5 + 1] = 1;
  a[3 * 5 + 2] = 1;
  a[4 * 5 + 3] = 1;
  memcpy(g_pow2[0], a, sizeof(a));
  for (int k = 1; k < 192; ++k) mat_mul(g_pow2[k - 1], g_pow2[k - 1], g_pow2[k]);
}

void orc_mrg_pow2_matrix(int k, uint32_t out[25]) {
  pthread_once(&g_pow2_once, build_pow2);
  memcpy(out, g_pow2[k], sizeof(g_pow2[k]));
}

void orc_mrg_seed_from_user(uint64_t s1, uint64_t s2, orc_mrg_state* st) {
  st->z[0] = (uint32_t)(s1 & 0x3FFFFFFF) + 1;
  st->z[1] = (uint32_t)((s1 >> 30) & 0x3FFFFFFF) + 1;
  st->z[2] = (uint32_t)(s2 & 0x3FFFFFFF) + 1;
  st->z[3] = (uint32_t)((s2 >> 30) & 0x3FFFFFFF) + 1;
  st->z[4] = (uint32_t)((s2 >> 60) << 4) + (uint32_t)(s1 >> 60) + 1;
}

uint32_t orc_mrg_next(orc_mrg_state* st) {
  uint32_t nz = mred64((uint64_t)mmul(MRG_X, st->z[0]) + mmul(MRG_Y, st->z[4]));
  st->z[4] = st->z[3];
  st->z[3] = st->z[2];
  st->z[2] = st->z[1];
  st->z[1] = st->z[0];
  st->z[0] = nz;
  return nz;
}

/* (2^31-1)^-1 and (2^31-1)^-2 */
#define MRG_INV1 4.656612875245796924105750827e-10
#define MRG_INV2 2.168404346990492787e-19

double orc_mrg_next_double(orc_mrg_state* st) {
  /* Both operands are evaluated left to right as in the reference
   * expression (splittable_mrg.c:330-336). */
  double a = (double)orc_mrg_next(st) * MRG_INV1;
  double b = (double)orc_mrg_next(st) * MRG_INV2;
  return a + b;
}

void orc_mrg_skip(orc_mrg_state* st, uint64_t hi, uint64_t mid, uint64_t lo) {
  pthread_once(&g_pow2_once, build_pow2);
  uint64_t w[3] = {lo, mid, hi};
  for (int q = 0; q < 3; ++q)
    for (int b = 0; b < 64; ++b)
      if ((w[q] >> b) & 1) mat_apply(g_pow2[q * 64 + b], st);
}

void orc_make_random_numbers(int64_t nvalues, uint64_t s1, uint64_t s2,
                             int64_t position, double* result) {
  orc_mrg_state st;
  orc_mrg_seed_from_user(s1, s2, &st);
  orc_mrg_skip(&st, 2, 0, 2 * (uint64_t)position);
  for (int64_t i = 0; i < nvalues; ++i) result[i] = orc_mrg_next_double(&st);
}

/* ----------------------------- generator -------------------------------- */

void orc_scramble_values(uint64_t s1, uint64_t s2, uint64_t* val0,
                         uint64_t* val1) {
  orc_mrg_state st;
  orc_mrg_seed_from_user(s1, s2, &st);
  orc_mrg_skip(&st, 50, 7, 0);
  uint64_t v0 = orc_mrg_next(&st);
  v0 *= UINT64_C(0xFFFFFFFF);
  v0 += orc_mrg_next(&st);
  uint64_t v1 = orc_mrg_next(&st);
  v1 *= UINT64_C(0xFFFFFFFF);
  v1 += orc_mrg_next(&st);
  *val0 = v0;
  *val1 = v1;
}

static inline uint64_t bitrev64(uint64_t x) {
  x = __builtin_bswap64(x);
  x = ((x >> 4) & UINT64_C(0x0F0F0F0F0F0F0F0F)) | ((x & UINT64_C(0x0F0F0F0F0F0F0F0F)) << 4);
  x = ((x >> 2) & UINT64_C(0x3333333333333333)) | ((x & UINT64_C(0x3333333333333333)) << 2);
  x = ((x >> 1) & UINT64_C(0x5555555555555555)) | ((x & UINT64_C(0x5555555555555555)) << 1);
  return x;
}

int64_t orc_scramble(int64_t v0, int scale, uint64_t val0, uint64_t val1) {
  uint64_t v = (uint64_t)v0;
  v += val0 + val1;
  v *= (val0 | UINT64_C(0x4519840211493211));
  v = bitrev64(v) >> (64 - scale);
  v *= (val1 | UINT64_C(0x3050852102C843A5));
  v = bitrev64(v) >> (64 - scale);
  return (int64_t)v;
}

/* 4-way Bernoulli draw with initiator (A, B, C) = (5700, 1900, 1900)/10000
 * and rejection of draws below 2^32-1 mod 10000
 * (graph_generator.hpp:830-865, limit at :818-819). */
static inline int draw_quadrant(orc_mrg_state* st) {
  const uint32_t limit = UINT32_C(0xFFFFFFFF) % 10000u;
  uint32_t val = orc_mrg_next(st);
  while (val < limit) val = orc_mrg_next(st);
  val %= 10000u;
  if (val < 1900u) return 1;
  val -= 1900u;
  if (val < 1900u) return 2;
  val -= 1900u;
  if (val < 5700u) return 0;
  return 3;
}

void orc_generate_edges(int scale, uint64_t s1, uint64_t s2, int64_t start,
                        int64_t end, int64_t* out) {
  pthread_once(&g_pow2_once, build_pow2);
  orc_mrg_state seed;
  orc_mrg_seed_from_user(s1, s2, &seed);
  uint64_t val0, val1;
  orc_scramble_values(s1, s2, &val0, &val1);
  const int64_t nv = INT64_C(1) << scale;
  /* Each edge e uses the seed advanced by e * 2^64 (mrg_skip(0, e, 0),
   * graph_generator.hpp:803-806).  A chunk is entered by skipping once and
   * then stepping by A^(2^64) per edge. */
  const uint32_t* step = g_pow2[64];
  const int64_t CH = 4096;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t c0 = start; c0 < end; c0 += CH) {
    const int64_t c1 = c0 + CH < end ? c0 + CH : end;
    orc_mrg_state st = seed;
    orc_mrg_skip(&st, 0, (uint64_t)c0, 0);
    for (int64_t e = c0; e < c1; ++e) {
      orc_mrg_state w = st;
      int64_t n = nv, bs = 0, bt = 0;
      while (n > 1) {
        int sq = draw_quadrant(&w);
        int so = sq / 2, to = sq % 2;
        if (bs == bt && so > to) {
          int t = so;
          so = to;
          to = t;
        }
        n /= 2;
        bs += n * so;
        bt += n * to;
      }
      out[2 * (e - start) + 0] = orc_scramble(bs, scale, val0, val1);
      out[2 * (e - start) + 1] = orc_scramble(bt, scale, val0, val1);
      mat_apply(step, &st);
    }
  }
}
