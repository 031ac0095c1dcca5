// Golden-vector driver: runs the reference's own Kronecker generator
// (generator/graph_generator.hpp RmatGraphGenerator<...,5700,1900>, the one
// generate_graph_spec2010 uses, mpi/benchmark_helper.hpp:234-241) and its
// make_random_numbers (graph_generator.hpp:506-520), compiled unchanged from
// the reference tree, and prints edge ranges and doubles as text.
// Build + run: oracle/ref/make_golden.sh (writes tests/golden/).
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "../generator/graph_generator.hpp"

StubMpiGlobals mpi;
void print_with_prefix(const char*, ...) {}
void* cache_aligned_xmalloc(size_t size) { return malloc(size); }

int main(int argc, char** argv) {
  // edges: scale start count
  static const long long ranges[][3] = {
      {10, 0, 500},            {10, 14384, 500},   {16, 0, 500},
      {16, 1048576 - 500, 500},  {20, 123456, 500},  {28, 0, 500},
      {28, 2147483648LL, 500},  {28, 4294967296LL - 500, 500}};
  for (const auto& r : ranges) {
    RmatGraphGenerator<UnweightedPackedEdge, 5700, 1900> gen((int)r[0], 16, 255, 2, 3,
                                                              InitialEdgeType::NONE);
    std::vector<UnweightedPackedEdge> buf(r[2]);
    gen.generateRange(buf.data(), r[1], r[1] + r[2]);
    for (long long i = 0; i < r[2]; ++i)
      printf("E %lld %lld %lld %lld\n", r[0], r[1] + i, (long long)buf[i].v0(),
             (long long)buf[i].v1());
  }
  // make_random_numbers(n, s1, s2, position): find_roots uses (2+r1, 3+r2)
  static const long long rn[][3] = {{2, 3, 0}, {2, 3, 1}, {2, 3, 1000}, {3, 3, 0}, {2, 3, 123457},
                                    {7, 3, 99}, {2, 3, 1LL << 33}};
  for (const auto& q : rn) {
    double d[4];
    make_random_numbers(4, (uint64_t)q[0], (uint64_t)q[1], q[2], d);
    for (int i = 0; i < 4; ++i) printf("R %lld %lld %lld %d %.17g\n", q[0], q[1], q[2], i, d[i]);
  }
  return 0;
}
