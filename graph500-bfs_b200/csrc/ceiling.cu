// Random-access ceiling of the device: how many independent random 4-byte
// loads, or non-returning ORs (RED), the SMs issue per second into a buffer
// of a given size.  A top-down level is made of exactly these accesses (one
// visited-bitmap probe per adjacency entry, one OR per claim, into a bitmap
// of R / 8 bytes that L2 holds), so its rate, not the HBM bandwidth, is the
// ceiling its kernels are measured against beside the HBM roofline.
#include <cstdint>
#include <cuda_runtime.h>

#include "b200bfs.h"

namespace b200bfs {
namespace {

constexpr int kThreads = 256;
constexpr int kBlocksPerSm = 8;
constexpr int kIters = 1024;  // accesses per thread, a multiple of 4

__device__ __forceinline__ uint32_t xorshift(uint32_t h) {
  h ^= h << 13;
  h ^= h >> 17;
  h ^= h << 5;
  return h;
}

// Four accesses per step, with addresses that do not depend on loaded data,
// so they are all in flight together, as the probes of a top-down step are.
template <int kKind>
__global__ void __launch_bounds__(kThreads) random_access_kernel(uint32_t* words, uint32_t mask,
                                                                 uint32_t* sink) {
  uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u + 12345u;
  uint32_t acc = 0;
  for (int i = 0; i < kIters; i += 4) {
    const uint32_t a0 = (h = xorshift(h)) & mask;
    const uint32_t a1 = (h = xorshift(h)) & mask;
    const uint32_t a2 = (h = xorshift(h)) & mask;
    const uint32_t a3 = (h = xorshift(h)) & mask;
    if (kKind == 0) {
      acc += words[a0] + words[a1] + words[a2] + words[a3];
    } else {
      atomicOr(words + a0, 1u << (h & 31));
      atomicOr(words + a1, 1u << ((h >> 5) & 31));
      atomicOr(words + a2, 1u << ((h >> 10) & 31));
      atomicOr(words + a3, 1u << ((h >> 15) & 31));
    }
  }
  if (kKind == 0 && acc == 0x9e3779b9u) sink[0] = acc;  // keeps the loads
}

}  // namespace
}  // namespace b200bfs

extern "C" int b200bfs_random_access_rate(void* words, int log2_words, int kind, void* stream,
                                          double* per_s) {
  using namespace b200bfs;
  if (!words || !per_s || log2_words < 10 || log2_words > 30 || (kind != 0 && kind != 1) ||
      (reinterpret_cast<uintptr_t>(words) & 3) != 0)
    return B200BFS_ERR_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      sms < 1) {
    cudaGetLastError();
    return B200BFS_ERR_CUDA;
  }
  uint32_t* w = static_cast<uint32_t*>(words);
  const uint32_t mask = (1u << log2_words) - 1u;  // every address is inside the buffer
  const int grid = sms * kBlocksPerSm;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    return B200BFS_ERR_CUDA;
  }
  float best = 0.f;
  cudaError_t err = cudaSuccess;
  for (int rep = 0; rep < 4 && err == cudaSuccess; ++rep) {  // one warm-up, then the best of 3
    cudaEventRecord(e0, s);
    if (kind == 0)
      random_access_kernel<0><<<grid, kThreads, 0, s>>>(w, mask, w);
    else
      random_access_kernel<1><<<grid, kThreads, 0, s>>>(w, mask, w);
    cudaEventRecord(e1, s);
    err = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    if (err == cudaSuccess && rep > 0 && (best == 0.f || ms < best)) best = ms;
  }
  if (err == cudaSuccess) err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess || best <= 0.f) {
    cudaGetLastError();
    return B200BFS_ERR_CUDA;
  }
  *per_s = (double)grid * kThreads * kIters / (best * 1e-3);
  return B200BFS_OK;
}
