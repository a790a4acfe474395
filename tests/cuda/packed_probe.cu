// Checks the search kernels' packed FP32x2 distance (packed.cuh: dist2_pair) against the
// scalar reference-order distance (common.cuh: dist2_ref) bit for bit, on 2^24 random
// pairs of candidates for each of three value ranges: uniform in [0, 1), clustered near
// 1000 (large coordinates, small differences), and random exponents over 2^-37 .. 2^32.
// Prints one line per range, "range R: D of N distances differ", and exits 1 on any
// difference or CUDA error.
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
#include "packed.cuh"

namespace {

__device__ __forceinline__ uint32_t mix(uint32_t x) {   // 32-bit integer hash
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}

__device__ __forceinline__ float value(uint32_t s, int range) {
  const uint32_t h = mix(s);
  const float u = (float)(h >> 8) * (1.0f / 16777216.0f);
  if (range == 0) return u;
  if (range == 1) return 1000.f + u * 0.01f;
  const uint32_t e = 90u + mix(s * 7u + 1u) % 70u;   // biased exponent 90 .. 159
  return __uint_as_float((h & 0x807fffffu) | (e << 23));
}

__global__ void k_probe(uint32_t n, int range, unsigned long long* differ) {
  unsigned long long nd = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t s = i * 9u + (uint32_t)range * 0x9e3779b9u;
    float v[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) v[j] = value(s + j, range);
    uint32_t d0, d1;
    rtnn::dist2_pair(rtnn::pk2(v[0], v[0]), rtnn::pk2(v[1], v[1]), rtnn::pk2(v[2], v[2]),
                     rtnn::pk2(v[3], v[6]), rtnn::pk2(v[4], v[7]), rtnn::pk2(v[5], v[8]), d0, d1);
    const uint32_t r0 = __float_as_uint(rtnn::dist2_ref(v[0], v[1], v[2], v[3], v[4], v[5]));
    const uint32_t r1 = __float_as_uint(rtnn::dist2_ref(v[0], v[1], v[2], v[6], v[7], v[8]));
    nd += (d0 != r0) + (d1 != r1);
  }
  atomicAdd(differ, nd);
}

}  // namespace

int main() {
  unsigned long long* differ = nullptr;
  if (cudaMalloc(&differ, sizeof(unsigned long long)) != cudaSuccess) return 1;
  int rc = 0;
  const uint32_t n = 1u << 24;
  for (int range = 0; range < 3; ++range) {
    unsigned long long h = ~0ull;
    cudaMemset(differ, 0, sizeof(h));
    k_probe<<<1184, 256>>>(n, range, differ);
    const cudaError_t e = cudaMemcpy(&h, differ, sizeof(h), cudaMemcpyDeviceToHost);
    std::printf("range %d: %llu of %u distances differ (%s)\n", range, h, 2 * n,
                cudaGetErrorString(e));
    if (e != cudaSuccess || h != 0) rc = 1;
  }
  cudaFree(differ);
  return rc;
}
