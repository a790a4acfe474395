// radix_sort.cu -- stable LSD radix sort of (key, uint32 value) pairs, 8-bit digits.
//
// Replaces the CUB radix sorts behind thrust::sort_by_key in the reference
// (thrust_helper.cu:13-43; call sites sort.cpp:415,487-488,612). Used to put queries
// in (cloud, density bucket, Hilbert index) order. Each pass: (1) per-tile digit
// histograms, column-major [digit][tile]; (2) one exclusive scan of that table (scan.cu),
// giving every (digit, tile) its global output offset; (3) a stable scatter: each warp ranks its
// sub-tile with __match_any_sync, warps are combined through a shared-memory prefix per
// digit, the tile is placed in digit order in shared memory, and written out from there
// so that consecutive threads write consecutive output positions of a digit's run (keys
// keep their input order within a digit).
#include "common.cuh"
#include "kernels.h"

namespace rtnn {
namespace {

constexpr int kWarps = kRadixThreads / 32;
constexpr int kSub = 32 * kRadixItems;   // keys per warp sub-tile

template <typename KeyT>
__global__ void __launch_bounds__(kRadixThreads)
k_radix_hist(const KeyT* __restrict__ keys, uint32_t n, uint32_t shift, uint32_t dmask,
             uint32_t* __restrict__ hist, uint32_t n_tiles) {
  __shared__ uint32_t s_h[kWarps][256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kWarps * 256; i += blockDim.x) (&s_h[0][0])[i] = 0u;
  __syncthreads();
  const uint32_t base = blockIdx.x * (uint32_t)kRadixTile + warp * kSub;
#pragma unroll 4
  for (int it = 0; it < kRadixItems; ++it) {
    const uint32_t i = base + it * 32 + lane;
    if (i < n) atomicAdd(&s_h[warp][(uint32_t)(keys[i] >> shift) & dmask], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x) {
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s += s_h[w][d];
    hist[(uint64_t)d * n_tiles + blockIdx.x] = s;
  }
}

template <typename KeyT>
__global__ void __launch_bounds__(kRadixThreads)
k_radix_scatter(const KeyT* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                KeyT* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n,
                uint32_t shift, uint32_t dmask, const uint32_t* __restrict__ offsets,
                uint32_t n_tiles) {
  __shared__ uint32_t s_cnt[kWarps][256];   // per warp and digit: count, then tile position
  __shared__ uint32_t s_start[256];         // per digit: first tile position
  __shared__ uint32_t s_dst[256];           // per digit: global offset minus s_start
  __shared__ KeyT s_keys[kRadixTile];       // the tile in digit order
  __shared__ uint32_t s_vals[kRadixTile];
  __shared__ uint32_t s_wsum[kRadixThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kWarps * 256; i += blockDim.x) (&s_cnt[0][0])[i] = 0u;
  __syncthreads();
  const uint32_t base = blockIdx.x * (uint32_t)kRadixTile + warp * kSub;
  KeyT k[kRadixItems];
  uint32_t v[kRadixItems], rk[kRadixItems];
  const uint32_t lt = lanemask_lt();
  // 1. rank every key among the equal digits of its warp, in input order
#pragma unroll
  for (int it = 0; it < kRadixItems; ++it) {
    const uint32_t i = base + it * 32 + lane;
    const bool valid = i < n;
    k[it] = valid ? keys_in[i] : (KeyT)0;
    v[it] = valid ? (vals_in ? vals_in[i] : i) : 0u;
    const uint32_t digit = valid ? ((uint32_t)(k[it] >> shift) & dmask) : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, digit);
    uint32_t before = 0;
    if (valid) before = s_cnt[warp][digit];
    __syncwarp();
    rk[it] = before + __popc(peers & lt);
    if (valid && (peers & lt) == 0) s_cnt[warp][digit] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // 2. tile positions: digits in order, warps in order within a digit (stable)
  static_assert(kRadixThreads == 256, "one thread per digit");
  {
    const int d = threadIdx.x;
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) tot += s_cnt[w][d];
    // exclusive scan of the 256 digit totals: warp scans, then the warp sums
    uint32_t incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += x;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += s_wsum[w];
    const uint32_t start = before + incl - tot;
    s_start[d] = start;
    s_dst[d] = offsets[(uint64_t)d * n_tiles + blockIdx.x] - start;
    uint32_t run = start;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t c = s_cnt[w][d];
      s_cnt[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
  // 3. the tile into shared memory in digit order
#pragma unroll
  for (int it = 0; it < kRadixItems; ++it) {
    const uint32_t i = base + it * 32 + lane;
    if (i < n) {
      const uint32_t digit = (uint32_t)(k[it] >> shift) & dmask;
      const uint32_t li = s_cnt[warp][digit] + rk[it];
      s_keys[li] = k[it];
      s_vals[li] = v[it];
    }
  }
  __syncthreads();
  // 4. consecutive tile positions of one digit go to consecutive output positions
  const uint32_t count = min((uint32_t)kRadixTile, n - blockIdx.x * (uint32_t)kRadixTile);
  for (uint32_t j = threadIdx.x; j < count; j += blockDim.x) {
    const KeyT key = s_keys[j];
    const uint32_t dst = s_dst[(uint32_t)(key >> shift) & dmask] + j;
    keys_out[dst] = key;
    vals_out[dst] = s_vals[j];
  }
}

}  // namespace

uint32_t radix_tiles_for(uint64_t n) { return (uint32_t)((n + kRadixTile - 1) / kRadixTile); }

// Sorts n pairs on bits [0, bits) (bits above are ignored). Ping-pongs between (keys0, vals0) and (keys1, vals1);
// *result_in_1 tells where the sorted pairs ended up. identity_values: the first pass
// reads value i for position i instead of vals0.
cudaError_t radix_sort_pairs(bool key64, void* keys0, uint32_t* vals0, void* keys1,
                             uint32_t* vals1, uint32_t n, uint32_t bits, bool identity_values,
                             uint32_t* hist, uint64_t* scan_state, uint32_t* scan_counters,
                             Counters* ctr, bool* result_in_1, cudaStream_t s) {
  *result_in_1 = false;
  if (n == 0) return cudaSuccess;
  const uint32_t n_tiles = radix_tiles_for(n);
  const uint32_t passes = (bits + 7) / 8;
  bool in1 = false;
  cudaError_t e = cudaSuccess;
  for (uint32_t p = 0; p < passes; ++p) {
    void* kin = in1 ? keys1 : keys0;
    void* kout = in1 ? keys0 : keys1;
    const uint32_t* vin = (p == 0 && identity_values) ? nullptr : (in1 ? vals1 : vals0);
    uint32_t* vout = in1 ? vals0 : vals1;
    const uint32_t shift = 8 * p;
    // the last pass sorts only the bits below `bits` (keys may hold more above them)
    const uint32_t dmask = bits - shift >= 8 ? 0xffu : (1u << (bits - shift)) - 1u;
    if (key64)
      k_radix_hist<uint64_t><<<n_tiles, kRadixThreads, 0, s>>>((const uint64_t*)kin, n, shift,
                                                                dmask, hist, n_tiles);
    else
      k_radix_hist<uint32_t><<<n_tiles, kRadixThreads, 0, s>>>((const uint32_t*)kin, n, shift,
                                                                dmask, hist, n_tiles);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const uint64_t hn = 256ull * n_tiles;
    e = launch_scan_excl(hist, hn, nullptr, 0, hn, scan_state, scan_counters + p, ctr, s);
    if (e != cudaSuccess) return e;
    if (key64)
      k_radix_scatter<uint64_t><<<n_tiles, kRadixThreads, 0, s>>>(
          (const uint64_t*)kin, vin, (uint64_t*)kout, vout, n, shift, dmask, hist, n_tiles);
    else
      k_radix_scatter<uint32_t><<<n_tiles, kRadixThreads, 0, s>>>(
          (const uint32_t*)kin, vin, (uint32_t*)kout, vout, n, shift, dmask, hist, n_tiles);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    in1 = !in1;
  }
  *result_in_1 = in1;
  return cudaSuccess;
}

}  // namespace rtnn
