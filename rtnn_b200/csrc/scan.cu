// scan.cu -- single-pass exclusive scan of uint32 with decoupled look-back.
//
// Replaces thrust::exclusive_scan of the reference (thrust_helper.cu:79-91, called at
// sort.cpp:547 to turn per-cell counts into cell offsets). One pass over HBM: each
// block scans a 4096-element tile, publishes its aggregate, and its first warp looks
// back over predecessors 32 at a time until it meets an inclusive prefix. Tiles are
// claimed from an atomic counter, so a block only waits on blocks that started
// earlier. Every wait is bounded: after kSpinLimit polls the block records
// kErrScanTimeout and carries on, so the host sees an error status instead of a hang.
#include "common.cuh"
#include "kernels.h"

namespace rtnn {
namespace {

constexpr uint32_t kFlagAggregate = 1u;
constexpr uint32_t kFlagPrefix = 2u;
constexpr uint32_t kSpinLimit = 1u << 22;   // polls per predecessor window (~1 s with backoff)

__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// n may live on the device (n_dev != nullptr: n = *n_dev + n_add), so the scan can
// run inside a captured graph whose sizes are only known on the device.
__global__ void __launch_bounds__(kScanThreads)
k_scan_excl(uint32_t* __restrict__ data, uint64_t n_host, const uint32_t* n_dev,
            uint32_t n_add, uint64_t* __restrict__ tile_state, uint32_t* tile_counter,
            Counters* ctr) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_prefix;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t n = n_dev ? (uint64_t)(*n_dev) + n_add : n_host;
  const uint64_t tile_start = (uint64_t)tile * kScanTile;
  if (tile_start >= n) return;   // surplus block of a device-sized scan
  const uint64_t base = tile_start + (uint64_t)tid * kScanItems;

  uint32_t v[kScanItems];
  if (base + kScanItems <= n) {
    const uint4* p4 = reinterpret_cast<const uint4*>(data + base);
#pragma unroll
    for (int i = 0; i < kScanItems / 4; ++i) {
      uint4 t = p4[i];
      v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) v[i] = (base + i < n) ? data[base + i] : 0u;
  }
  uint32_t sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) sum += v[i];

  uint32_t incl = warp_incl_scan(sum, lane);
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = (lane < kScanThreads / 32) ? s_warp[lane] : 0u;
    uint32_t wi = warp_incl_scan(w, lane);
    if (lane < kScanThreads / 32) s_warp[lane] = wi - w;   // exclusive warp offsets
    const uint32_t aggregate = __shfl_sync(0xffffffffu, wi, kScanThreads / 32 - 1);
    uint32_t prefix = 0;
    if (tile == 0) {
      if (lane == 0) st_relaxed(&tile_state[0], ((uint64_t)kFlagPrefix << 32) | aggregate);
    } else {
      if (lane == 0) st_relaxed(&tile_state[tile], ((uint64_t)kFlagAggregate << 32) | aggregate);
      int64_t look = (int64_t)tile - 1;
      uint32_t spins = 0;
      bool timed_out = false;
      while (true) {
        const int64_t idx = look - lane;
        uint64_t st = (idx >= 0) ? ld_relaxed(&tile_state[idx])
                                 : ((uint64_t)kFlagPrefix << 32);
        uint32_t flag = (uint32_t)(st >> 32);
        if (__any_sync(0xffffffffu, flag == 0u)) {
          if (++spins > kSpinLimit) {
            if (lane == 0) set_error(ctr, kErrScanTimeout, tile);
            timed_out = true;
            break;
          }
          __nanosleep(spins < 64 ? 32 : 256);
          continue;
        }
        const uint32_t val = (uint32_t)st;
        const uint32_t pmask = __ballot_sync(0xffffffffu, flag == kFlagPrefix);
        if (pmask) {
          const int first = __ffs(pmask) - 1;   // nearest predecessor with a full prefix
          uint32_t part = (lane <= first) ? val : 0u;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
          prefix += part;
          break;
        }
        uint32_t part = val;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        prefix += part;
        look -= 32;
        spins = 0;
      }
      (void)timed_out;
      if (lane == 0)
        st_relaxed(&tile_state[tile], ((uint64_t)kFlagPrefix << 32) | (prefix + aggregate));
    }
    if (lane == 0) s_prefix = prefix;
  }
  __syncthreads();
  uint32_t run = s_prefix + s_warp[warp] + (incl - sum);
  uint32_t out[kScanItems];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) { out[i] = run; run += v[i]; }
  if (base + kScanItems <= n) {
    uint4* p4 = reinterpret_cast<uint4*>(data + base);
#pragma unroll
    for (int i = 0; i < kScanItems / 4; ++i)
      p4[i] = make_uint4(out[4 * i], out[4 * i + 1], out[4 * i + 2], out[4 * i + 3]);
  } else {
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
      if (base + i < n) data[base + i] = out[i];
  }
}

}  // namespace

uint64_t scan_tiles_for(uint64_t n) { return (n + kScanTile - 1) / kScanTile; }

cudaError_t launch_scan_excl(uint32_t* data, uint64_t n_host, const uint32_t* n_dev,
                             uint32_t n_add, uint64_t max_n, uint64_t* tile_state,
                             uint32_t* tile_counter, Counters* ctr, cudaStream_t s) {
  const uint64_t tiles = scan_tiles_for(max_n);
  if (tiles == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(tile_state, 0, tiles * sizeof(uint64_t), s);
  if (e != cudaSuccess) return e;
  k_scan_excl<<<(unsigned)tiles, kScanThreads, 0, s>>>(data, n_host, n_dev, n_add,
                                                       tile_state, tile_counter, ctr);
  return cudaGetLastError();
}

}  // namespace rtnn
