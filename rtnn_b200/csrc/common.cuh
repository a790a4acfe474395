// common.cuh -- shared device structs and helpers of the B200 neighbor-search engine.
//
// Layout in HBM (one pipeline = one set of clouds; a single cloud is a batch of one):
//   points (caller)    AoS float3, 12 B/point, read with 16-byte vector loads.
//   spts               float4 {x, y, z, original index bits}, 16 B/point, sorted by
//                      grid cell (raster order inside each cloud, clouds in order).
//   cells              uint32 per cell + 1: per-cell counts, scanned in place into
//                      cell start offsets (cells[total] == number of points).
//   sq                 float4 {x, y, z, original query index bits} in (cloud, density
//                      bucket, Hilbert index) order.
//   out (caller)       int32 [Q][K], -1 in unused slots.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rtnn {

constexpr int kChunk = 2048;        // points per block of the per-point kernels
constexpr int kTile = 32;           // queries per search work item (one warp)
constexpr int kScanItems = 16;      // items per thread of the scan
constexpr int kScanThreads = 256;
constexpr int kScanTile = kScanItems * kScanThreads;   // 4096
constexpr int kRadixThreads = 256;  // 8 warps
constexpr int kRadixItems = 8;      // per lane, per warp sub-tile of 256
constexpr int kRadixTile = kRadixThreads * kRadixItems; // 2048 keys per block
constexpr int kMaxK = 128;
constexpr int kMaxPasses = 8;       // main search pass + escalating fallback passes

// Device error codes (first one wins, written with atomicCAS into Counters::error).
enum DevError : uint32_t {
  kErrNone = 0,
  kErrScanTimeout = 1,     // decoupled look-back predecessor never published
  kErrCellCapacity = 2,    // grid plan needed more cells than were allocated
  kErrIndexRange = 3,      // a computed index fell outside its buffer (access skipped)
};

// Per-cloud uniform grid (written on the device by k_grid_plan).
struct __align__(16) CloudGrid {
  float ox, oy, oz;      // grid origin = min corner of the cloud's points
  float cell;            // cell edge
  float inv_cell;        // 1 / cell
  int dx, dy, dz;        // cells per axis
  uint32_t cell_base;    // first cell of this cloud in the global cell array
  float order_scale;    // query order: Hilbert index of floor((x - origin) * order_scale)
  uint32_t n_cells;      // dx * dy * dz
  uint32_t pad;
};

// Small counters zeroed at the start of every pipeline run.
struct Counters {
  uint32_t error;          // DevError
  uint32_t error_info;     // extra detail (e.g. scan tile that timed out)
  uint32_t work[kMaxPasses];      // persistent-kernel work queue of each search pass
  uint32_t fb_count[kMaxPasses];  // queries appended to the fallback list by each pass
  uint32_t total_cells;    // sum of cloud cells (written by k_grid_plan)
  uint32_t scan_tiles[24]; // dynamic tile counters, one per scan invocation
  uint32_t pad[3];
  unsigned long long n_loaded;   // candidate points streamed by the search (all passes)
  unsigned long long n_tested;   // candidates that passed the tile-box filter (x 32 lanes)
};

// Tables describing the clouds of one pipeline (all device arrays of n_clouds + 1).
struct CloudTables {
  const uint32_t* point_off;   // first point of cloud c; [n] = N
  const uint32_t* query_off;   // first query of cloud c; [n] = Q
  const uint32_t* chunk_base;  // first point chunk of cloud c; [n] = point chunks
  const uint32_t* qchunk_base; // first query chunk of cloud c; [n] = query chunks
  const uint32_t* tile_base;   // first 32-query tile of cloud c; [n] = tiles
  const uint32_t* lead_base;   // lead tiles before cloud c; [n] = all lead tiles (below)
  uint32_t n_clouds;
};

// The lead tiles of a cloud are the first eighth of its tiles (rounded up): the queries
// are sorted widest width bucket first, so they hold the cloud's widest searches -- the
// longest tiles by far (up to a few ms where a wide box reaches a dense blob). The first
// search pass takes the lead tiles of the clouds at the end of the pass (lead_base counts
// them; the host gives lead tiles to the clouds whose tiles start in the last eighth)
// before any other tile, so that no long tile starts near the end of the pass and holds it
// while the other SMs are idle.
constexpr uint32_t kLeadShift = 3;
__host__ __device__ __forceinline__ uint32_t lead_tiles(uint32_t tiles) {
  return (tiles + (1u << kLeadShift) - 1u) >> kLeadShift;
}

__device__ __forceinline__ void set_error(Counters* c, uint32_t code, uint32_t info) {
  if (atomicCAS(&c->error, 0u, code) == 0u) c->error_info = info;
}

// Largest c with base[c] <= x (base ascending, base[0] == 0, n_clouds + 1 entries).
__device__ __forceinline__ uint32_t find_cloud(const uint32_t* base, uint32_t n_clouds,
                                               uint32_t x) {
  uint32_t lo = 0, hi = n_clouds;  // invariant: base[lo] <= x < base[hi] (base[n] is total)
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (__ldg(base + mid) <= x) lo = mid; else hi = mid;
  }
  return lo;
}

// Work item w of the first search pass -> (cloud, tile j of that cloud): items
// [0, lead_base[n]) are the clouds' lead tiles in cloud order, the rest their other tiles
// in cloud order.
__device__ __forceinline__ void main_tile(const CloudTables& t, uint32_t w, uint32_t& cloud,
                                          uint32_t& j) {
  const uint32_t lead = __ldg(t.lead_base + t.n_clouds);
  if (w < lead) {
    cloud = find_cloud(t.lead_base, t.n_clouds, w);
    j = w - __ldg(t.lead_base + cloud);
    return;
  }
  // other tiles before cloud c: tile_base[c] - lead_base[c] (non-decreasing in c)
  const uint32_t r = w - lead;
  uint32_t lo = 0, hi = t.n_clouds;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(t.tile_base + mid) - __ldg(t.lead_base + mid) <= r) lo = mid; else hi = mid;
  }
  cloud = lo;
  const uint32_t lead_c = __ldg(t.lead_base + lo + 1) - __ldg(t.lead_base + lo);
  j = lead_c + (r - (__ldg(t.tile_base + lo) - __ldg(t.lead_base + lo)));
}

// Order-preserving map float -> uint32 (for atomicMin/Max on floats).
__device__ __forceinline__ uint32_t f2o(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ __forceinline__ float o2f(uint32_t o) {
#ifdef __CUDA_ARCH__
  return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
#else
  uint32_t b = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
  float f; __builtin_memcpy(&f, &b, 4); return f;
#endif
}

// Squared distance with the reference's operation order and rounding:
// dot(d, d) = d.x*d.x + d.y*d.y + d.z*d.z evaluated left to right, every product and
// sum rounded to FP32, no FMA (src/sutil/vec_math.h:527-530, check.cpp:36-37).
__device__ __forceinline__ float dist2_ref(float qx, float qy, float qz,
                                          float px, float py, float pz) {
  float dx = __fsub_rn(qx, px), dy = __fsub_rn(qy, py), dz = __fsub_rn(qz, pz);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// Cell coordinate of v along one axis: floor((v - o) * inv), clamped to [0, d-1].
// The same monotone expression bins points and bounds query ranges.
__device__ __forceinline__ float cell_coord_f(float v, float o, float inv) {
  return floorf(__fmul_rn(__fsub_rn(v, o), inv));
}
__device__ __forceinline__ int clamp_cell(float c, int d) {
  c = fminf(fmaxf(c, 0.f), (float)(d - 1));  // NaN -> 0 via fmaxf
  return (int)c;
}

// 21-bit-per-axis Morton interleave into 64 bits (bit i of x -> bit 3i, y -> 3i+1, z -> 3i+2,
// the reference's convention, helper_mortonCode.h:30-33).
__device__ __forceinline__ uint64_t spread3_64(uint64_t x) {
  x &= 0x1fffffull;
  x = (x | (x << 32)) & 0x001f00000000ffffull;
  x = (x | (x << 16)) & 0x001f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}
__device__ __forceinline__ uint64_t morton3_64(uint32_t x, uint32_t y, uint32_t z) {
  return spread3_64(x) | (spread3_64(y) << 1) | (spread3_64(z) << 2);
}

// Hilbert index of a cell (b bits per axis), after J. Skilling, "Programming the Hilbert
// curve" (AIP Conf. Proc. 707, 2004): the axes are turned into the curve's transposed
// form (undo the excess work: invert or exchange low bits, top bit down; then Gray-encode),
// and the transposed words interleave bit by bit, the first word most significant.
// Consecutive indices are face-adjacent cells, so a run of consecutive queries stays
// compact where the Morton order jumps.
// Every step is a select, not a branch (the lanes of a warp never diverge), and the final
// Gray-code correction t = XOR of (Q - 1) over the set bits Q > 1 of X2 is a prefix XOR
// of X2's bits taken from the top, shifted down by one. For x, y, z < 2^b this gives the
// same index as the step-by-step form of the published method (checked on 3.2 M inputs,
// b = 1..16).
__device__ __forceinline__ uint64_t hilbert3_64(uint32_t x, uint32_t y, uint32_t z, uint32_t b) {
  uint32_t X0 = x, X1 = y, X2 = z;
  for (int s = (int)b - 1; s > 0; --s) {
    const uint32_t Q = 1u << s, P = Q - 1;
    X0 ^= (X0 & Q) ? P : 0u;
    const uint32_t t1 = (X0 ^ X1) & P;
    const bool b1 = (X1 & Q) != 0;
    X0 ^= b1 ? P : t1;
    X1 ^= b1 ? 0u : t1;
    const uint32_t t2 = (X0 ^ X2) & P;
    const bool b2 = (X2 & Q) != 0;
    X0 ^= b2 ? P : t2;
    X2 ^= b2 ? 0u : t2;
  }
  X1 ^= X0;
  X2 ^= X1;
  uint32_t v = X2 & ~1u;
  v ^= v >> 1;
  v ^= v >> 2;
  v ^= v >> 4;
  v ^= v >> 8;
  v ^= v >> 16;
  const uint32_t t = v >> 1;
  return morton3_64(X2 ^ t, X1 ^ t, X0 ^ t);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m; asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m)); return m;
}

}  // namespace rtnn
