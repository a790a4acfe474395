// build_grid.cu -- scene bounds, grid plan, per-cell counts, scatter, query keys.
//
// Reference steps replaced (src/optixNSearch/):
//   kComputeMinMax / computeMinMax (grid.cu:213-240, sort.cpp:34-71): scene bounds;
//     here a block reduce + one atomic per block, over each cloud's points.
//   genGridInfo (sort.cpp:73-136): cell size and dims; here on the device, per cloud,
//     with the cell edge grown when the grid would exceed its cell budget.
//   kInsertParticles_* (grid.cu:242-310): cell id + atomic per-cell count + rank.
//   kCountingSortIndices + sortByKey(pos, particles) (grid.cu:312-329, sort.cpp:612):
//     here a direct scatter into cell-sorted float4 {x, y, z, index} (no radix sort).
//   ToCellIndex_MortonMetaGrid / MortonCode3 (grid.cu:13-31, helper_mortonCode.h:19-33):
//     Hilbert-curve keys of queries (queries are then radix-sorted, radix_sort.cu).
#include "common.cuh"
#include "kernels.h"

namespace rtnn {
namespace {

// Loads the points [begin, end) of one chunk into shared memory with 16-byte vector loads
// (the AoS float3 input is read as float4 words; edge words fall back to scalars). Every
// thread issues all of its loads before it stores any of them (kChunkWords words per
// thread at most), so a block keeps its whole chunk in flight at once.
constexpr int kChunkThreads = 256;
constexpr int kChunkWords = (kChunk * 3 / 4 + 1 + kChunkThreads - 1) / kChunkThreads;   // 7
__device__ __forceinline__ void load_chunk_xyz(const float* __restrict__ xyz, uint32_t begin,
                                               uint32_t end, uint64_t total_floats,
                                               bool aligned, float* s_xyz) {
  const uint64_t f0 = (uint64_t)begin * 3, f1 = (uint64_t)end * 3;
  if (aligned) {
    const uint64_t a0 = f0 & ~3ull;            // first float4 word touching the chunk
    const uint64_t full_end = total_floats & ~3ull;  // words fully inside the array
    const uint64_t nw = (f1 - a0 + 3) >> 2;
    const float4* w4 = reinterpret_cast<const float4*>(xyz + a0);
    float4 v[kChunkWords];
#pragma unroll
    for (int u = 0; u < kChunkWords; ++u) {
      const uint64_t w = threadIdx.x + (uint64_t)u * kChunkThreads;
      const uint64_t f = a0 + 4 * w;
      v[u] = (w < nw && f + 4 <= full_end) ? __ldg(w4 + w) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < kChunkWords; ++u) {
      const uint64_t w = threadIdx.x + (uint64_t)u * kChunkThreads;
      if (w >= nw) continue;
      const uint64_t f = a0 + 4 * w;
      float vals[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
      if (f + 4 > full_end) {
#pragma unroll
        for (int i = 0; i < 4; ++i) vals[i] = (f + i < total_floats) ? __ldg(xyz + f + i) : 0.f;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const uint64_t fi = f + i;
        if (fi >= f0 && fi < f1) s_xyz[fi - f0] = vals[i];
      }
    }
  } else {
    for (uint64_t f = f0 + threadIdx.x; f < f1; f += blockDim.x) s_xyz[f - f0] = __ldg(xyz + f);
  }
  __syncthreads();
}

struct ChunkRange { uint32_t cloud, begin, end; };

__device__ __forceinline__ ChunkRange chunk_range(const uint32_t* chunk_base,
                                                  const uint32_t* off, uint32_t n_clouds,
                                                  uint32_t chunk) {
  __shared__ ChunkRange s_r;
  if (threadIdx.x == 0) {
    ChunkRange r;
    r.cloud = find_cloud(chunk_base, n_clouds, chunk);
    const uint32_t c0 = off[r.cloud], c1 = off[r.cloud + 1];
    r.begin = c0 + (chunk - chunk_base[r.cloud]) * (uint32_t)kChunk;
    r.end = min(r.begin + (uint32_t)kChunk, c1);
    s_r = r;
  }
  __syncthreads();
  return s_r;
}

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// bbox layout: [3 * n_clouds] ordered mins, then [3 * n_clouds] ordered maxs.
// Each block streams one contiguous range of point chunks straight from HBM: the AoS
// float3 input is read as 16-byte words (edge words of a chunk and an unaligned input fall
// back to scalars), and float f of a chunk starting at float f0 is component (f - f0) % 3 of
// its point, so each thread folds the four floats of a word into the components they
// belong to -- no staging through shared memory. Per-thread extrema are reduced over the
// block and merged with one atomic per component only when the range moves on to another
// cloud, and once at its end. Non-finite coordinates are skipped.
__device__ __forceinline__ void bbox_flush(float* mn, float* mx, float (*s_red)[8],
                                           uint32_t cloud, uint32_t n_clouds, uint32_t* bbox) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 3; ++a) { mn[a] = warp_min(mn[a]); mx[a] = warp_max(mx[a]); }
  if (lane == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) { s_red[a][warp] = mn[a]; s_red[3 + a][warp] = mx[a]; }
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    const int a = threadIdx.x;
    float v = s_red[a][0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      v = (a < 3) ? fminf(v, s_red[a][w]) : fmaxf(v, s_red[a][w]);
    if (isfinite(v)) {
      if (a < 3) atomicMin(&bbox[3 * cloud + a], f2o(v));
      else atomicMax(&bbox[3 * n_clouds + 3 * cloud + (a - 3)], f2o(v));
    }
  }
  __syncthreads();
#pragma unroll
  for (int a = 0; a < 3; ++a) { mn[a] = INFINITY; mx[a] = -INFINITY; }
}

__global__ void __launch_bounds__(256)
k_bbox(const float* __restrict__ xyz, uint64_t total_floats, bool aligned, CloudTables t,
       uint32_t n_chunks, uint32_t* __restrict__ bbox) {
  __shared__ float s_red[6][8];
  __shared__ uint32_t s_cloud;
  const uint32_t per = (n_chunks + gridDim.x - 1) / gridDim.x;
  const uint32_t c0 = min(n_chunks, blockIdx.x * per), c1 = min(n_chunks, c0 + per);
  if (c0 >= c1) return;
  if (threadIdx.x == 0) s_cloud = find_cloud(t.chunk_base, t.n_clouds, c0);
  __syncthreads();
  uint32_t cloud = s_cloud;
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t chunk = c0; chunk < c1; ++chunk) {
    while (chunk >= __ldg(t.chunk_base + cloud + 1)) {   // the range moved to the next cloud
      bbox_flush(mn, mx, s_red, cloud, t.n_clouds, bbox);
      ++cloud;
    }
    const uint32_t pb = __ldg(t.point_off + cloud), pe = __ldg(t.point_off + cloud + 1);
    const uint32_t begin = pb + (chunk - __ldg(t.chunk_base + cloud)) * (uint32_t)kChunk;
    const uint32_t end = min(begin + (uint32_t)kChunk, pe);
    const uint64_t f0 = (uint64_t)begin * 3, f1 = (uint64_t)end * 3;
    // float f >= f0 of the array is component (f - f0) % 3 (f0 is a point's first float)
    auto fold = [&](uint64_t f, float v) {
      const uint32_t c = (uint32_t)(f - f0) % 3u;
      const bool ok = isfinite(v);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        mn[a] = (ok && c == (uint32_t)a) ? fminf(mn[a], v) : mn[a];
        mx[a] = (ok && c == (uint32_t)a) ? fmaxf(mx[a], v) : mx[a];
      }
    };
    if (aligned) {
      const uint64_t a0 = f0 & ~3ull;                  // first 16-byte word touching the chunk
      const uint64_t full_end = total_floats & ~3ull;  // words wholly inside the array
      const uint64_t nw = (f1 - a0 + 3) >> 2;
      const float4* w4 = reinterpret_cast<const float4*>(xyz + a0);
      // four words per thread in flight: the loads of a round are issued before any fold
      for (uint64_t w0 = threadIdx.x; w0 < nw; w0 += 4ull * blockDim.x) {
        float4 v[4];
        bool whole[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const uint64_t w = w0 + (uint64_t)u * blockDim.x;
          const uint64_t f = a0 + 4 * w;
          whole[u] = w < nw && f >= f0 && f + 4 <= f1 && f + 4 <= full_end;
          v[u] = whole[u] ? __ldg(w4 + w) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const uint64_t w = w0 + (uint64_t)u * blockDim.x;
          if (w >= nw) continue;
          const uint64_t f = a0 + 4 * w;
          if (whole[u]) {
            fold(f, v[u].x); fold(f + 1, v[u].y); fold(f + 2, v[u].z); fold(f + 3, v[u].w);
          } else {
#pragma unroll
            for (int i = 0; i < 4; ++i)
              if (f + i >= f0 && f + i < f1) fold(f + i, __ldg(xyz + f + i));
          }
        }
      }
    } else {
      for (uint64_t f = f0 + threadIdx.x; f < f1; f += blockDim.x) fold(f, __ldg(xyz + f));
    }
  }
  bbox_flush(mn, mx, s_red, cloud, t.n_clouds, bbox);
}

// One block: per-cloud grid geometry and the global cell offsets (block-wide scan over
// clouds). Cell edge = radius * cell_ratio, grown by 1.25x until the cloud's grid fits
// its budget of max(64, cell_budget * points) cells.
__global__ void __launch_bounds__(1024)
k_grid_plan(CloudTables t, const uint32_t* __restrict__ bbox, float radius, float cell_ratio,
            float min_cell_ratio, float points_per_cell, float cell_budget,
            uint32_t order_bits, uint64_t cell_capacity, CloudGrid* __restrict__ grids,
            Counters* ctr) {
  __shared__ uint32_t s_sum[32];
  __shared__ uint64_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t n = t.n_clouds;
  for (uint32_t base = 0; base < n; base += blockDim.x) {
    const uint32_t c = base + threadIdx.x;
    uint32_t ncell = 0;
    CloudGrid g{};
    if (c < n) {
      const uint32_t np = t.point_off[c + 1] - t.point_off[c];
      float mn[3], mx[3];
      for (int a = 0; a < 3; ++a) {
        const uint32_t omn = bbox[3 * c + a], omx = bbox[3 * n + 3 * c + a];
        const bool valid = (omn != 0xffffffffu) && (omx != 0u);
        mn[a] = valid ? o2f(omn) : 0.f;
        mx[a] = valid ? o2f(omx) : 0.f;
        if (mx[a] < mn[a]) mx[a] = mn[a];
      }
      const double budget = fmin(fmax(64.0, (double)cell_budget * (double)np), 2147483647.0);
      float cell = radius * cell_ratio;
      if (points_per_cell > 0.f && np > 0) {
        // dense cloud: shrink the cell until its box holds ~points_per_cell per cell
        const float lo = radius * min_cell_ratio;
        double vol = 1.0;
        for (int a = 0; a < 3; ++a) vol *= fmax((double)(mx[a] - mn[a]), (double)lo);
        const float cd = (float)cbrt(vol * (double)points_per_cell / (double)np);
        cell = fminf(cell, fmaxf(cd, lo));
      }
      int d[3] = {1, 1, 1};
      bool fits = false;
      for (int it = 0; it < 64 && !fits; ++it) {
        const float inv = 1.0f / cell;
        double total = 1.0;
        for (int a = 0; a < 3; ++a) {
          // same expression as a point's cell: floor((max - min) * inv), then +1
          float f = floorf(__fmul_rn(__fsub_rn(mx[a], mn[a]), inv));
          f = fminf(fmaxf(f, 0.f), 2097151.f);
          d[a] = (int)f + 1;
          total *= (double)d[a];
        }
        fits = total <= budget;
        if (!fits) cell *= fmaxf(1.25f, (float)cbrt(total / budget));
      }
      if (!fits) {   // degenerate radius: one cell holding the whole cloud
        cell = fmaxf(fmaxf(mx[0] - mn[0], mx[1] - mn[1]), fmaxf(mx[2] - mn[2], 1e-30f)) * 2.f;
        d[0] = d[1] = d[2] = 1;
      }
      g.ox = mn[0]; g.oy = mn[1]; g.oz = mn[2];
      g.cell = cell; g.inv_cell = 1.0f / cell;
      g.dx = d[0]; g.dy = d[1]; g.dz = d[2];
      g.n_cells = (uint32_t)((uint64_t)d[0] * d[1] * d[2]);
      // query order: Hilbert index on 2^order_bits steps across the cloud's longest side
      // (finer than the cells, so dense cells still yield compact 32-query tiles)
      const float ext = fmaxf(fmaxf(mx[0] - mn[0], mx[1] - mn[1]), fmaxf(mx[2] - mn[2], 1e-30f));
      g.order_scale = (float)((1u << order_bits) - 1u) / ext;
      ncell = g.n_cells;
    }
    // block-wide exclusive scan of ncell (values < 2^32, carry kept in 64 bits)
    uint32_t v = ncell;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t x = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += x;
    }
    if (lane == 31) s_sum[warp] = v;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = (lane < (int)(blockDim.x >> 5)) ? s_sum[lane] : 0u;
      uint32_t wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t x = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += x;
      }
      s_sum[lane] = wi - w;
    }
    __syncthreads();
    const uint64_t excl = s_carry + s_sum[warp] + (v - ncell);
    if (c < n) {
      g.cell_base = (uint32_t)excl;
      grids[c] = g;
      if (excl + ncell > cell_capacity) set_error(ctr, kErrCellCapacity, c);
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_carry = excl + ncell;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const uint64_t tot = s_carry;
    ctr->total_cells = (uint32_t)(tot <= cell_capacity ? tot : cell_capacity);
  }
}

// Zeroes the total_cells + 1 counters with 16-byte stores (cells is 16-byte aligned).
__global__ void k_zero_cells(uint32_t* __restrict__ cells, const Counters* ctr) {
  const uint64_t n = (uint64_t)ctr->total_cells + 1;
  const uint64_t n4 = n >> 2;
  uint4* c4 = reinterpret_cast<uint4*>(cells);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t i = tid; i < n4; i += stride) c4[i] = make_uint4(0u, 0u, 0u, 0u);
  if (tid < (n & 3)) cells[4 * n4 + tid] = 0u;
}

__device__ __forceinline__ uint32_t point_cell(const CloudGrid& g, float x, float y, float z) {
  const int cx = clamp_cell(cell_coord_f(x, g.ox, g.inv_cell), g.dx);
  const int cy = clamp_cell(cell_coord_f(y, g.oy, g.inv_cell), g.dy);
  const int cz = clamp_cell(cell_coord_f(z, g.oz, g.inv_cell), g.dz);
  return g.cell_base + ((uint32_t)cz * (uint32_t)g.dy + (uint32_t)cy) * (uint32_t)g.dx +
         (uint32_t)cx;
}

// Per point: global cell id, rank within the cell from the atomic count. Each thread takes
// kChunk / 256 points of the staged chunk: all cells first, then all atomics (independent,
// in flight together), then the ranks (coalesced).
constexpr int kPerThread = kChunk / kChunkThreads;   // 8
__global__ void __launch_bounds__(kChunkThreads)
k_count(const float* __restrict__ xyz, uint64_t total_floats, bool aligned, CloudTables t,
        const CloudGrid* __restrict__ grids, uint32_t* __restrict__ cells,
        uint32_t* __restrict__ rank, Counters* ctr) {
  __shared__ float s_xyz[kChunk * 3];
  const ChunkRange r = chunk_range(t.chunk_base, t.point_off, t.n_clouds, blockIdx.x);
  load_chunk_xyz(xyz, r.begin, r.end, total_floats, aligned, s_xyz);
  const CloudGrid g = grids[r.cloud];
  const uint32_t lim = min(g.cell_base + g.n_cells, ctr->total_cells);
  const uint32_t n = r.end - r.begin;
  uint32_t cell[kPerThread];
#pragma unroll
  for (int u = 0; u < kPerThread; ++u) {
    const uint32_t i = threadIdx.x + u * kChunkThreads;
    cell[u] = i < n ? point_cell(g, s_xyz[3 * i], s_xyz[3 * i + 1], s_xyz[3 * i + 2]) : lim;
    if (i < n && cell[u] >= lim) set_error(ctr, kErrIndexRange, r.begin + i);
  }
  uint32_t rk[kPerThread];
#pragma unroll
  for (int u = 0; u < kPerThread; ++u) rk[u] = cell[u] < lim ? atomicAdd(&cells[cell[u]], 1u) : 0u;
#pragma unroll
  for (int u = 0; u < kPerThread; ++u) {
    const uint32_t i = threadIdx.x + u * kChunkThreads;
    if (cell[u] < lim) rank[r.begin + i] = rk[u];
  }
}

// Scatter into cell-sorted float4 {x, y, z, original index}. sorted_pos (optional): the
// inverse map, sorted_pos[original index] = position in spts. Per thread as in k_count:
// every cell offset and rank is loaded before any point is written.
__global__ void __launch_bounds__(kChunkThreads)
k_scatter(const float* __restrict__ xyz, uint64_t total_floats, bool aligned, CloudTables t,
          const CloudGrid* __restrict__ grids, const uint32_t* __restrict__ cells,
          const uint32_t* __restrict__ rank, float4* __restrict__ spts, uint32_t n_points,
          uint32_t* __restrict__ sorted_pos, Counters* ctr) {
  __shared__ float s_xyz[kChunk * 3];
  const ChunkRange r = chunk_range(t.chunk_base, t.point_off, t.n_clouds, blockIdx.x);
  load_chunk_xyz(xyz, r.begin, r.end, total_floats, aligned, s_xyz);
  const CloudGrid g = grids[r.cloud];
  const uint32_t lim = min(g.cell_base + g.n_cells, ctr->total_cells);
  const uint32_t n = r.end - r.begin;
  uint32_t pos[kPerThread];
#pragma unroll
  for (int u = 0; u < kPerThread; ++u) {
    const uint32_t i = threadIdx.x + u * kChunkThreads;
    const uint32_t cell = i < n ? point_cell(g, s_xyz[3 * i], s_xyz[3 * i + 1], s_xyz[3 * i + 2]) : lim;
    // a point outside its grid was already reported by k_count; both loads stay in bounds
    // whatever the point (cells holds total_cells + 1 entries, i is clamped to the chunk)
    const uint32_t off = __ldg(cells + min(cell, lim));
    const uint32_t rk = __ldg(rank + r.begin + min(i, n - 1));
    pos[u] = cell < lim ? off + rk : 0xffffffffu;
  }
#pragma unroll
  for (int u = 0; u < kPerThread; ++u) {
    const uint32_t i = threadIdx.x + u * kChunkThreads;
    if (i >= n || pos[u] == 0xffffffffu) continue;
    if (pos[u] >= n_points) { set_error(ctr, kErrIndexRange, r.begin + i); continue; }
    spts[pos[u]] = make_float4(s_xyz[3 * i], s_xyz[3 * i + 1], s_xyz[3 * i + 2],
                               __uint_as_float(r.begin + i));
    if (sorted_pos) sorted_pos[r.begin + i] = pos[u];
  }
}

// Density bucket of a width: 0 for the full radius, then `per_halving` buckets for each
// halving of the width (0: one bucket for every narrowed width).
__device__ __forceinline__ uint32_t width_level(float w, float radius, uint32_t level_bits,
                                                float per_halving) {
  if (!(w < radius)) return 0u;
  const uint32_t top = (1u << level_bits) - 1u;
  const float l = ceilf(-per_halving * log2f(fmaxf(w, 1e-30f) / radius));
  return (uint32_t)fminf(fmaxf(l, 1.f), (float)top);
}

// Sort key per query: cloud | density bucket of its width | Hilbert index of its cell.
template <typename KeyT>
__global__ void __launch_bounds__(256)
k_query_keys(const float* __restrict__ xyz, uint64_t total_floats, bool aligned,
             CloudTables t, const CloudGrid* __restrict__ grids, uint32_t order_bits,
             const float* __restrict__ qwidth, float radius, uint32_t level_bits,
             float per_halving, KeyT* __restrict__ keys) {
  __shared__ float s_xyz[kChunk * 3];
  const ChunkRange r = chunk_range(t.qchunk_base, t.query_off, t.n_clouds, blockIdx.x);
  load_chunk_xyz(xyz, r.begin, r.end, total_floats, aligned, s_xyz);
  const CloudGrid g = grids[r.cloud];
  const int top = (int)((1u << order_bits) - 1u);
  for (uint32_t i = threadIdx.x; i < r.end - r.begin; i += blockDim.x) {
    const int fx = clamp_cell(cell_coord_f(s_xyz[3 * i], g.ox, g.order_scale), top + 1);
    const int fy = clamp_cell(cell_coord_f(s_xyz[3 * i + 1], g.oy, g.order_scale), top + 1);
    const int fz = clamp_cell(cell_coord_f(s_xyz[3 * i + 2], g.oz, g.order_scale), top + 1);
    const uint64_t m = hilbert3_64((uint32_t)fx, (uint32_t)fy, (uint32_t)fz, order_bits);
    const uint32_t lvl = qwidth ? width_level(qwidth[r.begin + i], radius, level_bits, per_halving) : 0u;
    keys[r.begin + i] = ((KeyT)r.cloud << (3 * order_bits + level_bits)) |
                        ((KeyT)lvl << (3 * order_bits)) | (KeyT)m;
  }
}

// Sorted queries as float4 {x, y, z, original query index} (+ their widths). Each thread
// takes kGather queries a round: their order entries, then all gathers, then the stores.
constexpr int kGather = 4;
__global__ void __launch_bounds__(256)
k_gather_queries(const float* __restrict__ xyz, const uint32_t* __restrict__ order, uint32_t n,
                 float4* __restrict__ sq, const float* __restrict__ w_in, float* __restrict__ w_out) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x + threadIdx.x; base < n; base += kGather * stride) {
    uint32_t q[kGather];
#pragma unroll
    for (int u = 0; u < kGather; ++u) {
      const uint32_t i = base + u * stride;
      q[u] = i < n ? __ldg(order + i) : 0u;
    }
    float4 v[kGather];
#pragma unroll
    for (int u = 0; u < kGather; ++u) {
      const float* p = xyz + 3ull * q[u];   // q[u] == 0 past the end: an in-bounds address
      v[u] = make_float4(__ldg(p), __ldg(p + 1), __ldg(p + 2), __uint_as_float(q[u]));
    }
#pragma unroll
    for (int u = 0; u < kGather; ++u) {
      const uint32_t i = base + u * stride;
      if (i < n) sq[i] = v[u];
    }
    if (w_in) {
#pragma unroll
      for (int u = 0; u < kGather; ++u) {
        const uint32_t i = base + u * stride;
        if (i < n) w_out[i] = w_in[q[u]];
      }
    }
  }
}

// Tables of a single cloud written on the device (no host copy per call).
__global__ void k_single_tables(uint32_t* tab, uint32_t n_points, uint32_t n_queries) {
  // tab layout: point_off[2] query_off[2] chunk_base[2] qchunk_base[2] tile_base[2]
  // lead_base[2]
  tab[0] = 0; tab[1] = n_points;
  tab[2] = 0; tab[3] = n_queries;
  tab[4] = 0; tab[5] = (n_points + kChunk - 1) / kChunk;
  tab[6] = 0; tab[7] = (n_queries + kChunk - 1) / kChunk;
  tab[8] = 0; tab[9] = (n_queries + kTile - 1) / kTile;
  tab[10] = 0; tab[11] = lead_tiles(tab[9]);
}

}  // namespace

cudaError_t launch_single_tables(uint32_t* tab, uint32_t n_points, uint32_t n_queries,
                                 cudaStream_t s) {
  k_single_tables<<<1, 1, 0, s>>>(tab, n_points, n_queries);
  return cudaGetLastError();
}

cudaError_t launch_bbox(const float* xyz, uint64_t n_points, bool aligned, const CloudTables& t,
                        uint32_t n_chunks, uint32_t* bbox, int n_sms, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(bbox, 0xff, 3ull * t.n_clouds * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(bbox + 3ull * t.n_clouds, 0, 3ull * t.n_clouds * 4, s);
  if (e != cudaSuccess) return e;
  if (n_chunks == 0) return cudaSuccess;
  // eight blocks per SM, each streaming a contiguous range of chunks (measured faster than
  // one wave of resident blocks: 257 against 270 us for 54.8 M points)
  const unsigned blocks = (unsigned)min((uint64_t)n_chunks, (uint64_t)n_sms * 8);
  k_bbox<<<blocks, 256, 0, s>>>(xyz, 3 * n_points, aligned, t, n_chunks, bbox);
  return cudaGetLastError();
}

cudaError_t launch_grid_plan(const CloudTables& t, const uint32_t* bbox, float radius,
                             float cell_ratio, float min_cell_ratio, float points_per_cell,
                             float cell_budget, uint32_t order_bits, uint64_t cell_capacity,
                             CloudGrid* grids, Counters* ctr, cudaStream_t s) {
  k_grid_plan<<<1, 1024, 0, s>>>(t, bbox, radius, cell_ratio, min_cell_ratio, points_per_cell,
                                 cell_budget, order_bits, cell_capacity, grids, ctr);
  return cudaGetLastError();
}

cudaError_t launch_zero_cells(uint32_t* cells, const Counters* ctr, int n_sms, cudaStream_t s) {
  k_zero_cells<<<n_sms * 8, 256, 0, s>>>(cells, ctr);
  return cudaGetLastError();
}

cudaError_t launch_count(const float* xyz, uint64_t n_points, bool aligned, const CloudTables& t,
                         uint32_t n_chunks, const CloudGrid* grids, uint32_t* cells,
                         uint32_t* rank, Counters* ctr, cudaStream_t s) {
  if (n_chunks == 0) return cudaSuccess;
  k_count<<<n_chunks, 256, 0, s>>>(xyz, 3 * n_points, aligned, t, grids, cells, rank, ctr);
  return cudaGetLastError();
}

cudaError_t launch_scatter(const float* xyz, uint64_t n_points, bool aligned,
                           const CloudTables& t, uint32_t n_chunks, const CloudGrid* grids,
                           const uint32_t* cells, const uint32_t* rank, float4* spts,
                           Counters* ctr, cudaStream_t s, uint32_t* sorted_pos) {
  if (n_chunks == 0) return cudaSuccess;
  k_scatter<<<n_chunks, 256, 0, s>>>(xyz, 3 * n_points, aligned, t, grids, cells, rank, spts,
                                     (uint32_t)n_points, sorted_pos, ctr);
  return cudaGetLastError();
}

cudaError_t launch_query_keys(const float* xyz, uint64_t n_queries, bool aligned,
                              const CloudTables& t, uint32_t n_qchunks, const CloudGrid* grids,
                              uint32_t order_bits, const float* qwidth, float radius,
                              uint32_t level_bits, float per_halving, bool key64, void* keys,
                              cudaStream_t s) {
  if (n_qchunks == 0) return cudaSuccess;
  if (key64)
    k_query_keys<uint64_t><<<n_qchunks, 256, 0, s>>>(xyz, 3 * n_queries, aligned, t, grids,
                                                     order_bits, qwidth, radius, level_bits,
                                                     per_halving, (uint64_t*)keys);
  else
    k_query_keys<uint32_t><<<n_qchunks, 256, 0, s>>>(xyz, 3 * n_queries, aligned, t, grids,
                                                     order_bits, qwidth, radius, level_bits,
                                                     per_halving, (uint32_t*)keys);
  return cudaGetLastError();
}

cudaError_t launch_gather_queries(const float* xyz, const uint32_t* order, uint32_t n,
                                  float4* sq, const float* w_in, float* w_out, int n_sms,
                                  cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  unsigned blocks = (unsigned)min((uint64_t)n_sms * 16, ((uint64_t)n + 255) / 256);
  k_gather_queries<<<blocks, 256, 0, s>>>(xyz, order, n, sq, w_in, w_out);
  return cudaGetLastError();
}

}  // namespace rtnn
