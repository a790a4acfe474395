// partition.cu -- density buckets: search widths, analytic or learned, and the width model.
//
// Replaces the reference's query partitioning (src/optixNSearch/):
//   calcSearchSize / kGenCellMask (grid.cu:84-211, 354-382): per occupied cell, grow a
//     box of cells shell by shell until it holds K+1 points; iter -> width
//     (2*iter+2)*cellSize (getWidthFromIter, grid.cu:33-44);
//   sortGenBatch / genBatches / radiusFromMegacell (sort.cpp:262-269, 346-391, 393-498):
//     queries grouped by that width, each group launched with radius 0.62 * width
//     (approxMode 2, radiusEquiVolume, util.cpp:422-426).
// Analytic (k_widths): every query reads the box counts N_s (s = 0..2 cells around its
// cell) straight from the scanned cell offsets (one subtraction per row of cells) and gets
//   w = alpha * (s* + 1) * cell, s* = first s with N_s >= K + 1
// (alpha = 1.24 reproduces the reference's equal-volume radius); the width's level then
// joins the query sort key, so a tile shares one width band.
// Learned: the bucket is the search's 32-query tile, and the search kernel itself predicts
// its width from the tile's features (tile_model.cuh). This file holds the width model's
// training: one sample per tile of a plain search (k_tile_samples), and the hand-written
// loss/gradient, Adam and inference kernels of the MLP.
// A width >= r means "search at r". Exactness never depends on w: the search kernel
// re-searches wider every query that finds fewer than K neighbors inside w.
#include "common.cuh"
#include "kernels.h"
#include "tile_model.cuh"

namespace rtnn {
namespace {

// ---- MLP (6 -> 16 -> 16 -> 1, ReLU) ------------------------------------------------
static_assert(kFeatDim == kTileFeat && kHidden == kTileHidden,
              "the trained MLP is the one the search evaluates");

struct MlpView {
  const float* in_mean; const float* in_std; float out_mean, out_std;
  const float* W1; const float* b1; const float* W2; const float* b2; const float* W3; float b3;
};
__device__ __forceinline__ MlpView mlp_view(const float* P) {
  MlpView v;
  v.in_mean = P; v.in_std = P + kFeatDim;
  v.out_mean = P[2 * kFeatDim]; v.out_std = P[2 * kFeatDim + 1];
  const float* T = P + kNormParams;
  v.W1 = T; v.b1 = v.W1 + kHidden * kFeatDim;
  v.W2 = v.b1 + kHidden; v.b2 = v.W2 + kHidden * kHidden;
  v.W3 = v.b2 + kHidden; v.b3 = v.W3[kHidden];
  return v;
}

// ---- inference: normalised output o (before out_mean/out_std) of one sample. The second
// layer uses packed FP32x2 FMAs (sm_100a): two hidden units per instruction, each element
// rounded like fmaf, accumulated over the inputs in order, so the result is the bits of the
// plain one-unit-at-a-time loop. W2p holds W2 with the rows of units 2m and 2m + 1
// interleaved ({W2[2m][i], W2[2m+1][i]} at W2p[m * 2 * kHidden + 2 i]; 16-byte aligned),
// one 16-byte load per two inputs.
__device__ __forceinline__ uint64_t f2pack(float lo, float hi) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2unpack(uint64_t v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
static_assert(kHidden % 2 == 0, "hidden units are paired");

// Block-wide: the parameters into shared memory, plus W2 with unit pairs interleaved.
__device__ __forceinline__ void load_model_smem(const float* P, float* s_p, float* s_w2p) {
  for (int i = threadIdx.x; i < kModelParams; i += blockDim.x) s_p[i] = P[i];
  __syncthreads();
  const float* W2 = mlp_view(s_p).W2;
  for (int e = threadIdx.x; e < kHidden * kHidden; e += blockDim.x) {
    const int j = e / kHidden, i = e % kHidden;   // W2[j][i]
    s_w2p[(j >> 1) * 2 * kHidden + 2 * i + (j & 1)] = W2[e];
  }
  __syncthreads();
}

__device__ __forceinline__ float mlp_forward_norm_x2(const MlpView& m, const float* W2p,
                                                     const float* x) {
  float xn[kFeatDim];
#pragma unroll
  for (int f = 0; f < kFeatDim; ++f) xn[f] = (x[f] - m.in_mean[f]) / m.in_std[f];
  float h1[kHidden];
#pragma unroll
  for (int j = 0; j < kHidden; ++j) {
    float s = m.b1[j];
#pragma unroll
    for (int f = 0; f < kFeatDim; ++f) s = fmaf(m.W1[j * kFeatDim + f], xn[f], s);
    h1[j] = fmaxf(s, 0.f);
  }
  float o = m.b3;
#pragma unroll 1
  for (int j = 0; j < kHidden; j += 2) {
    uint64_t acc = f2pack(m.b2[j], m.b2[j + 1]);
    // two inputs per 16-byte load: {W2[j][i], W2[j+1][i], W2[j][i+1], W2[j+1][i+1]}
    const float4* w = reinterpret_cast<const float4*>(W2p + j * kHidden);
#pragma unroll
    for (int i = 0; i < kHidden; i += 2) {
      const float4 ww = w[i >> 1];
      acc = fma2(f2pack(ww.x, ww.y), f2pack(h1[i], h1[i]), acc);
      acc = fma2(f2pack(ww.z, ww.w), f2pack(h1[i + 1], h1[i + 1]), acc);
    }
    float s0, s1;
    f2unpack(acc, s0, s1);
    o = fmaf(m.W3[j], fmaxf(s0, 0.f), o);
    o = fmaf(m.W3[j + 1], fmaxf(s1, 0.f), o);
  }
  return o;
}

// The three box counts N_0..N_2 in one pass over the 25 rows of the 5 x 5 x 5 box: the six
// offsets a row needs (x - 2 .. x + 3) sit in one or two 32-byte sectors. The 25 rows are
// unrolled and every load is issued unconditionally (a row outside the grid reads the
// query's own row and counts nothing), so the ~70 loads of a query are in flight together
// instead of one row after another.
static_assert(kShells == 3, "box_counts3 counts three shells");
__device__ __forceinline__ void box_counts3(const CloudGrid& g, const uint32_t* cells, int cx,
                                            int cy, int cz, uint32_t* N) {
  const int x0 = max(cx - 2, 0), x1 = min(cx + 2, g.dx - 1);
  const int i0 = max(cx - 1, 0), i1 = min(cx + 1, g.dx - 1);
  const uint32_t* base = cells + g.cell_base;
  uint32_t n0 = 0, n1 = 0, n2 = 0;
#pragma unroll
  for (int dz = -2; dz <= 2; ++dz) {
#pragma unroll
    for (int dy = -2; dy <= 2; ++dy) {
      const int z = cz + dz, y = cy + dy;
      const bool in = z >= 0 && z < g.dz && y >= 0 && y < g.dy;
      const uint32_t* row =
          base + ((uint32_t)(in ? z : cz) * (uint32_t)g.dy + (uint32_t)(in ? y : cy)) * (uint32_t)g.dx;
      const uint32_t c2 = __ldg(row + x1 + 1) - __ldg(row + x0);
      n2 += in ? c2 : 0u;
      if (dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1) {
        const uint32_t c1 = __ldg(row + i1 + 1) - __ldg(row + i0);
        n1 += in ? c1 : 0u;
        if (dy == 0 && dz == 0) n0 += __ldg(row + cx + 1) - __ldg(row + cx);
      }
    }
  }
  N[0] = n0;
  N[1] = n1;
  N[2] = n2;
}

__device__ __forceinline__ float wmin_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float wmax_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// A width per query: the box counts around its cell, then the analytic rule or the
// per-query width model. Per-query model features:
//   f0..f2 log1p of the points in cell shells 0, 1, 2 around the query's cell,
//   f3     log(K + 1) - log1p(N2),
//   f4     log(cell / r),
//   f5     the query's distance from its cell's centre, in cells (at most 1).
__global__ void __launch_bounds__(256)
k_widths(WidthArgs a) {
  __shared__ float s_model[kModelParams];
  __shared__ __align__(16) float s_w2p[kHidden * kHidden];   // W2, unit pairs interleaved
  if (a.model) load_model_smem(a.model, s_model, s_w2p);
  const MlpView mv = mlp_view(s_model);
  const uint32_t total_cells = a.total_cells ? *a.total_cells : 0u;
  // queries that are the points are taken in cell order (neighbouring threads read the
  // same cell rows); only the points placed in cells are there, the rest keep no width
  // (that happens only when the grid plan failed, which the call reports as an error)
  const uint32_t n_items = a.spts ? min(a.n_queries, __ldg(a.cells + total_cells)) : a.n_queries;
  // each block walks one contiguous range of items, so a thread's items only move forward
  // through the clouds: the cloud of the block's first item is looked up once, and each
  // item then advances the thread's cloud while it lies past that cloud's end (the clouds
  // are contiguous both in query order and in the cell-sorted point order)
  const uint32_t* off = a.spts ? a.t.point_off : a.t.query_off;
  const uint32_t per_block = (n_items + gridDim.x - 1) / gridDim.x;
  const uint32_t b0 = min(n_items, blockIdx.x * per_block);
  const uint32_t b1 = min(n_items, b0 + per_block);
  __shared__ uint32_t s_cloud0;
  if (threadIdx.x == 0) s_cloud0 = b0 < b1 ? find_cloud(off, a.t.n_clouds, b0) : 0u;
  __syncthreads();
  uint32_t cloud = s_cloud0;
  for (uint32_t it = b0 + threadIdx.x; it < b1; it += blockDim.x) {
    while (cloud + 1 < a.t.n_clouds && it >= __ldg(off + cloud + 1)) ++cloud;
    uint32_t i = it;
    float qx, qy, qz;
    if (a.spts) {
      const float4 p = __ldg(a.spts + it);
      i = __float_as_uint(p.w);
      if (i >= a.n_queries) continue;
      qx = p.x; qy = p.y; qz = p.z;
    } else {
      qx = __ldg(a.xyz + 3ull * i); qy = __ldg(a.xyz + 3ull * i + 1); qz = __ldg(a.xyz + 3ull * i + 2);
    }
    const CloudGrid g = a.grids[cloud];
    if ((uint64_t)g.cell_base + g.n_cells > (uint64_t)total_cells) {  // overran: full radius
      a.qwidth[i] = a.radius;
      continue;
    }
    const int cx = clamp_cell(cell_coord_f(qx, g.ox, g.inv_cell), g.dx);
    const int cy = clamp_cell(cell_coord_f(qy, g.oy, g.inv_cell), g.dy);
    const int cz = clamp_cell(cell_coord_f(qz, g.oz, g.inv_cell), g.dz);
    uint32_t N[kShells];
    box_counts3(g, a.cells, cx, cy, cz, N);
    // offset of the query from its cell's centre, in cells (0 .. 0.87)
    const float ox = (qx - g.ox) * g.inv_cell - ((float)cx + 0.5f);
    const float oy = (qy - g.oy) * g.inv_cell - ((float)cy + 0.5f);
    const float oz = (qz - g.oz) * g.inv_cell - ((float)cz + 0.5f);
    float feat[kFeatDim];
    feat[0] = log1pf((float)N[0]);
    feat[1] = log1pf((float)(N[1] - N[0]));
    feat[2] = log1pf((float)(N[2] - N[1]));
    feat[3] = logf((float)a.need) - log1pf((float)N[2]);
    feat[4] = logf(g.cell / a.radius);
    feat[5] = fminf(sqrtf(ox * ox + oy * oy + oz * oz), 1.f);
    float w;
    if (a.model) {
      const float o = mlp_forward_norm_x2(mv, s_w2p, feat);
      const float y = fmaf(o, mv.out_std, mv.out_mean);
      w = a.margin * g.cell * expf(fminf(y, 30.f));
    } else {
      w = INFINITY;
#pragma unroll
      for (int s = 0; s < kShells; ++s)
        if (w == INFINITY && N[s] >= a.need) w = a.alpha * (float)(s + 1) * g.cell;
    }
    a.qwidth[i] = (w < a.radius) ? w : a.radius;
    if (a.feats) {
#pragma unroll
      for (int f = 0; f < kFeatDim; ++f) a.feats[(size_t)i * kFeatDim + f] = feat[f];
    }
    if (a.cellsz) a.cellsz[i] = g.cell;
  }
}

// One training sample per tile of a plain search: the tile's features (the same function
// the search evaluates) and log(largest K-th neighbor distance of its queries / cell);
// queries with fewer than K neighbors within r do not count (a tile made only of them
// gets log(1.5 r / cell), beyond the radius). One warp per tile.
__global__ void __launch_bounds__(256)
k_tile_samples(TileSampleArgs a) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t total_cells = *a.total_cells;
  for (uint32_t tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile < a.n_tiles;
       tile += warps) {
    uint32_t c = 0;
    if (lane == 0) c = find_cloud(a.t.tile_base, a.t.n_clouds, tile);
    const uint32_t cloud = __shfl_sync(0xffffffffu, c, 0);
    const uint32_t pos = a.t.query_off[cloud] + (tile - a.t.tile_base[cloud]) * 32u + lane;
    bool valid = pos < a.t.query_off[cloud + 1];
    const float4 q = valid ? a.sq[pos] : make_float4(0.f, 0.f, 0.f, 0.f);
    valid = valid && isfinite(q.x) && isfinite(q.y) && isfinite(q.z);
    const float kq = valid ? a.kth[__float_as_uint(q.w)] : -1.f;
    const float bx0 = wmin_f(valid ? q.x : INFINITY), bx1 = wmax_f(valid ? q.x : -INFINITY);
    const float by0 = wmin_f(valid ? q.y : INFINITY), by1 = wmax_f(valid ? q.y : -INFINITY);
    const float bz0 = wmin_f(valid ? q.z : INFINITY), bz1 = wmax_f(valid ? q.z : -INFINITY);
    const float kmax = wmax_f(kq);
    const CloudGrid g = a.grids[cloud];
    const bool ok = __any_sync(0xffffffffu, valid) &&
                    (uint64_t)g.cell_base + g.n_cells <= (uint64_t)total_cells;
    float feat[kTileFeat];
    if (ok) {
      tile_features(g, a.cells, bx0, bx1, by0, by1, bz0, bz1, a.need, a.radius, feat);
    } else {
#pragma unroll
      for (int f = 0; f < kTileFeat; ++f) feat[f] = 0.f;
    }
    const float d = kmax >= 0.f ? fmaxf(kmax, 1e-6f * a.radius) : 1.5f * a.radius;
    if (lane < kTileFeat) {
      float v = feat[0];
#pragma unroll
      for (int f = 1; f < kTileFeat; ++f) v = lane == f ? feat[f] : v;
      a.feats[(size_t)tile * kTileFeat + lane] = v;
    }
    if (lane == 0) a.target[tile] = logf(d / g.cell);
  }
}

// ---- training: loss and gradient of 0.5 * mean((o - t_n)^2) over a batch ---------
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(256)
k_mlp_loss_grad(const float* __restrict__ P, MlpBatch b, float* __restrict__ grad,
                float* __restrict__ loss_sum) {
  __shared__ float s_p[kModelParams];
  __shared__ float s_g[kTrainParams];
  for (int i = threadIdx.x; i < kModelParams; i += blockDim.x) s_p[i] = P[i];
  for (int i = threadIdx.x; i < kTrainParams; i += blockDim.x) s_g[i] = 0.f;
  __syncthreads();
  const MlpView m = mlp_view(s_p);
  const int lane = threadIdx.x & 31;
  float* gW1 = s_g;
  float* gb1 = gW1 + kHidden * kFeatDim;
  float* gW2 = gb1 + kHidden;
  float* gb2 = gW2 + kHidden * kHidden;
  float* gW3 = gb2 + kHidden;
  float* gb3 = gW3 + kHidden;
  float lsum = 0.f;
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t n_iter = (b.n + stride - 1) / stride;
  for (uint32_t it = 0; it < n_iter; ++it) {
    const uint32_t i = it * stride + blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < b.n;   // invalid lanes run with zero error (no contribution)
    float xn[kFeatDim];
#pragma unroll
    for (int f = 0; f < kFeatDim; ++f) {
      const float x = valid ? b.feats[(size_t)i * kFeatDim + f] : m.in_mean[f];
      xn[f] = (x - m.in_mean[f]) / m.in_std[f];
    }
    float h1[kHidden], h2[kHidden];
#pragma unroll
    for (int j = 0; j < kHidden; ++j) {
      float s = m.b1[j];
#pragma unroll
      for (int f = 0; f < kFeatDim; ++f) s = fmaf(m.W1[j * kFeatDim + f], xn[f], s);
      h1[j] = fmaxf(s, 0.f);
    }
    float o = m.b3;
#pragma unroll
    for (int j = 0; j < kHidden; ++j) {
      float s = m.b2[j];
#pragma unroll
      for (int k = 0; k < kHidden; ++k) s = fmaf(m.W2[j * kHidden + k], h1[k], s);
      h2[j] = fmaxf(s, 0.f);
      o = fmaf(m.W3[j], h2[j], o);
    }
    const float tn = valid ? (b.target[i] - m.out_mean) / m.out_std : o;
    const float err = o - tn;          // d(0.5 err^2)/do
    lsum += 0.5f * err * err;
    // output layer
    float g = warp_sum(err);
    if (lane == 0) atomicAdd(gb3, g);
    float dh2[kHidden];
#pragma unroll
    for (int j = 0; j < kHidden; ++j) {
      g = warp_sum(err * h2[j]);
      if (lane == 0) atomicAdd(&gW3[j], g);
      dh2[j] = (h2[j] > 0.f) ? err * m.W3[j] : 0.f;
    }
    // hidden layer 2
    float dh1[kHidden];
#pragma unroll
    for (int k = 0; k < kHidden; ++k) dh1[k] = 0.f;
#pragma unroll
    for (int j = 0; j < kHidden; ++j) {
      g = warp_sum(dh2[j]);
      if (lane == 0) atomicAdd(&gb2[j], g);
#pragma unroll
      for (int k = 0; k < kHidden; ++k) {
        g = warp_sum(dh2[j] * h1[k]);
        if (lane == 0) atomicAdd(&gW2[j * kHidden + k], g);
        dh1[k] = fmaf(dh2[j], m.W2[j * kHidden + k], dh1[k]);
      }
    }
    // hidden layer 1
#pragma unroll
    for (int k = 0; k < kHidden; ++k) {
      const float d = (h1[k] > 0.f) ? dh1[k] : 0.f;
      g = warp_sum(d);
      if (lane == 0) atomicAdd(&gb1[k], g);
#pragma unroll
      for (int f = 0; f < kFeatDim; ++f) {
        g = warp_sum(d * xn[f]);
        if (lane == 0) atomicAdd(&gW1[k * kFeatDim + f], g);
      }
    }
  }
  lsum = warp_sum(lsum);
  if (lane == 0) atomicAdd(loss_sum, lsum);
  __syncthreads();
  for (int i = threadIdx.x; i < kTrainParams; i += blockDim.x) atomicAdd(&grad[i], s_g[i]);
}

__global__ void k_mlp_adam(float* __restrict__ P, const float* __restrict__ grad,
                           float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                           float b2, float eps, uint32_t step, float scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kTrainParams) return;
  const float g = grad[i] * scale;
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi; v[i] = vi;
  const float mh = mi / (1.f - powf(b1, (float)step));
  const float vh = vi / (1.f - powf(b2, (float)step));
  P[kNormParams + i] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void __launch_bounds__(256)
k_mlp_forward(const float* __restrict__ P, const float* __restrict__ feats, uint32_t n,
              float* __restrict__ y) {
  __shared__ float s_p[kModelParams];
  __shared__ __align__(16) float s_w2p[kHidden * kHidden];
  load_model_smem(P, s_p, s_w2p);
  const MlpView m = mlp_view(s_p);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float x[kFeatDim];
#pragma unroll
    for (int f = 0; f < kFeatDim; ++f) x[f] = feats[(size_t)i * kFeatDim + f];
    y[i] = fmaf(mlp_forward_norm_x2(m, s_w2p, x), m.out_std, m.out_mean);
  }
}

// K-th neighbor distance of each query from rows sorted by (distance, index);
// -1 when the row has fewer than K neighbors.
__global__ void k_kth_dist(const int32_t* __restrict__ rows, uint32_t nq, uint32_t k,
                           const float* __restrict__ pts, const float* __restrict__ qs,
                           float* __restrict__ kth) {
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
    const int32_t p = rows[(size_t)q * k + (k - 1)];
    float d = -1.f;
    if (p >= 0) {
      const float* a = qs + 3ull * q;
      const float* b = pts + 3ull * (uint32_t)p;
      d = sqrtf(dist2_ref(a[0], a[1], a[2], b[0], b[1], b[2]));
    }
    kth[q] = d;
  }
}

}  // namespace

cudaError_t launch_widths(const WidthArgs& a, int n_sms, cudaStream_t s) {
  if (a.n_queries == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)min((uint64_t)n_sms * 8, ((uint64_t)a.n_queries + 255) / 256);
  k_widths<<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_tile_samples(const TileSampleArgs& a, int n_sms, cudaStream_t s) {
  if (a.n_tiles == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)min((uint64_t)n_sms * 8, ((uint64_t)a.n_tiles + 7) / 8);
  k_tile_samples<<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_mlp_loss_grad(const float* params, const MlpBatch& b, float* grad,
                                 float* loss_sum, int n_sms, cudaStream_t s) {
  if (b.n == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)min((uint64_t)n_sms * 2, ((uint64_t)b.n + 255) / 256);
  k_mlp_loss_grad<<<blocks, 256, 0, s>>>(params, b, grad, loss_sum);
  return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float* params, const float* grad, float* m, float* v, float lr,
                            float beta1, float beta2, float eps, uint32_t step, float scale,
                            cudaStream_t s) {
  k_mlp_adam<<<(kTrainParams + 255) / 256, 256, 0, s>>>(params, grad, m, v, lr, beta1, beta2,
                                                         eps, step, scale);
  return cudaGetLastError();
}

cudaError_t launch_mlp_forward(const float* params, const float* feats, uint32_t n, float* y,
                               int n_sms, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)min((uint64_t)n_sms * 8, ((uint64_t)n + 255) / 256);
  k_mlp_forward<<<blocks, 256, 0, s>>>(params, feats, n, y);
  return cudaGetLastError();
}

cudaError_t launch_kth_dist(const int32_t* rows, uint32_t n_queries, uint32_t k,
                            const float* points, const float* queries, float* kth_d,
                            cudaStream_t s) {
  if (n_queries == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)min(4096u, (n_queries + 255) / 256);
  k_kth_dist<<<blocks, 256, 0, s>>>(rows, n_queries, k, points, queries, kth_d);
  return cudaGetLastError();
}

}  // namespace rtnn
