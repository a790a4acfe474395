// tile_model.cuh -- the learned search width of a bucket (one 32-query tile of the search).
//
// Replaces the reference's analytic partition widths (calcSearchSize / kGenCellMask,
// src/optixNSearch/grid.cu:84-211, 354-382; radiusFromMegacell, sort.cpp:262-269): there
// each occupied cell grows a box of cells until it holds K + 1 points and its queries are
// launched with the equal-volume radius of that box. Here the bucket is the tile of 32
// consecutive queries (Hilbert order) that one warp of the search handles, and a small MLP
// (6 -> 16 -> 16 -> 1, ReLU) reads the bucket's features
//   f0..f2  log1p of the points in cell shells 0, 1, 2 around the cell of the tile's
//           bounding-box centre (the occupancy histogram: N0, N1 - N0, N2 - N1),
//   f3      log(K + 1) - log1p(N2),
//   f4      log(cell / r),
//   f5      log1p(tile extent / cell) (the bucket's extent: longest side of its box),
// and predicts log(largest K-th neighbor distance of the tile's queries / cell). The tile
// is searched at margin * cell * exp(prediction), capped at r; its queries that find fewer
// than K neighbors there are searched again wider, so results never depend on the model.
//
// Both device functions are warp-collective (all 32 lanes, the same arguments) and return
// the same value in every lane: the search kernels call them once per tile, and the
// training-sample kernel (partition.cu) once per tile of a plain search.
#pragma once
#include "common.cuh"

namespace rtnn {

constexpr int kTileFeat = 6;       // MLP input features per tile
constexpr int kTileHidden = 16;    // hidden units: lanes j and j + 16 compute unit j
static_assert(32 % kTileHidden == 0 && kTileHidden % 4 == 0,
              "the warp-collective MLP spreads the hidden units over the lanes");

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ uint32_t warp_sum_u(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Features of the tile whose query bounding box is [b0, b1] (every lane the same box).
// The three box counts read the 25 cell rows of the 5 x 5 x 5 box around the box-centre
// cell, one row per lane (lanes 0..24): per row the offsets of the x ranges [cx-2, cx+2],
// [cx-1, cx+1] and [cx, cx] from the scanned cell offsets.
__device__ __forceinline__ void tile_features(const CloudGrid& g, const uint32_t* __restrict__ cells,
                                              float bx0, float bx1, float by0, float by1,
                                              float bz0, float bz1, uint32_t need, float radius,
                                              float* feat) {
  const int lane = threadIdx.x & 31;
  const int cx = clamp_cell(cell_coord_f(0.5f * (bx0 + bx1), g.ox, g.inv_cell), g.dx);
  const int cy = clamp_cell(cell_coord_f(0.5f * (by0 + by1), g.oy, g.inv_cell), g.dy);
  const int cz = clamp_cell(cell_coord_f(0.5f * (bz0 + bz1), g.oz, g.inv_cell), g.dz);
  uint32_t n0 = 0, n1 = 0, n2 = 0;
  if (lane < 25) {
    const int dy = lane % 5 - 2, dz = lane / 5 - 2;
    const int y = cy + dy, z = cz + dz;
    if (y >= 0 && y < g.dy && z >= 0 && z < g.dz) {
      const uint32_t* row =
          cells + g.cell_base + ((uint32_t)z * (uint32_t)g.dy + (uint32_t)y) * (uint32_t)g.dx;
      const int x0 = max(cx - 2, 0), x1 = min(cx + 2, g.dx - 1);
      n2 = __ldg(row + x1 + 1) - __ldg(row + x0);
      if (dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1) {
        const int i0 = max(cx - 1, 0), i1 = min(cx + 1, g.dx - 1);
        n1 = __ldg(row + i1 + 1) - __ldg(row + i0);
        if (dy == 0 && dz == 0) n0 = __ldg(row + cx + 1) - __ldg(row + cx);
      }
    }
  }
  n0 = warp_sum_u(n0);
  n1 = warp_sum_u(n1);
  n2 = warp_sum_u(n2);
  const float ext = fmaxf(fmaxf(bx1 - bx0, by1 - by0), bz1 - bz0) * g.inv_cell;
  feat[0] = log1pf((float)n0);
  feat[1] = log1pf((float)(n1 - n0));
  feat[2] = log1pf((float)(n2 - n1));
  feat[3] = logf((float)need) - log1pf((float)n2);
  feat[4] = logf(g.cell / radius);
  feat[5] = log1pf(fmaxf(ext, 0.f));
}

// The model's prediction (denormalised: log(K-th distance / cell)) for one feature vector.
// Parameter layout (floats): in_mean[6] in_std[6] out_mean out_std | W1[H][6] b1[H]
// W2[H][H] b2[H] W3[H] b3 (H = kTileHidden), P at least 8-byte aligned (a device allocation
// is). Lane j computes hidden unit j mod H of both layers (the lanes past H repeat the
// first H and add nothing to the output); the first layer's units reach every lane through
// `scratch` (32 floats of this warp's shared memory, 16-byte aligned), read back as H / 4
// broadcast 16-byte loads, and the second layer sums in four independent chains, so the
// evaluation is a few short dependency chains instead of H shuffles in a row; the output
// is a warp sum. (The sums run in another order than the inference kernel's: the two agree to
// FP32 rounding, which only moves a search width, never a result.)
__device__ __forceinline__ float tile_mlp(const float* __restrict__ P, const float* feat,
                                          float* scratch) {
  constexpr int F = kTileFeat, H = kTileHidden;
  const int lane = threadIdx.x & 31;
  const int j = lane & (H - 1);
  const float* W1 = P + 2 * F + 2;
  const float* b1 = W1 + H * F;
  const float* W2 = b1 + H;
  const float* b2 = W2 + H * H;
  const float* W3 = b2 + H;
  float xn[F];
#pragma unroll
  for (int f = 0; f < F; ++f) xn[f] = __fdividef(feat[f] - __ldg(P + f), __ldg(P + F + f));
  float h1 = __ldg(b1 + j);
#pragma unroll
  for (int f = 0; f < F; ++f) h1 = fmaf(__ldg(W1 + j * F + f), xn[f], h1);
  __syncwarp();
  if (lane < H) scratch[j] = fmaxf(h1, 0.f);
  __syncwarp();
  // W2 starts 2 F + 2 + H (F + 1) floats into P (126): 8-byte aligned (P itself is
  // 256-byte aligned), not 16
  const float2* w2 = reinterpret_cast<const float2*>(W2 + j * H);
  const float4* hv = reinterpret_cast<const float4*>(scratch);
  float acc[4] = {__ldg(b2 + j), 0.f, 0.f, 0.f};
#pragma unroll
  for (int i4 = 0; i4 < H / 4; ++i4) {
    const float4 h = hv[i4];
    const float2 wa = __ldg(w2 + 2 * i4), wb = __ldg(w2 + 2 * i4 + 1);
    acc[0] = fmaf(wa.x, h.x, acc[0]);
    acc[1] = fmaf(wa.y, h.y, acc[1]);
    acc[2] = fmaf(wb.x, h.z, acc[2]);
    acc[3] = fmaf(wb.y, h.w, acc[3]);
  }
  __syncwarp();
  const float h2 = fmaxf((acc[0] + acc[1]) + (acc[2] + acc[3]), 0.f);
  const float o = warp_sum_f(lane < H ? __ldg(W3 + j) * h2 : 0.f) + __ldg(W3 + H);
  return fmaf(o, __ldg(P + 2 * F + 1), __ldg(P + 2 * F));
}

// Search width of a tile from its features: margin * cell * exp(prediction), at most r.
// scratch: 32 floats of the warp's shared memory (16-byte aligned) for the MLP.
__device__ __forceinline__ float tile_width(const CloudGrid& g, const uint32_t* __restrict__ cells,
                                            const float* __restrict__ model, float margin,
                                            float bx0, float bx1, float by0, float by1, float bz0,
                                            float bz1, uint32_t need, float radius,
                                            float* scratch) {
  float feat[kTileFeat];
  tile_features(g, cells, bx0, bx1, by0, by1, bz0, bz1, need, radius, feat);
  const float y = tile_mlp(model, feat, scratch);
  const float w = margin * g.cell * __expf(fminf(y, 30.f));
  return w < radius ? w : radius;
}

}  // namespace rtnn
