// search.cu -- warp-cooperative cell-walk search (fixed-radius and KNN).
//
// Replaces the OptiX traversal of the reference: __raygen__radius / __raygen__knn
// (camera.cu:39-146) launching one zero-length ray per query, and the intersection
// programs __intersection__sphere_radius / __intersection__sphere_knn with
// check_intersect, write_res_radius and insertTopKQ (geometry.cu:38-191).
//
// Work item = a tile of 32 Hilbert-ordered queries of one cloud, handled by one warp;
// a persistent grid pulls tiles from an atomic counter. Per tile:
//   1. the warp reduces the tile's bounding box and widest search width R (per run of
//      nearby queries, see below);
//   2. the candidate cells are the grid box covering bbox +- R; in raster order each
//      (y, z) row of that box is one contiguous range of the cell-sorted points, so a
//      row costs two offset loads (computed lane-parallel, 32 rows at a time); rows, and
//      the ends of rows, farther than R from the bbox are skipped (RowClip);
//   3. 32 rows at a time are streamed as one flattened candidate sequence with 16-byte
//      loads issued one batch of 32 ahead (rows in a stride-permuted order), the points
//      farther than R from the tile box are dropped, and the survivors are compacted with
//      __ballot_sync into a per-warp shared-memory stage;
//   4. every lane tests every staged point against its own query with the reference's
//      FP32 distance (common.cuh: dist2_ref) and keeps its K smallest (distance, index)
//      pairs in a per-lane column in shared memory ([slot][lane], conflict-free): hits are
//      appended branch-free and merged into a max-heap of the K kept when a column fills;
//   5. rows are written warp-cooperatively (coalesced), unused slots = -1.
// Queries whose search width was narrowed by the partition (width < r) and that found
// fewer than K neighbors inside it are flagged; the host pipeline compacts them into a
// list that the next pass (this kernel or k_search_q below) searches at a wider width,
// and the last pass at the full radius, so every row is exact.
#include "common.cuh"
#include "kernels.h"
#include "packed.cuh"
#include "tile_model.cuh"

namespace rtnn {
namespace {

__device__ __forceinline__ void heap_sift_down(uint64_t* h, uint32_t i, uint32_t k, uint64_t x) {
  while (true) {
    uint32_t c = 2 * i + 1;
    if (c >= k) break;
    uint64_t cv = h[c * 32];
    if (c + 1 < k) {
      const uint64_t c2 = h[(c + 1) * 32];
      if (c2 > cv) { cv = c2; ++c; }
    }
    if (cv <= x) break;
    h[i * 32] = cv;
    i = c;
  }
  h[i * 32] = x;
}

// Depth of a K-entry heap below its root: floor(log2(K)).
__host__ __device__ constexpr int heap_depth(int k) { return k <= 1 ? 0 : 1 + heap_depth(k / 2); }

// heap_sift_down for a compile-time K, starting at node I: a fixed number of levels, every
// step predicated instead of branched, so that the 32 lanes of a warp (each sifting its
// own heap) stay on one path. A level whose nodes all have two children skips the bound
// checks (decided at compile time, the level being a constant of the unrolled loop).
template <int K, int I>
__device__ __forceinline__ void heap_sift_fixed(uint64_t* h, uint64_t x) {
  constexpr int kLevels = heap_depth(K) - heap_depth(I + 1);
  uint32_t i = I;
  bool go = true;
#pragma unroll
  for (int l = 0; l < kLevels; ++l) {
    // nodes of this level: [(I + 1) * 2^l - 1, (I + 2) * 2^l - 2]
    const int last = (I + 2) * (1 << l) - 2;
    const bool all_two = 2 * last + 2 < K;   // constant per unrolled level
    const uint32_t c = 2 * i + 1;
    const bool has1 = all_two || c < (uint32_t)K;
    const bool has2 = all_two || c + 1 < (uint32_t)K;
    uint64_t cv = has1 ? h[c * 32] : 0ull;
    const uint64_t c2 = has2 ? h[(c + 1) * 32] : 0ull;
    const bool right = c2 > cv;
    cv = right ? c2 : cv;
    const bool move = go && has1 && cv > x;
    if (move) h[i * 32] = cv;
    go = move;
    i = move ? c + (right ? 1u : 0u) : i;
  }
  h[i * 32] = x;
}

template <int K, int I = K / 2 - 1>
__device__ __forceinline__ void heapify_fixed(uint64_t* h) {
  if constexpr (I >= 0) {
    heap_sift_fixed<K, I>(h, h[I * 32]);
    heapify_fixed<K, I - 1>(h);
  }
}

// Staged candidates are kept in pairs, {x0 x1 y0 y1 | z0 z1 w0 w1} (32 bytes per two
// slots), so two 16-byte loads give two candidates already packed for the f32x2 math.
__device__ __forceinline__ void stage_put(float* st, uint32_t slot, float4 p) {
  float* b = st + (slot >> 1) * 8 + (slot & 1);
  b[0] = p.x; b[2] = p.y; b[4] = p.z; b[6] = p.w;
}
__device__ __forceinline__ float4 stage_get(const float* st, uint32_t slot) {
  const float* b = st + (slot >> 1) * 8 + (slot & 1);
  return make_float4(b[0], b[2], b[4], b[6]);
}

// Splits a row number rq of a box nx rows wide into (rq % n, rq / n) for an n fixed over a
// walk: a float estimate of the quotient corrected by one step, exact while rq / n < 2^22
// (rows of a box; `exact` false only for boxes of more than 2^22 rows, which divide).
struct RowSplit {
  uint32_t n;
  float inv;
  bool exact;
  __device__ __forceinline__ RowSplit(uint32_t n_, uint32_t total) : n(n_), inv(1.0f / (float)n_),
                                                                     exact(total < (1u << 22)) {}
  __device__ __forceinline__ void split(uint32_t rq, uint32_t& rem, uint32_t& quo) const {
    if (!exact) { quo = rq / n; rem = rq - quo * n; return; }
    uint32_t q = __float2uint_rz((float)rq * inv);
    int r = (int)rq - (int)(q * n);
    if (r < 0) { --q; r += (int)n; } else if (r >= (int)n) { ++q; r -= (int)n; }
    quo = q;
    rem = (uint32_t)r;
  }
};

constexpr int kCheck = 4;          // candidates tested between two buffer-full votes
constexpr uint32_t kFixedPending = 16;   // appended-hit slots of the compiled-K searches
constexpr uint32_t kQueryCap = 128;   // k_search_q hit buffer per warp (k <= 64)
constexpr int kStage = 64;         // staged candidates per warp (float4)
constexpr int kLaneRows = 8;       // lane walk: cell rows whose offsets are loaded together
constexpr uint64_t kRowStride = 4294967311ull;   // prime > 2^32 > any row count of a box

// Cell rows of a candidate box clipped to the points within R of the query box, in cell
// units: c(v) = (v - origin) * inv_cell with the rounding that bins the points, so a point
// of cell i has i <= c(p) < i + 1 along each axis. [X0, X1] x [Y0, Y1] x [Z0, Z1] is the
// query box (one point for a single query) in those units. A point within R of a query
// of the box lies in a row (cy, cz) whose cell square is within Rc = R * inv_cell of the
// box's (y, z) rectangle, and inside that row in the cells floor(X0 - e) .. floor(X1 + e)
// with e = sqrt(Rc^2 - gap_y^2 - gap_z^2). Every extent is widened by s, which exceeds the
// FP32 rounding of the map (a few ulps of the largest coordinate) and of this arithmetic,
// so a row or cell is only ever dropped when none of its points can be a hit. Past 2^23
// cells (coordinates without a fraction left, or a width far beyond any grid, where the
// squares could overflow) the clip is off: coordinates 0, s = inf and Rs2 = 1 make every
// gap 0 and e infinite, and the saturating float-to-int conversion then gives the whole
// row [lx, hx] of the box.
constexpr float kClipLimit = 8388608.f;
struct RowClip {
  float X0, X1, Y0, Y1, Z0, Z1, Rs2, s;
  __device__ __forceinline__ RowClip(const CloudGrid& g, float bx0, float bx1, float by0,
                                     float by1, float bz0, float bz1, float R) {
    X0 = __fmul_rn(__fsub_rn(bx0, g.ox), g.inv_cell);
    X1 = __fmul_rn(__fsub_rn(bx1, g.ox), g.inv_cell);
    Y0 = __fmul_rn(__fsub_rn(by0, g.oy), g.inv_cell);
    Y1 = __fmul_rn(__fsub_rn(by1, g.oy), g.inv_cell);
    Z0 = __fmul_rn(__fsub_rn(bz0, g.oz), g.inv_cell);
    Z1 = __fmul_rn(__fsub_rn(bz1, g.oz), g.inv_cell);
    const float Rc = __fmul_ru(R, g.inv_cell);
    const float M = fmaxf(fmaxf(fmaxf(fabsf(X0), fabsf(X1)), fmaxf(fabsf(Y0), fabsf(Y1))),
                          fmaxf(fabsf(Z0), fabsf(Z1)));
    s = 0.01f + 1e-6f * (M + Rc);
    const float Rs = __fadd_ru(Rc, s);
    Rs2 = __fmul_ru(Rs, Rs);
    if (!(M + Rc < kClipLimit)) {
      X0 = X1 = Y0 = Y1 = Z0 = Z1 = 0.f;
      s = INFINITY;
      Rs2 = 1.f;
    }
  }
  // The cells [xl, xh] of row (cy, cz) within the box's x range [lx, hx]; false: none.
  __device__ __forceinline__ bool row(int cy, int cz, int lx, int hx, int& xl, int& xh) const {
    const float fy = (float)cy, fz = (float)cz;
    const float gy = fmaxf(fmaxf(Y0 - (fy + 1.f + s), (fy - s) - Y1), 0.f);
    const float gz = fmaxf(fmaxf(Z0 - (fz + 1.f + s), (fz - s) - Z1), 0.f);
    const float rem = Rs2 - (gy * gy + gz * gz);
    if (!(rem >= 0.f)) return false;
    const float r2 = fmaxf(rem, 1e-20f);
    const float e = r2 * rsqrtf(r2) + s;   // sqrt within a few ulps, far inside s
    xl = max(__float2int_rd(X0 - e), lx);
    xh = min(__float2int_rd(X1 + e), hx);
    return xl <= xh;
  }
};

// RowClip of a single query (a box of one point): three coordinates instead of six, so
// the per-query walk keeps its registers.
struct RowClipPoint {
  float X, Y, Z, Rs2, s;
  __device__ __forceinline__ RowClipPoint(const CloudGrid& g, float qx, float qy, float qz,
                                          float R) {
    X = __fmul_rn(__fsub_rn(qx, g.ox), g.inv_cell);
    Y = __fmul_rn(__fsub_rn(qy, g.oy), g.inv_cell);
    Z = __fmul_rn(__fsub_rn(qz, g.oz), g.inv_cell);
    const float Rc = __fmul_ru(R, g.inv_cell);
    const float M = fmaxf(fmaxf(fabsf(X), fabsf(Y)), fabsf(Z));
    s = 0.01f + 1e-6f * (M + Rc);
    const float Rs = __fadd_ru(Rc, s);
    Rs2 = __fmul_ru(Rs, Rs);
    if (!(M + Rc < kClipLimit)) {   // off, as in RowClip
      X = Y = Z = 0.f;
      s = INFINITY;
      Rs2 = 1.f;
    }
  }
  __device__ __forceinline__ bool row(int cy, int cz, int lx, int hx, int& xl, int& xh) const {
    const float fy = (float)cy, fz = (float)cz;
    const float gy = fmaxf(fmaxf(Y - (fy + 1.f + s), (fy - s) - Y), 0.f);
    const float gz = fmaxf(fmaxf(Z - (fz + 1.f + s), (fz - s) - Z), 0.f);
    const float rem = Rs2 - (gy * gy + gz * gz);
    if (!(rem >= 0.f)) return false;
    const float r2 = fmaxf(rem, 1e-20f);
    const float e = r2 * rsqrtf(r2) + s;
    xl = max(__float2int_rd(X - e), lx);
    xh = min(__float2int_rd(X + e), hx);
    return xl <= xh;
  }
};

// Hit window on the bits of a non-negative FP32 distance d (bit order == value order):
// radius: d < lim;  KNN: 0 < d < lim;  and, once the heap is full, d <= root distance
// (equal distances may still win on index). A hit is bits(d) - lo <= span (unsigned);
// an inactive lane gets a window that no sum of squares can hit (-0.0 only).
__device__ __forceinline__ void hit_window(bool active, float lim, float root_d, bool knn,
                                           uint32_t& lo, uint32_t& span) {
  const uint32_t l = knn ? 1u : 0u;
  uint32_t h = __float_as_uint(root_d);
  if (lim > 0.f) h = min(h, __float_as_uint(lim) - 1u);
  if (!active || !(lim > 0.f) || h < l) {
    lo = 0x80000000u;
    span = 0u;
  } else {
    lo = l;
    span = h - l;
  }
}

// Per-lane result column in shared memory ([slot][lane], so lanes never share a bank):
// slots [0, n) hold the lane's kept neighbors -- a max-heap on (distance, index) once
// n == k -- and slots [n, fill) the hits appended since the last merge. The test loop
// writes every candidate's key at slot `fill` and advances fill only on a hit, so an
// append costs no branch; merge_column folds the appended hits in when some lane's
// column is nearly full, and once at the end of a group. While fewer than k are kept
// nothing moves (the hits are already in place); the merge that crosses k heapifies the
// first k, and later hits replace the root when smaller.
struct LaneTop {
  uint64_t root;   // largest kept key once n == k (~0 before)
  uint32_t n;      // kept entries
  uint32_t fill;   // kept + appended entries
};

// Folds slots [n, fill) into the kept set. With any_k the first k hits are kept as they
// came and later ones dropped. Out of line: it is reached from several places of the
// test loop, and one copy keeps the hot loop small enough for the instruction cache.
// KC > 0: k == KC is a compile-time constant and the heap steps are the branch-free
// fixed-depth ones (heap_sift_fixed); KC == 0: any k, data-dependent loops.
template <int KC>
__device__ __noinline__ LaneTop merge_column(uint64_t* col, LaneTop s, uint32_t k, bool any_k) {
  if constexpr (KC > 0) k = KC;
  if (s.n < k) {
    if (s.fill < k || any_k) {   // at exactly k the heap is built below
      s.n = min(s.fill, k);
      s.fill = s.n;
      return s;
    }
    if constexpr (KC > 0) {
      heapify_fixed<KC>(col);
    } else {
      for (int i = (int)k / 2 - 1; i >= 0; --i) heap_sift_down(col, (uint32_t)i, k, col[i * 32]);
    }
    s.root = col[0];
    s.n = k;
  }
  if (any_k) {
    s.fill = k;
    return s;
  }
  // slots >= k are never written by a sift, so the next key can be read ahead
  uint64_t root = s.root;
  uint64_t key = k < s.fill ? col[k * 32] : 0ull;
  for (uint32_t j = k; j < s.fill; ++j) {
    const uint64_t next = j + 1 < s.fill ? col[(j + 1) * 32] : 0ull;
    if (key < root) {
      if constexpr (KC > 0) heap_sift_fixed<KC, 0>(col, key);
      else heap_sift_down(col, 0, k, key);
      root = col[0];
    }
    key = next;
  }
  s.root = root;
  s.fill = k;
  return s;
}

__device__ __forceinline__ float root_dist(const LaneTop& s, uint32_t k) {
  return s.n == k ? __uint_as_float((uint32_t)(s.root >> 32)) : INFINITY;
}

__device__ __forceinline__ float wmin(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float wmax(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Learned widths, main pass: the width of the tile (the bucket; every lane the same value)
// from its features -- the bounding box of its searchable queries and the box counts
// around its centre -- through the width model (tile_model.cuh). A tile with no searchable
// query, or a grid that overran the cell array, keeps the full radius.
__device__ __forceinline__ float learned_tile_width(const SearchArgs& a, uint32_t cloud,
                                                   const float4& q, bool valid,
                                                   uint32_t total_cells, float* scratch) {
  if (!__any_sync(0xffffffffu, valid)) return a.radius;
  const float bx0 = wmin(valid ? q.x : INFINITY), bx1 = wmax(valid ? q.x : -INFINITY);
  const float by0 = wmin(valid ? q.y : INFINITY), by1 = wmax(valid ? q.y : -INFINITY);
  const float bz0 = wmin(valid ? q.z : INFINITY), bz1 = wmax(valid ? q.z : -INFINITY);
  const CloudGrid g = a.grids[cloud];
  if ((uint64_t)g.cell_base + g.n_cells > (uint64_t)total_cells) return a.radius;
  return tile_width(g, a.cells, a.model, a.margin, bx0, bx1, by0, by1, bz0, bz1, a.k + 1,
                    a.radius, scratch);
}

// KC > 0: the search for K == KC compiled in (the reference compiles its K in,
// camera.cu:66-72, CMakeLists.txt:58-61), with kFixedPending appended-hit slots, so the
// column length and every heap loop bound are constants; KC == 0: any K and slot count.
// Small compiled K (short result columns, so shared memory allows more resident warps):
// registers are capped so that 6 blocks of 4 warps fit an SM.
// LANES: every tile is searched lane by lane (each lane walks the cells of its own query's
// box, no shared candidate stream and no stage): the walk for dense narrow searches, where
// a tile's shared box holds many times the points of one query's ball.
template <bool KNN, int KC, bool LANES>
__global__ void __launch_bounds__(256, (KC > 0 && KC <= 16) ? 3 : 2)
k_search(SearchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const uint32_t k = KC > 0 ? (uint32_t)KC : a.k;
  const uint32_t slots = k + (KC > 0 ? kFixedPending : a.pending);   // column length per lane
  const size_t stage_bytes = LANES ? 0 : (size_t)kStage * 16;
  float* stage = reinterpret_cast<float*>(smem + (size_t)warp * stage_bytes);   // pair layout
  uint64_t* heapw = reinterpret_cast<uint64_t*>(smem + (size_t)wpb * stage_bytes) +
                    (size_t)warp * slots * 32;
  uint64_t* col = heapw + lane;   // this lane's column: col[i * 32]
  const uint32_t lt = lanemask_lt();
  const bool sorted_rows = (a.flags & kSearchSortedRows) != 0;
  const bool local_idx = (a.flags & kSearchLocalIndices) != 0;
  const bool any_k = (a.flags & kSearchAnyK) != 0;
  const bool main_pass = a.pass == kPassMain;
  const uint32_t fb_total = main_pass ? 0u : *a.fb_in_count;
  const uint32_t n_tiles = main_pass ? a.n_tiles : (fb_total + 31) / 32;
  const uint32_t total_cells = a.ctr->total_cells;

  while (true) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(a.work, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= n_tiles) break;

    bool valid;
    uint32_t pos, cloud, entry;
    float wq = a.radius;
    if (main_pass) {
      uint32_t c = 0, jt = 0;
      if (lane == 0) main_tile(a.t, tile, c, jt);
      cloud = __shfl_sync(0xffffffffu, c, 0);
      const uint32_t q0 = a.t.query_off[cloud] + __shfl_sync(0xffffffffu, jt, 0) * 32u;
      pos = q0 + lane;
      entry = pos;
      valid = pos < a.t.query_off[cloud + 1];
      if (valid && a.qwidth) wq = a.qwidth[pos];
    } else {
      entry = tile * 32u + lane;
      valid = entry < fb_total;
      pos = valid ? a.fb_in_pos[entry] : 0u;
      cloud = valid ? a.fb_in_cloud[entry] : 0u;
      if (valid && a.pass == kPassEscalate) wq = a.fb_in_width[entry];
    }
    const bool in_range = valid;
    float4 q = valid ? a.sq[pos] : make_float4(0.f, 0.f, 0.f, 0.f);
    valid = valid && isfinite(q.x) && isfinite(q.y) && isfinite(q.z);
    // the stage (the result columns of the lane walk) is free between tiles: it lends the
    // width model its 32 floats
    if (main_pass && a.model)
      wq = learned_tile_width(a, cloud, q, valid, total_cells,
                              LANES ? reinterpret_cast<float*>(heapw) : stage);
    if (a.width_out && main_pass && in_range) a.width_out[__float_as_uint(q.w)] = wq;
    float w = a.radius, lim = a.r2;
    if (wq < a.radius) { w = wq; lim = __fmul_rn(wq, wq); }

    bool short_lane = false;   // narrowed search that found fewer than K neighbors
    // The tile is searched as runs of consecutive queries: a run ends where the next query
    // (in sort order) belongs to another cloud or lies farther than gap_ratio x the widest
    // width from its predecessor, so a jump of the curve (between clouds, buckets or sparse
    // regions) never stretches one candidate box over the space between two distant groups.
    const float gap = a.gap_ratio * wmax(valid ? w : 0.f);
    const float prx = __shfl_up_sync(0xffffffffu, q.x, 1);
    const float pry = __shfl_up_sync(0xffffffffu, q.y, 1);
    const float prz = __shfl_up_sync(0xffffffffu, q.z, 1);
    const uint32_t prc = __shfl_up_sync(0xffffffffu, cloud, 1);
    const bool prv = __shfl_up_sync(0xffffffffu, valid ? 1u : 0u, 1) != 0u;
    bool run_start = valid && (lane == 0 || !prv || prc != cloud);
    if (!LANES && valid && !run_start && a.gap_ratio > 0.f) {
      const float ex = q.x - prx, ey = q.y - pry, ez = q.z - prz;
      run_start = ex * ex + ey * ey + ez * ez > gap * gap;
    }
    const uint32_t starts = __ballot_sync(0xffffffffu, run_start);
    uint32_t pending = __ballot_sync(0xffffffffu, valid);
    while (pending) {
      const int leader = __ffs(pending) - 1;   // always a run start
      const uint32_t later = starts & ~((2u << leader) - 1u);
      const int next = later ? __ffs(later) - 1 : 32;
      const uint32_t group = pending & (next == 32 ? 0xffffffffu : ((1u << next) - 1u));
      const uint32_t gcloud = __shfl_sync(0xffffffffu, cloud, leader);
      pending &= ~group;
      const bool act = (group >> lane) & 1u;
      if constexpr (!LANES) {
        // width clip (flagging passes only, whose short queries are searched again): the
        // run's widest widths are clipped to the (width_clip + 1)-th widest, at most a
        // quarter of the run, so that the candidate box follows the bulk of the run
        const uint32_t n_act = __popc(group);
        const uint32_t rank = min(a.width_clip, n_act / 4u);
        if (rank > 0 && a.fb_flag && a.pass != kPassFinal) {
          float v = act ? w : -INFINITY;   // bitonic sort, ascending over the lanes
#pragma unroll
          for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
              const float o = __shfl_xor_sync(0xffffffffu, v, stride);
              const bool up = (lane & size) == 0, low = (lane & stride) == 0;
              v = (low == up) ? fminf(v, o) : fmaxf(v, o);
            }
          }
          const float wc = __shfl_sync(0xffffffffu, v, 31 - (int)rank);
          if (act && w > wc) {
            w = wc;
            lim = __fmul_rn(wc, wc);
          }
        }
      }

      // 1. group bounding box and widest width
      const float bx0 = wmin(act ? q.x : INFINITY), bx1 = wmax(act ? q.x : -INFINITY);
      const float by0 = wmin(act ? q.y : INFINITY), by1 = wmax(act ? q.y : -INFINITY);
      const float bz0 = wmin(act ? q.z : INFINITY), bz1 = wmax(act ? q.z : -INFINITY);
      // widen by 2^-20 relative: covers every point whose rounded FP32 distance passes
      const float R = __fmul_ru(wmax(act ? w : 0.f), 1.000001f);
      const float Rk = __fmul_ru(R, 1.0001f);
      const float R2k = __fmul_ru(Rk, Rk);
      const CloudGrid g = a.grids[gcloud];
      // a grid that overran the cell array (reported by the plan) is never read
      const bool grid_ok = (uint64_t)g.cell_base + g.n_cells <= (uint64_t)total_cells;

      // 2. candidate cell box
      const float fx0 = cell_coord_f(__fsub_rn(bx0, R), g.ox, g.inv_cell);
      const float fx1 = cell_coord_f(__fadd_rn(bx1, R), g.ox, g.inv_cell);
      const float fy0 = cell_coord_f(__fsub_rn(by0, R), g.oy, g.inv_cell);
      const float fy1 = cell_coord_f(__fadd_rn(by1, R), g.oy, g.inv_cell);
      const float fz0 = cell_coord_f(__fsub_rn(bz0, R), g.oz, g.inv_cell);
      const float fz1 = cell_coord_f(__fadd_rn(bz1, R), g.oz, g.inv_cell);
      const bool empty = !(grid_ok && fx0 <= (float)(g.dx - 1) && fx1 >= 0.f &&
                           fy0 <= (float)(g.dy - 1) && fy1 >= 0.f && fz0 <= (float)(g.dz - 1) &&
                           fz1 >= 0.f);
      const int lx = (int)fmaxf(fx0, 0.f), hx = (int)fminf(fx1, (float)(g.dx - 1));
      const int ly = (int)fmaxf(fy0, 0.f), hy = (int)fminf(fy1, (float)(g.dy - 1));
      const int lz = (int)fmaxf(fz0, 0.f), hz = (int)fminf(fz1, (float)(g.dz - 1));
      const int ny = hy - ly + 1, nz = hz - lz + 1;
      const int nrows = empty ? 0 : ny * nz;
      const RowClip clip(g, bx0, bx1, by0, by1, bz0, bz1, R);

      const float lim_l = act ? lim : -1.f;
      LaneTop top{~0ull, 0u, 0u};
      uint32_t fill = 0;                 // kept + appended entries of this lane's column
      uint32_t loaded = 0, tested = 0;   // work counters of this group (warp-uniform)
      // hit test on the distance bits: lo <= bits(d) <= lo + span (see hit_window)
      uint32_t wlo, wspan;
      hit_window(act, lim_l, INFINITY, KNN, wlo, wspan);

      // 4. every lane against a staged point; a hit only appends to the lane's pending
      //    column, and the columns are merged once some lane's column has fewer than
      //    kCheck free slots (checked every kCheck candidates)
      // four candidates at a time: loads first, four independent distance chains, then
      // branch-free appends (the slot is always written, the count moves on a hit only)
      const uint64_t qx2 = pk2(q.x, q.x), qy2 = pk2(q.y, q.y), qz2 = pk2(q.z, q.z);
      auto test_pair = [&](uint64_t px, uint64_t py, uint64_t pz, uint32_t i0, uint32_t i1) {
        uint32_t d0, d1;
        dist2_pair(qx2, qy2, qz2, px, py, pz, d0, d1);
        col[fill * 32] = ((uint64_t)d0 << 32) | i0;
        fill += (d0 - wlo <= wspan) ? 1u : 0u;
        col[fill * 32] = ((uint64_t)d1 << 32) | i1;
        fill += (d1 - wlo <= wspan) ? 1u : 0u;
      };
      // four staged candidates (slots c0..c0+3, c0 even): two pairs, two f32x2 chains
      auto test4_staged = [&](int c0) {
        const float4 a0 = *reinterpret_cast<const float4*>(stage + (c0 >> 1) * 8);
        const float4 b0 = *reinterpret_cast<const float4*>(stage + (c0 >> 1) * 8 + 4);
        const float4 a1 = *reinterpret_cast<const float4*>(stage + (c0 >> 1) * 8 + 8);
        const float4 b1 = *reinterpret_cast<const float4*>(stage + (c0 >> 1) * 8 + 12);
        test_pair(pk2(a0.x, a0.y), pk2(a0.z, a0.w), pk2(b0.x, b0.y), __float_as_uint(b0.z),
                  __float_as_uint(b0.w));
        test_pair(pk2(a1.x, a1.y), pk2(a1.z, a1.w), pk2(b1.x, b1.y), __float_as_uint(b1.z),
                  __float_as_uint(b1.w));
      };
      auto test4 = [&](const float4 p0, const float4 p1, const float4 p2, const float4 p3) {
        test_pair(pk2(p0.x, p1.x), pk2(p0.y, p1.y), pk2(p0.z, p1.z), __float_as_uint(p0.w),
                  __float_as_uint(p1.w));
        test_pair(pk2(p2.x, p3.x), pk2(p2.y, p3.y), pk2(p2.z, p3.z), __float_as_uint(p2.w),
                  __float_as_uint(p3.w));
      };
      auto check = [&]() {
        if (__any_sync(0xffffffffu, fill > slots - kCheck)) {
          top.fill = fill;
          top = merge_column<KC>(col, top, k, any_k);
          fill = top.fill;
          hit_window(act && !(any_k && top.n >= k), lim_l, root_dist(top, k), KNN, wlo, wspan);
        }
      };
      uint32_t sc = 0;   // staged candidates (warp-uniform, < 32 between batches)
      // Tiles whose queries spread far beyond their width (dense clouds, narrow widths)
      // walk per lane: each lane visits only the cells of its own query's box, so it tests
      // a few times K points instead of everything near the whole tile.
      const float spread = fmaxf(fmaxf(bx1 - bx0, by1 - by0), bz1 - bz0);
      const bool lane_walk = LANES || (a.lane_walk_ratio > 0.f && spread > a.lane_walk_ratio * R);

      if (lane_walk) {
        if constexpr (LANES) {
          // This lane's box: its query +- its own width, rows clipped to the ball
          // (RowClipPoint). Rows are taken kLaneRows at a time: the row ends of a batch are
          // computed and their 2 x kLaneRows offset loads issued together, then each row's
          // points are tested four at a time (loads first, past the row's end points at
          // infinity). All lanes walk their rows in the same relative order (y fastest from
          // the low corner of the box), so lanes whose queries share a cell row read the same
          // cache lines at the same step.
          const float INF = INFINITY;
          const float4 far = make_float4(INF, INF, INF, 0.f);
          int l0 = 0, h0 = -1, l1 = 0, h1 = -1, l2 = 0, h2 = -1;
          const float Rl = act ? __fmul_ru(w, 1.000001f) : 0.f;
          if (act && grid_ok) {
            const float gx0 = cell_coord_f(__fsub_rn(q.x, Rl), g.ox, g.inv_cell);
            const float gx1 = cell_coord_f(__fadd_rn(q.x, Rl), g.ox, g.inv_cell);
            const float gy0 = cell_coord_f(__fsub_rn(q.y, Rl), g.oy, g.inv_cell);
            const float gy1 = cell_coord_f(__fadd_rn(q.y, Rl), g.oy, g.inv_cell);
            const float gz0 = cell_coord_f(__fsub_rn(q.z, Rl), g.oz, g.inv_cell);
            const float gz1 = cell_coord_f(__fadd_rn(q.z, Rl), g.oz, g.inv_cell);
            if (gx0 <= (float)(g.dx - 1) && gx1 >= 0.f && gy0 <= (float)(g.dy - 1) && gy1 >= 0.f &&
                gz0 <= (float)(g.dz - 1) && gz1 >= 0.f) {
              l0 = (int)fmaxf(gx0, 0.f); h0 = (int)fminf(gx1, (float)(g.dx - 1));
              l1 = (int)fmaxf(gy0, 0.f); h1 = (int)fminf(gy1, (float)(g.dy - 1));
              l2 = (int)fmaxf(gz0, 0.f); h2 = (int)fminf(gz1, (float)(g.dz - 1));
            }
          }
          const int nrl = (h0 >= l0 && h1 >= l1 && h2 >= l2) ? (h1 - l1 + 1) * (h2 - l2 + 1) : 0;
          const RowClipPoint lclip(g, q.x, q.y, q.z, Rl);
          int cy = l1, cz = l2;   // the next row of the walk
          uint32_t mine = 0;
          constexpr int kRows = kLaneRows;
          for (int rb = 0; __any_sync(0xffffffffu, rb < nrl); rb += kRows) {
            uint32_t rs[kRows], re[kRows];
#pragma unroll
            for (int j = 0; j < kRows; ++j) {
              rs[j] = 0u;
              re[j] = 0u;
              int xl, xh;
              if (rb + j < nrl && lclip.row(cy, cz, l0, h0, xl, xh)) {
                const uint32_t rowc =
                    g.cell_base + ((uint32_t)cz * (uint32_t)g.dy + (uint32_t)cy) * (uint32_t)g.dx;
                rs[j] = __ldg(a.cells + rowc + xl);
                re[j] = __ldg(a.cells + rowc + xh + 1);
              }
              const bool wrap = cy >= h1;
              cy = wrap ? l1 : cy + 1;
              cz = wrap ? cz + 1 : cz;
            }
#pragma unroll
            for (int j = 0; j < kRows; ++j) {
              uint32_t ptr = rs[j];
              const uint32_t end = re[j];
              while (__any_sync(0xffffffffu, ptr < end)) {
                const float4 p0 = ptr < end ? __ldg(a.spts + ptr) : far;
                const float4 p1 = ptr + 1 < end ? __ldg(a.spts + ptr + 1) : far;
                const float4 p2 = ptr + 2 < end ? __ldg(a.spts + ptr + 2) : far;
                const float4 p3 = ptr + 3 < end ? __ldg(a.spts + ptr + 3) : far;
                const uint32_t took = ptr < end ? min(end - ptr, 4u) : 0u;
                mine += took;
                ptr += took;
                test4(p0, p1, p2, p3);
                check();
              }
            }
          }
          // counters in units of 32 lane-tests, like one staged point of the shared walk
          uint32_t sum = mine;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
          loaded += sum;
          tested += (sum + 31) / 32;
        } else {
          // the tile walk's spread tiles: one row at a time over the lane's box
          const float INF = INFINITY;
          const float4 far = make_float4(INF, INF, INF, 0.f);
          int l0 = 0, h0 = -1, l1 = 0, h1 = -1, l2 = 0, h2 = -1;
          if (act && grid_ok) {
            const float Rl = __fmul_ru(w, 1.000001f);
            const float gx0 = cell_coord_f(__fsub_rn(q.x, Rl), g.ox, g.inv_cell);
            const float gx1 = cell_coord_f(__fadd_rn(q.x, Rl), g.ox, g.inv_cell);
            const float gy0 = cell_coord_f(__fsub_rn(q.y, Rl), g.oy, g.inv_cell);
            const float gy1 = cell_coord_f(__fadd_rn(q.y, Rl), g.oy, g.inv_cell);
            const float gz0 = cell_coord_f(__fsub_rn(q.z, Rl), g.oz, g.inv_cell);
            const float gz1 = cell_coord_f(__fadd_rn(q.z, Rl), g.oz, g.inv_cell);
            if (gx0 <= (float)(g.dx - 1) && gx1 >= 0.f && gy0 <= (float)(g.dy - 1) && gy1 >= 0.f &&
                gz0 <= (float)(g.dz - 1) && gz1 >= 0.f) {
              l0 = (int)fmaxf(gx0, 0.f); h0 = (int)fminf(gx1, (float)(g.dx - 1));
              l1 = (int)fmaxf(gy0, 0.f); h1 = (int)fminf(gy1, (float)(g.dy - 1));
              l2 = (int)fmaxf(gz0, 0.f); h2 = (int)fminf(gz1, (float)(g.dz - 1));
            }
          }
          const int nyl = h1 - l1 + 1;
          const int nrl = (h0 >= l0 && h1 >= l1 && h2 >= l2) ? nyl * (h2 - l2 + 1) : 0;
          int ri = 0;
          uint32_t ptr = 0, end = 0, mine = 0;
          while (true) {
            while (ptr >= end && ri < nrl) {   // next non-empty row of this lane's box
              const int cy = l1 + ri % nyl, cz = l2 + ri / nyl;
              const uint32_t rowc =
                  g.cell_base + ((uint32_t)cz * (uint32_t)g.dy + (uint32_t)cy) * (uint32_t)g.dx;
              ptr = __ldg(a.cells + rowc + l0);
              end = __ldg(a.cells + rowc + h0 + 1);
              ++ri;
            }
            if (!__any_sync(0xffffffffu, ptr < end)) break;
            // four points of this lane's current row; past its end, points at infinity
            const float4 p0 = ptr < end ? __ldg(a.spts + ptr) : far;
            const float4 p1 = ptr + 1 < end ? __ldg(a.spts + ptr + 1) : far;
            const float4 p2 = ptr + 2 < end ? __ldg(a.spts + ptr + 2) : far;
            const float4 p3 = ptr + 3 < end ? __ldg(a.spts + ptr + 3) : far;
            const uint32_t took = min(end - ptr, 4u);
            mine += took;
            ptr += took;
            test4(p0, p1, p2, p3);
            check();
          }
          // counters in units of 32 lane-tests, like one staged point of the shared walk
          uint32_t sum = mine;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
          loaded += sum;
          tested += (sum + 31) / 32;
        }
      }

      // rows in a scattered order (stride permutation: kRowStride is a prime above any row
      // count, so i -> i * kRowStride mod nrows is a bijection of [0, nrows)): a lane's hits
      // are spread over the walk instead of arriving in one burst, which keeps the lanes'
      // appended counts level and the merges short. With s = kRowStride mod nrows, row
      // number ri + 32 is row number ri plus 32 s (mod nrows): three 64-bit remainders per
      // group, then one add and one compare per batch of 32 rows.
      uint32_t rq = 0, step32 = 0;
      if (nrows > 0) {
        const uint64_t sn = kRowStride % (uint64_t)nrows;
        rq = (uint32_t)(((uint64_t)lane * sn) % (uint64_t)nrows);
        step32 = (uint32_t)((32ull * sn) % (uint64_t)nrows);
      }
      const RowSplit split(ny > 0 ? (uint32_t)ny : 1u, (uint32_t)nrows);
      for (int rb = 0; rb < (lane_walk ? 0 : nrows); rb += 32) {
        uint32_t rs = 0, re = 0;
        const int ri = rb + lane;
        if (ri < nrows) {
          uint32_t ry, rz;
          split.split(rq, ry, rz);
          const int cy = ly + (int)ry, cz = lz + (int)rz;
          int xl, xh;
          if (clip.row(cy, cz, lx, hx, xl, xh)) {
            const uint32_t rowc =
                g.cell_base + ((uint32_t)cz * (uint32_t)g.dy + (uint32_t)cy) * (uint32_t)g.dx;
            rs = __ldg(a.cells + rowc + xl);
            re = __ldg(a.cells + rowc + xh + 1);
          }
        }
        rq += step32;
        if (rq >= (uint32_t)nrows) rq -= (uint32_t)nrows;
        // the (up to) 32 rows as one sequence of candidates: an inclusive scan of the row
        // lengths; candidate t belongs to the row whose scanned end is the first above t
        const uint32_t len = re - rs;
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint32_t shift = rs - (incl - len);   // candidate t of this row: spts[t + shift]
        // index in spts of candidate t: rows whose end is <= t (binary search over the
        // lanes' scanned ends), then that row's shift
        auto cand = [&](uint32_t t) -> uint32_t {
          int row = 0;
#pragma unroll
          for (int step = 16; step > 0; step >>= 1) {
            const uint32_t e = __shfl_sync(0xffffffffu, incl, row + step - 1);
            if (e <= t) row += step;
          }
          return t + __shfl_sync(0xffffffffu, shift, row);
        };
        // the loads run one batch ahead: the next 32 candidates are in flight while this
        // batch is filtered, compacted and (once 32 are staged) tested
        float4 pn = make_float4(0.f, 0.f, 0.f, 0.f);
        if (total > 0) {
          const uint32_t idx0 = cand(lane);
          if (lane < total) pn = __ldg(a.spts + idx0);
        }
        for (uint32_t b = 0; b < total; b += 32) {
          // 3. stream 32 candidates, drop those farther than R from the box, compact the
          //    survivors behind the ones already staged (rows accumulate)
          const uint32_t t = b + lane;
          const float4 p = pn;
          if (b + 32 < total) {
            const uint32_t idxn = cand(t + 32);
            if (t + 32 < total) pn = __ldg(a.spts + idxn);
          }
          bool keep = false;
          if (t < total) {
            const float ex = fmaxf(fmaxf(bx0 - p.x, p.x - bx1), 0.f);
            const float ey = fmaxf(fmaxf(by0 - p.y, p.y - by1), 0.f);
            const float ez = fmaxf(fmaxf(bz0 - p.z, p.z - bz1), 0.f);
            keep = ex * ex + ey * ey + ez * ez <= R2k;
          }
          const uint32_t m = __ballot_sync(0xffffffffu, keep);
          if (keep) stage_put(stage, sc + __popc(m & lt), p);
          sc += __popc(m);
          loaded += min(32u, total - b);
          tested += __popc(m);
          if (sc >= 32) {
            __syncwarp();
#pragma unroll 2
            for (int c0 = 0; c0 < 32; c0 += kCheck) {
              test4_staged(c0);
              check();
            }
            __syncwarp();
            sc -= 32;
            float4 carry = make_float4(0.f, 0.f, 0.f, 0.f);
            if (lane < sc) carry = stage_get(stage, 32 + lane);
            __syncwarp();
            if (lane < sc) stage_put(stage, lane, carry);
            __syncwarp();
          }
        }
      }
      if (sc > 0) {
        // pad the last batch with points at infinity: their distance never passes
        if (lane >= sc) stage_put(stage, lane, make_float4(INFINITY, INFINITY, INFINITY, 0.f));
        __syncwarp();
        for (uint32_t c0 = 0; c0 < sc; c0 += kCheck) {
          test4_staged((int)c0);
          check();
        }
        __syncwarp();
      }

      top.fill = fill;
      top = merge_column<KC>(col, top, k, any_k);
      const uint32_t n = top.n;
      if (lane == 0 && loaded) {
        atomicAdd(&a.ctr->n_loaded, (unsigned long long)loaded);
        atomicAdd(&a.ctr->n_tested, (unsigned long long)tested);
      }
      // completion: a narrowed search that found fewer than K neighbors is redone wider.
      // The next width assumes the local density it saw: n points within w means about
      // K + 1 within w * cbrt((K + 1) / (n + 1)); a 10 % margin on that, at least 1.15 w
      // (progress) and at most 2 w (a query that found nothing doubles)
      const bool incomplete = act && (lim_l < a.r2) && (n < k);
      const bool done = act && !incomplete;
      if (act) short_lane = incomplete;
      if (incomplete && a.fb_next_w) {
        const float grow = fminf(fmaxf(1.1f * cbrtf((k + 1.f) / (n + 1.f)), 1.15f), 2.f);
        a.fb_next_w[entry] = fminf(grow * w, a.radius);
      }
      if (done && sorted_rows) {
        for (uint32_t i = 1; i < n; ++i) {
          const uint64_t x = col[i * 32];
          uint32_t j = i;
          while (j > 0 && col[(j - 1) * 32] > x) { col[j * 32] = col[(j - 1) * 32]; --j; }
          col[j * 32] = x;
        }
      }
      __syncwarp();
      // 5. coalesced row writes
      // row entries: index within the cloud (local) or + index_base (a part of a batch)
      const uint32_t sub = local_idx ? a.t.point_off[gcloud] : 0u - a.index_base;
      uint32_t wm = __ballot_sync(0xffffffffu, done);
      while (wm) {
        const int L = __ffs(wm) - 1;
        wm &= wm - 1;
        const uint32_t nL = __shfl_sync(0xffffffffu, n, L);
        const uint32_t qi = __float_as_uint(__shfl_sync(0xffffffffu, q.w, L));
        const uint32_t pL = __shfl_sync(0xffffffffu, pos, L);
        int32_t* row = a.out + (size_t)(a.ref_ppos ? pL : qi) * k;
        for (uint32_t jj = lane; jj < k; jj += 32) {
          int32_t v = -1;
          if (jj < nL) {
            const uint32_t pi = (uint32_t)heapw[jj * 32 + L];
            v = (int32_t)((a.ref_ppos ? __ldg(a.ref_ppos + pi) : pi) - sub);
          }
          row[jj] = v;
        }
      }
      __syncwarp();
    }
    // a query that cannot be searched (a non-finite coordinate) gets an empty row
    for (uint32_t m = __ballot_sync(0xffffffffu, in_range && !valid); m; m &= m - 1) {
      const int L = __ffs(m) - 1;
      const uint32_t qi = __float_as_uint(__shfl_sync(0xffffffffu, q.w, L));
      const uint32_t pL = __shfl_sync(0xffffffffu, pos, L);
      const size_t ri = a.ref_ppos ? pL : qi;
      for (uint32_t jj = lane; jj < k; jj += 32) a.out[ri * k + jj] = -1;
    }
    // flag per entry; the compaction keeps the flagged ones in this pass's order
    if (a.fb_flag && in_range) {
      a.fb_flag[entry] = short_lane ? 1u : 0u;
    }
  }
}

// ---- one warp per query ---------------------------------------------------------------
// The alternative walk for narrow widths: a warp takes a tile of 32 sorted queries like
// k_search but searches them one after another, each over its own candidate box only
// (a tile box holds many times more points than the box of one of its queries). The
// box's cell rows, clipped to the ball of radius R around the query (RowClipPoint: a
// third fewer candidates than the cube), are flattened 64 candidates at a time, two per
// lane (prefix sum of the
// row lengths, shuffle search for a candidate's row), every lane tests its candidates
// against the query, and the hits are compacted into a per-warp buffer in shared memory
// with ballots. When the buffer could overflow, and at the end when it holds more than
// K, a warp-wide bitonic sort keeps the K nearest; the sorted buffer is then the row.

// Sorts buf[0, n) ascending with the whole warp (n <= 32 E, E <= 4; position e * 32 + lane, E per
// lane, padding ~0 sorts last), writes the first `keep` (1 <= keep <= n) back to
// buf[0, keep) and returns the key at sorted position keep - 1.
template <int E>
__device__ __forceinline__ uint64_t warp_sort_keep(uint64_t* buf, uint32_t n, uint32_t keep) {
  const int lane = threadIdx.x & 31;
  uint64_t v[E];
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const uint32_t p = (uint32_t)(e * 32 + lane);
    v[e] = p < n ? buf[p] : ~0ull;
  }
  // loops over log2(size) and log2(stride): constant trip counts, fully unrolled, so v[]
  // stays in registers
  constexpr int kLog = E == 1 ? 5 : E == 2 ? 6 : 7;
#pragma unroll
  for (int ls = 1; ls <= kLog; ++ls) {
    const int size = 1 << ls;
#pragma unroll
    for (int lt = ls - 1; lt >= 0; --lt) {
      const int stride = 1 << lt;
      if (stride >= 32) {   // partner in this lane; size >= 64, so the direction is e's
        const int es = stride >> 5;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          if (e & es) continue;
          const bool up = ((e * 32) & size) == 0;
          const uint64_t x = v[e], y = v[e | es];
          const bool sw = up ? (x > y) : (x < y);
          v[e] = sw ? y : x;
          v[e | es] = sw ? x : y;
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const uint64_t o = __shfl_xor_sync(0xffffffffu, v[e], stride);
          const bool up = ((uint32_t)(e * 32 + lane) & (uint32_t)size) == 0;
          const bool low = (lane & stride) == 0;
          const uint64_t lo = v[e] < o ? v[e] : o, hi = v[e] < o ? o : v[e];
          v[e] = (low == up) ? lo : hi;
        }
      }
    }
  }
  __syncwarp();
  uint64_t kth = 0;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const uint32_t p = (uint32_t)(e * 32 + lane);
    if (p < keep) buf[p] = v[e];
    if (e == (int)((keep - 1) >> 5)) kth = v[e];
  }
  __syncwarp();
  return __shfl_sync(0xffffffffu, kth, (int)((keep - 1) & 31));
}

// Keeps the `keep` smallest of buf[0, n) (n <= 128; sorted, at buf[0, keep)); the sort is
// sized to n. Out of line: one call target keeps the query loop's registers and code small.
__device__ __noinline__ uint64_t warp_select(uint64_t* buf, uint32_t n, uint32_t keep) {
  if (n <= 32) return warp_sort_keep<1>(buf, n, keep);
  if (n <= 64) return warp_sort_keep<2>(buf, n, keep);
  return warp_sort_keep<4>(buf, n, keep);
}

// Keeps the `keep` smallest of buf[0, n) (keep < n <= 128) at buf[0, keep), in no
// particular order, and returns the largest kept key. Instead of sorting, the warp finds a
// threshold on the distance bits with exactly `keep` keys below it: every count is one
// ballot per held key (up to four per lane), the first probe is a guess -- within a ball the
// count grows as d^(3/2), so the keep-th distance lies about (2/3) log2(n / keep) octaves
// below the largest, a fixed offset on the float bits -- and the rest bisect on the bits.
// Equal distances straddling the keep-th place (lattices) are settled on the index by the
// same count-and-bisect over the indices at that distance. The kept keys are then compacted
// to the front with ballots. Out of line, like warp_select.
__device__ __noinline__ uint64_t warp_threshold_keep(uint64_t* buf, uint32_t n, uint32_t keep) {
  const int lane = threadIdx.x & 31;
  const uint32_t lt = lanemask_lt();
  uint64_t v[4];
  uint32_t lo = 0xffffffffu, hi = 0u;
  __syncwarp();
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const uint32_t p = (uint32_t)(e * 32 + lane);
    v[e] = p < n ? buf[p] : ~0ull;
    if (p < n) {
      const uint32_t d = (uint32_t)(v[e] >> 32);
      lo = min(lo, d);
      hi = max(hi, d);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  // keys whose distance bits are below t (padding ~0 never counts: its bits exceed any t)
  auto count_below = [&](uint32_t t) {
    uint32_t c = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) c += __popc(__ballot_sync(0xffffffffu, (uint32_t)(v[e] >> 32) < t));
    return c;
  };
  // invariant: count_below(L) < keep < count_below(H); hi + 1 <= 0x7f800000 (finite d)
  uint32_t L = lo, H = hi + 1u, T = 0u;
  const float drop = -0.6667f * __log2f((float)keep / (float)n) * 8388608.f;
  uint32_t t = hi - min((uint32_t)drop, hi - lo);
  while (true) {
    if (t <= L || t >= H) t = L + ((H - L) >> 1);
    if (t == L) break;   // H == L + 1: the keep-th place falls among equal distances L
    const uint32_t c = count_below(t);
    if (c == keep) { T = t; break; }
    if (c < keep) L = t; else H = t;
    t = L + ((H - L) >> 1);
  }
  const bool tie = T == 0u;
  uint32_t tie_idx = 0u;   // tie: keys at distance L with an index below tie_idx are kept
  if (tie) {
    T = L;
    const uint32_t need = keep - count_below(L);
    uint64_t IL = 0, IH = 0x100000000ull;   // indices differ: the count reaches `need`
    while (IH - IL > 1) {
      const uint64_t mid = IL + ((IH - IL) >> 1);
      uint32_t c = 0;
#pragma unroll
      for (int e = 0; e < 4; ++e)
        c += __popc(__ballot_sync(0xffffffffu, (uint32_t)(v[e] >> 32) == T && (uint32_t)v[e] < mid));
      if (c == need) { IL = mid; break; }
      if (c < need) IL = mid; else IH = mid;
    }
    tie_idx = (uint32_t)IL;
  }
  __syncwarp();
  uint32_t base = 0;
  uint64_t top = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const uint32_t d = (uint32_t)(v[e] >> 32);
    const bool kept = d < T || (tie && d == T && (uint32_t)v[e] < tie_idx);
    const uint32_t m = __ballot_sync(0xffffffffu, kept);
    if (kept) {
      buf[base + __popc(m & lt)] = v[e];
      top = max(top, v[e]);
    }
    base += __popc(m);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) top = max(top, __shfl_xor_sync(0xffffffffu, top, o));
  __syncwarp();
  return top;
}

// KC > 0: K == KC compiled in (as for k_search).
template <bool KNN, int KC>
// three blocks per SM (80 registers): the walk is latency-bound, more resident warps
// outweigh the few spills around the out-of-line sort (measured)
__global__ void __launch_bounds__(256, 3)
k_search_q(SearchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t cap = a.qcap;   // hit buffer entries per warp: k + 64 <= cap = 128
  uint64_t* buf = reinterpret_cast<uint64_t*>(smem) + (size_t)warp * cap;
  const uint32_t lt = lanemask_lt();
  const uint32_t k = KC > 0 ? (uint32_t)KC : a.k;
  const bool sorted_rows = (a.flags & kSearchSortedRows) != 0;
  const bool local_idx = (a.flags & kSearchLocalIndices) != 0;
  const bool any_k = (a.flags & kSearchAnyK) != 0;
  const bool main_pass = a.pass == kPassMain;
  const uint32_t fb_total = main_pass ? 0u : *a.fb_in_count;
  const uint32_t n_tiles = main_pass ? a.n_tiles : (fb_total + 31) / 32;
  const uint32_t total_cells = a.ctr->total_cells;
  unsigned long long loaded = 0, lane_tests = 0;   // work counters of this warp

  while (true) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(a.work, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= n_tiles) break;

    // this lane's query of the tile (the same fetch as k_search)
    bool valid;
    uint32_t pos, cloud, entry;
    float wq = a.radius;
    if (main_pass) {
      uint32_t c = 0, jt = 0;
      if (lane == 0) main_tile(a.t, tile, c, jt);
      cloud = __shfl_sync(0xffffffffu, c, 0);
      pos = a.t.query_off[cloud] + __shfl_sync(0xffffffffu, jt, 0) * 32u + lane;
      entry = pos;
      valid = pos < a.t.query_off[cloud + 1];
      if (valid && a.qwidth) wq = a.qwidth[pos];
    } else {
      entry = tile * 32u + lane;
      valid = entry < fb_total;
      pos = valid ? a.fb_in_pos[entry] : 0u;
      cloud = valid ? a.fb_in_cloud[entry] : 0u;
      if (valid && a.pass == kPassEscalate) wq = a.fb_in_width[entry];
    }
    const bool in_range = valid;
    const float4 q = valid ? a.sq[pos] : make_float4(0.f, 0.f, 0.f, 0.f);
    valid = valid && isfinite(q.x) && isfinite(q.y) && isfinite(q.z);
    // the hit buffer is free between tiles: it lends the width model its 32 floats
    if (main_pass && a.model)
      wq = learned_tile_width(a, cloud, q, valid, total_cells, reinterpret_cast<float*>(buf));
    if (a.width_out && main_pass && in_range) a.width_out[__float_as_uint(q.w)] = wq;
    float w = a.radius, lim = a.r2;
    if (wq < a.radius) { w = wq; lim = __fmul_rn(wq, wq); }
    bool short_lane = false;

    for (uint32_t todo = __ballot_sync(0xffffffffu, in_range); todo; todo &= todo - 1) {
      const int j = __ffs(todo) - 1;
      const float qx = __shfl_sync(0xffffffffu, q.x, j), qy = __shfl_sync(0xffffffffu, q.y, j);
      const float qz = __shfl_sync(0xffffffffu, q.z, j);
      const uint32_t qi = __float_as_uint(__shfl_sync(0xffffffffu, q.w, j));
      const float wj = __shfl_sync(0xffffffffu, w, j), limj = __shfl_sync(0xffffffffu, lim, j);
      const uint32_t cj = __shfl_sync(0xffffffffu, cloud, j);
      const uint32_t ej = __shfl_sync(0xffffffffu, entry, j);
      const uint32_t pj = __shfl_sync(0xffffffffu, pos, j);
      const bool vj = __shfl_sync(0xffffffffu, valid ? 1u : 0u, j) != 0u;
      int32_t* row = a.out + (size_t)(a.ref_ppos ? pj : qi) * k;
      if (!vj) {   // a non-finite coordinate: nothing to search, an empty row
        for (uint32_t jj = lane; jj < k; jj += 32) row[jj] = -1;
        continue;
      }
      const CloudGrid g = a.grids[cj];
      const bool grid_ok = (uint64_t)g.cell_base + g.n_cells <= (uint64_t)total_cells;
      // candidate cells: the query's box +- R (R widened so every point whose rounded
      // FP32 distance passes is inside)
      const float R = __fmul_ru(wj, 1.000001f);
      const float fx0 = cell_coord_f(__fsub_rn(qx, R), g.ox, g.inv_cell);
      const float fx1 = cell_coord_f(__fadd_rn(qx, R), g.ox, g.inv_cell);
      const float fy0 = cell_coord_f(__fsub_rn(qy, R), g.oy, g.inv_cell);
      const float fy1 = cell_coord_f(__fadd_rn(qy, R), g.oy, g.inv_cell);
      const float fz0 = cell_coord_f(__fsub_rn(qz, R), g.oz, g.inv_cell);
      const float fz1 = cell_coord_f(__fadd_rn(qz, R), g.oz, g.inv_cell);
      const bool empty = !(grid_ok && fx0 <= (float)(g.dx - 1) && fx1 >= 0.f &&
                           fy0 <= (float)(g.dy - 1) && fy1 >= 0.f && fz0 <= (float)(g.dz - 1) &&
                           fz1 >= 0.f);
      const int lx = (int)fmaxf(fx0, 0.f), hx = (int)fminf(fx1, (float)(g.dx - 1));
      const int ly = (int)fmaxf(fy0, 0.f), hy = (int)fminf(fy1, (float)(g.dy - 1));
      const int lz = (int)fmaxf(fz0, 0.f), hz = (int)fminf(fz1, (float)(g.dz - 1));
      const int ny = hy - ly + 1, nz = hz - lz + 1;
      const int nrows = empty ? 0 : ny * nz;
      const RowClipPoint clip(g, qx, qy, qz, R);

      uint32_t wlo, wspan;   // hit window on the distance bits (see hit_window)
      hit_window(true, limj, INFINITY, KNN, wlo, wspan);
      const uint64_t qx2 = pk2(qx, qx), qy2 = pk2(qy, qy), qz2 = pk2(qz, qz);
      uint32_t nb = 0;       // hits in the buffer (warp-uniform)
      bool stop = false;     // any_k: k hits found
      const RowSplit split(ny > 0 ? (uint32_t)ny : 1u, (uint32_t)nrows);
      for (int rb = 0; rb < nrows && !stop; rb += 32) {
        uint32_t rs = 0, re = 0;
        const int ri = rb + lane;
        int xl, xh;
        uint32_t ry = 0, rz = 0;
        if (ri < nrows) split.split((uint32_t)ri, ry, rz);
        const int cy = ly + (int)ry, cz = lz + (int)rz;
        if (ri < nrows && clip.row(cy, cz, lx, hx, xl, xh)) {
          const uint32_t rowc = g.cell_base + ((uint32_t)cz * (uint32_t)g.dy + (uint32_t)cy) * (uint32_t)g.dx;
          rs = __ldg(a.cells + rowc + xl);
          re = __ldg(a.cells + rowc + xh + 1);
        }
        const uint32_t len = re - rs;
        uint32_t incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint32_t shift = rs - (incl - len);   // candidate t of this row: spts[t + shift]
        // two candidates per lane per step (t and t + 32): independent lookups and loads
        // for the latency to overlap, and one packed distance chain for the pair
        for (uint32_t b = 0; b < total; b += 64) {
          const uint32_t t0 = b + lane, t1 = b + 32 + lane;
          int r0 = 0, r1 = 0;
#pragma unroll
          for (int step = 16; step > 0; step >>= 1) {
            const uint32_t e0 = __shfl_sync(0xffffffffu, incl, r0 + step - 1);
            const uint32_t e1 = __shfl_sync(0xffffffffu, incl, r1 + step - 1);
            if (e0 <= t0) r0 += step;
            if (e1 <= t1) r1 += step;
          }
          const uint32_t idx0 = t0 + __shfl_sync(0xffffffffu, shift, r0);
          const uint32_t idx1 = t1 + __shfl_sync(0xffffffffu, shift, r1);
          bool hit0 = false, hit1 = false;
          uint64_t key0 = 0, key1 = 0;
          const float4 p0 = t0 < total ? __ldg(a.spts + idx0) : make_float4(0.f, 0.f, 0.f, 0.f);
          const float4 p1 = t1 < total ? __ldg(a.spts + idx1) : make_float4(0.f, 0.f, 0.f, 0.f);
          {
            uint32_t d0, d1;
            dist2_pair(qx2, qy2, qz2, pk2(p0.x, p1.x), pk2(p0.y, p1.y), pk2(p0.z, p1.z), d0, d1);
            hit0 = t0 < total && d0 - wlo <= wspan;
            hit1 = t1 < total && d1 - wlo <= wspan;
            key0 = ((uint64_t)d0 << 32) | __float_as_uint(p0.w);
            key1 = ((uint64_t)d1 << 32) | __float_as_uint(p1.w);
          }
          const uint32_t m0 = __ballot_sync(0xffffffffu, hit0);
          const uint32_t m1 = __ballot_sync(0xffffffffu, hit1);
          if (hit0) buf[nb + __popc(m0 & lt)] = key0;
          nb += __popc(m0);
          if (hit1) buf[nb + __popc(m1 & lt)] = key1;
          nb += __popc(m1);
          const uint32_t took = min(64u, total - b);
          loaded += took;
          lane_tests += took;
          if (any_k) {
            if (nb >= k) { stop = true; break; }
          } else if (nb > cap - 64) {
            // keep the k nearest; later hits must beat the k-th (ties may win on index)
            const uint64_t kth = warp_threshold_keep(buf, nb, k);
            nb = k;
            hit_window(true, limj, __uint_as_float((uint32_t)(kth >> 32)), KNN, wlo, wspan);
          }
        }
      }
      const uint32_t found = min(nb, k);
      const bool incomplete = (limj < a.r2) && (found < k);
      if (lane == j) short_lane = incomplete;
      if (incomplete) {
        if (a.fb_next_w && lane == 0) {
          // the next width assumes the local density this search saw (as in k_search)
          const float grow = fminf(fmaxf(1.1f * cbrtf((k + 1.f) / (found + 1.f)), 1.15f), 2.f);
          a.fb_next_w[ej] = fminf(grow * wj, a.radius);
        }
        continue;
      }
      if (any_k) {   // the first k found, in the order found (sorted on request)
        if (sorted_rows && found > 1) warp_select(buf, found, found);
      } else if (sorted_rows && nb > 1) {
        warp_select(buf, nb, found);
      } else if (nb > k) {
        warp_threshold_keep(buf, nb, k);
      }
      __syncwarp();
      const uint32_t sub = local_idx ? a.t.point_off[cj] : 0u - a.index_base;
      for (uint32_t jj = lane; jj < k; jj += 32) {
        int32_t v = -1;
        if (jj < found) {
          const uint32_t pi = (uint32_t)buf[jj];
          v = (int32_t)((a.ref_ppos ? __ldg(a.ref_ppos + pi) : pi) - sub);
        }
        row[jj] = v;
      }
      __syncwarp();
    }
    if (a.fb_flag && in_range) a.fb_flag[entry] = short_lane ? 1u : 0u;
  }
  if (lane == 0 && loaded) {
    atomicAdd(&a.ctr->n_loaded, loaded);
    atomicAdd(&a.ctr->n_tested, (lane_tests + 31) / 32);
  }
}

// Order-preserving compaction of the short queries of a pass: flags were scanned in
// place (n + 1 entries, flags[n] = total), entry e is short when flags[e+1] > flags[e].
__global__ void k_compact_fallback(const uint32_t* __restrict__ flags, uint32_t n_host,
                                   const uint32_t* n_dev, CloudTables t,
                                   const uint32_t* __restrict__ in_pos,
                                   const uint32_t* __restrict__ in_cloud,
                                   const float* __restrict__ next_w, uint32_t* __restrict__ out_pos,
                                   uint32_t* __restrict__ out_cloud, float* __restrict__ out_w,
                                   uint32_t* out_count) {
  const uint32_t n = n_dev ? *n_dev : n_host;
  if (blockIdx.x == 0 && threadIdx.x == 0) *out_count = flags[n];
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const uint32_t o = flags[e];
    if (flags[e + 1] == o) continue;
    out_pos[o] = in_pos ? in_pos[e] : e;
    out_cloud[o] = in_cloud ? in_cloud[e] : find_cloud(t.query_off, t.n_clouds, e);
    out_w[o] = next_w[e];
  }
}

}  // namespace

cudaError_t launch_compact_fallback(const uint32_t* flags, uint32_t n_host, const uint32_t* n_dev,
                                    const CloudTables& t, const uint32_t* in_pos,
                                    const uint32_t* in_cloud, const float* next_w,
                                    uint32_t* out_pos, uint32_t* out_cloud, float* out_w,
                                    uint32_t* out_count, int n_sms, cudaStream_t s) {
  k_compact_fallback<<<n_sms * 8, 256, 0, s>>>(flags, n_host, n_dev, t, in_pos, in_cloud, next_w,
                                               out_pos, out_cloud, out_w, out_count);
  return cudaGetLastError();
}

size_t search_smem_bytes(uint32_t k, uint32_t pending, int warps_per_block, bool lanes) {
  return (size_t)warps_per_block * ((lanes ? 0 : kStage * 16) + (size_t)(k + pending) * 32 * 8);
}

void fit_search_shape(uint32_t k, uint32_t pending_req, int wpb_req, uint32_t* pending, int* wpb) {
  // sized for the tile walk (the lane walk needs no stage, so the same shape fits it)
  uint32_t p = std::max(8u, std::min(256u, pending_req)) & ~3u;
  while (p > 8 && search_smem_bytes(k, p, 1, false) > kSearchSmemLimit) p -= 4;
  int w = std::max(1, std::min(8, wpb_req));
  while (w > 1 && search_smem_bytes(k, p, w, false) > kSearchSmemLimit) --w;
  *pending = p;
  *wpb = w;
}

// The K values compiled in (a fixed set, as the reference compiles one K per build); any
// other K, or a k_search slot count other than kFixedPending, runs the generic kernels.
#define RTNN_COMPILED_KS(X) X(5) X(8) X(16) X(32) X(50) X(64)

namespace {
int compiled_k(uint32_t k) {
#define RTNN_CASE(K) if (k == K) return K;
  RTNN_COMPILED_KS(RTNN_CASE)
#undef RTNN_CASE
  return 0;
}

// kernel entry of k_search (tile or lane walk) / k_search_q for (mode, compiled K or 0)
template <bool LANES>
const void* search_fn_walk(bool knn, int kc) {
#define RTNN_CASE(K)                                                                       \
  if (kc == K)                                                                             \
    return knn ? (const void*)k_search<true, K, LANES> : (const void*)k_search<false, K, LANES>;
  RTNN_COMPILED_KS(RTNN_CASE)
#undef RTNN_CASE
  return knn ? (const void*)k_search<true, 0, LANES> : (const void*)k_search<false, 0, LANES>;
}
const void* search_fn(bool knn, int kc, bool lanes) {
  return lanes ? search_fn_walk<true>(knn, kc) : search_fn_walk<false>(knn, kc);
}
const void* search_q_fn(bool knn, int kc) {
#define RTNN_CASE(K) if (kc == K) return knn ? (const void*)k_search_q<true, K> : (const void*)k_search_q<false, K>;
  RTNN_COMPILED_KS(RTNN_CASE)
#undef RTNN_CASE
  return knn ? (const void*)k_search_q<true, 0> : (const void*)k_search_q<false, 0>;
}
int tile_kc(uint32_t k, uint32_t pending) { return pending == kFixedPending ? compiled_k(k) : 0; }
}  // namespace

int search_compiled_k(uint32_t k) { return compiled_k(k); }

cudaError_t search_prepare(int device) {
  (void)device;
  cudaError_t e = cudaSuccess;
  for (int v = 0; v < 4 && e == cudaSuccess; ++v) {
    const bool knn = v & 1, lanes = v >> 1;
    e = cudaFuncSetAttribute(search_fn(knn, 0, lanes), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kSearchSmemLimit);
#define RTNN_CASE(K)                                                                      \
    if (e == cudaSuccess)                                                                 \
      e = cudaFuncSetAttribute(search_fn(knn, K, lanes),                                  \
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSearchSmemLimit);
    RTNN_COMPILED_KS(RTNN_CASE)
#undef RTNN_CASE
  }
  return e;
}

int search_blocks_per_sm(bool knn, uint32_t k, uint32_t pending, int warps_per_block, bool lanes) {
  int nb = 0;
  const size_t smem = search_smem_bytes(k, pending, warps_per_block, lanes);
  const int threads = warps_per_block * 32;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &nb, search_fn(knn, tile_kc(k, pending), lanes), threads, smem);
  if (e != cudaSuccess) return 1;
  return nb > 0 ? nb : 1;
}

size_t search_q_smem_bytes(uint32_t qcap, int warps_per_block) {
  return (size_t)warps_per_block * qcap * 8;
}

uint32_t search_q_cap(uint32_t k) { return k + 64 <= kQueryCap ? kQueryCap : 0u; }

int search_q_blocks_per_sm(bool knn, uint32_t k, int warps_per_block) {
  int nb = 0;
  const size_t smem = search_q_smem_bytes(search_q_cap(k), warps_per_block);
  const int threads = warps_per_block * 32;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &nb, search_q_fn(knn, compiled_k(k)), threads, smem);
  if (e != cudaSuccess) return 1;
  return nb > 0 ? nb : 1;
}

cudaError_t launch_search_q(bool knn, const SearchArgs& a, unsigned blocks, int warps_per_block,
                            cudaStream_t s) {
  const size_t smem = search_q_smem_bytes(a.qcap, warps_per_block);
  SearchArgs args = a;
  void* params[] = {&args};
  return cudaLaunchKernel(search_q_fn(knn, compiled_k(a.k)), dim3(blocks),
                          dim3(warps_per_block * 32), params, smem, s);
}

cudaError_t launch_search(bool knn, const SearchArgs& a, unsigned blocks, int warps_per_block,
                          bool lanes, cudaStream_t s) {
  const size_t smem = search_smem_bytes(a.k, a.pending, warps_per_block, lanes);
  SearchArgs args = a;
  void* params[] = {&args};
  return cudaLaunchKernel(search_fn(knn, tile_kc(a.k, a.pending), lanes), dim3(blocks),
                          dim3(warps_per_block * 32), params, smem, s);
}

}  // namespace rtnn
