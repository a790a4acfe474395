// kernels.h -- host-side launchers of the device kernels (one translation unit each).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace rtnn {

constexpr uint32_t kSearchSortedRows = 1u;
constexpr uint32_t kSearchLocalIndices = 2u;
constexpr uint32_t kSearchAnyK = 4u;          // stop at the first K qualifying points

struct SearchArgs {
  CloudTables t;
  const CloudGrid* grids;
  const uint32_t* cells;       // cell start offsets (scanned counts)
  const float4* spts;          // cell-sorted points {x, y, z, index}
  const float4* sq;            // sorted queries (cloud, bucket, Hilbert) {x, y, z, query index}
  const float* qwidth;         // per sorted query search width; nullptr: full radius
  // fallback passes read the list the previous pass wrote (sorted position, cloud,
  // width to search at) ...
  const uint32_t* fb_in_pos;
  const uint32_t* fb_in_cloud;
  const float* fb_in_width;
  const uint32_t* fb_in_count;
  // ... and flag each entry that is still short (flag per entry, and the wider width
  // it is retried at); nullptr in the final pass
  uint32_t* fb_flag;
  float* fb_next_w;
  int32_t* out;                // [Q][k]
  Counters* ctr;
  uint32_t* work;              // work-queue counter of this pass
  uint32_t n_tiles;            // main pass tile count
  float radius;                // user radius r
  float r2;                    // fl(r * r)
  uint32_t k;
  uint32_t pending;            // appended-hit slots per lane beyond the k kept ones
  uint32_t qcap;               // k_search_q: hit buffer entries per warp (search_q_cap)
  uint32_t flags;              // kSearch*
  uint32_t index_base;         // added to every point index written (0 unless the points
                               // passed are a part of the caller's array)
  const uint32_t* ref_ppos;    // reference layout: row = the query's sorted position, entry =
                               // ref_ppos[point index] (its position in spts); nullptr: the
                               // caller's layout (row = query index, entry = point index)
  const float* model;          // learned widths: MLP parameters; the main pass searches each
                               // tile (bucket) at its predicted width (tile_model.cuh);
                               // nullptr: qwidth or the full radius
  float margin;                // learned width = margin * predicted K-th distance
  float* width_out;            // optional: the main-pass width of each query (query index)
  int pass;                    // kPassMain, kPassEscalate or kPassFinal
  float lane_walk_ratio;       // tile spread > ratio * width: per-lane walk (0: never)
  uint32_t width_clip;         // tile walk, flagging passes: the widest widths of a run
                               // clipped to the (width_clip + 1)-th widest (0: none)
  float gap_ratio;             // split a tile where consecutive queries are farther apart
                               // than ratio * width (0: split at cloud changes only)
};
constexpr int kPassMain = 0;      // sorted queries, widths from the partition
constexpr int kPassEscalate = 1;  // fallback list at its (widened) widths
constexpr int kPassFinal = 2;     // fallback list at the full radius (always complete)

// scan.cu
uint64_t scan_tiles_for(uint64_t n);
cudaError_t launch_scan_excl(uint32_t* data, uint64_t n_host, const uint32_t* n_dev,
                             uint32_t n_add, uint64_t max_n, uint64_t* tile_state,
                             uint32_t* tile_counter, Counters* ctr, cudaStream_t s);

// radix_sort.cu
uint32_t radix_tiles_for(uint64_t n);
cudaError_t radix_sort_pairs(bool key64, void* keys0, uint32_t* vals0, void* keys1,
                             uint32_t* vals1, uint32_t n, uint32_t bits, bool identity_values,
                             uint32_t* hist, uint64_t* scan_state, uint32_t* scan_counters,
                             Counters* ctr, bool* result_in_1, cudaStream_t s);

// build_grid.cu
cudaError_t launch_single_tables(uint32_t* tab, uint32_t n_points, uint32_t n_queries,
                                 cudaStream_t s);
cudaError_t launch_bbox(const float* xyz, uint64_t n_points, bool aligned, const CloudTables& t,
                        uint32_t n_chunks, uint32_t* bbox, int n_sms, cudaStream_t s);
cudaError_t launch_grid_plan(const CloudTables& t, const uint32_t* bbox, float radius,
                             float cell_ratio, float min_cell_ratio, float points_per_cell,
                             float cell_budget, uint32_t order_bits, uint64_t cell_capacity,
                             CloudGrid* grids, Counters* ctr, cudaStream_t s);
cudaError_t launch_zero_cells(uint32_t* cells, const Counters* ctr, int n_sms, cudaStream_t s);
cudaError_t launch_count(const float* xyz, uint64_t n_points, bool aligned, const CloudTables& t,
                         uint32_t n_chunks, const CloudGrid* grids, uint32_t* cells,
                         uint32_t* rank, Counters* ctr, cudaStream_t s);
// sorted_pos (optional): written with each point's position in spts (the inverse map)
cudaError_t launch_scatter(const float* xyz, uint64_t n_points, bool aligned,
                           const CloudTables& t, uint32_t n_chunks, const CloudGrid* grids,
                           const uint32_t* cells, const uint32_t* rank, float4* spts,
                           Counters* ctr, cudaStream_t s, uint32_t* sorted_pos = nullptr);
cudaError_t launch_query_keys(const float* xyz, uint64_t n_queries, bool aligned,
                              const CloudTables& t, uint32_t n_qchunks, const CloudGrid* grids,
                              uint32_t order_bits, const float* qwidth, float radius,
                              uint32_t level_bits, float per_halving, bool key64, void* keys,
                              cudaStream_t s);
cudaError_t launch_gather_queries(const float* xyz, const uint32_t* order, uint32_t n,
                                  float4* sq, const float* w_in, float* w_out, int n_sms,
                                  cudaStream_t s);

// search.cu
constexpr size_t kSearchSmemLimit = 227 * 1024;   // dynamic shared memory per block
// lanes: the lane walk (k_search with LANES), which needs no candidate stage
size_t search_smem_bytes(uint32_t k, uint32_t pending, int warps_per_block, bool lanes);
cudaError_t search_prepare(int device);
int search_blocks_per_sm(bool knn, uint32_t k, uint32_t pending, int warps_per_block, bool lanes);
// K itself when the searches have an instantiation with K compiled in, else 0
int search_compiled_k(uint32_t k);
// appended-hit slots (multiple of 4, 8..256) and warps per block that fit the limit
void fit_search_shape(uint32_t k, uint32_t pending_req, int wpb_req, uint32_t* pending, int* wpb);
// one warp per query (k_search_q): buffer size for k, occupancy and launch
uint32_t search_q_cap(uint32_t k);
int search_q_blocks_per_sm(bool knn, uint32_t k, int warps_per_block);
cudaError_t launch_search_q(bool knn, const SearchArgs& a, unsigned blocks, int warps_per_block,
                            cudaStream_t s);
cudaError_t launch_search(bool knn, const SearchArgs& a, unsigned blocks, int warps_per_block,
                          bool lanes, cudaStream_t s);
cudaError_t launch_compact_fallback(const uint32_t* flags, uint32_t n_host, const uint32_t* n_dev,
                                    const CloudTables& t, const uint32_t* in_pos,
                                    const uint32_t* in_cloud, const float* next_w,
                                    uint32_t* out_pos, uint32_t* out_cloud, float* out_w,
                                    uint32_t* out_count, int n_sms, cudaStream_t s);

// partition.cu -- density buckets: per-query search widths (analytic or learned MLP)
constexpr int kShells = 3;                 // box counts N_0..N_2 around a query's cell
constexpr int kFeatDim = 6;                // MLP input features per query
constexpr int kHidden = 16;                // MLP hidden width (two hidden layers)
// parameter layout (floats): in_mean[F] in_std[F] out_mean out_std | W1[H][F] b1[H]
// W2[H][H] b2[H] W3[H] b3  -- only the part after '|' is trained
constexpr int kNormParams = 2 * kFeatDim + 2;
constexpr int kTrainParams = kHidden * kFeatDim + kHidden + kHidden * kHidden + kHidden + kHidden + 1;
constexpr int kModelParams = kNormParams + kTrainParams;

// a width per query before the sort: the analytic partition (RTNN_FLAG_PARTITION), or the
// per-query width model (RTNN_FLAG_LEARNED with rtnn_tuning.width_model == 0)
struct WidthArgs {
  CloudTables t;
  const CloudGrid* grids;
  const uint32_t* cells;
  const float* xyz;             // queries in the caller's order (AoS float3)
  const float4* spts;           // when the queries are the points: the cell-sorted points,
                                // walked instead of xyz (nullptr: walk xyz)
  const uint32_t* total_cells;  // cells in use (device)
  uint32_t n_queries;
  float radius;
  uint32_t need;          // points a width must enclose (K + 1)
  float alpha;            // analytic width = alpha * (s* + 1) * cell
  const float* model;     // per-query width model (nullptr: analytic)
  float margin;           // learned width = margin * predicted K-th distance
  float* qwidth;          // out: per query width, caller order (>= radius means full radius)
  float* feats;           // optional out: [query index][kFeatDim] features (caller order)
  float* cellsz;          // optional out: [query index] cell edge of the query's cloud
};
cudaError_t launch_widths(const WidthArgs& a, int n_sms, cudaStream_t s);

// learned widths: one training sample per tile (bucket) of a plain search -- the tile's
// features (tile_model.cuh) and target log(largest K-th distance of its queries / cell)
struct TileSampleArgs {
  CloudTables t;
  const CloudGrid* grids;
  const uint32_t* cells;
  const uint32_t* total_cells;  // cells in use (device)
  const float4* sq;             // the search's sorted queries {x, y, z, query index}
  const float* kth;             // K-th neighbor distance per query index (-1: fewer than K)
  uint32_t n_tiles;
  uint32_t need;                // K + 1
  float radius;
  float* feats;                 // out: [tile][kFeatDim]
  float* target;                // out: [tile]
};
cudaError_t launch_tile_samples(const TileSampleArgs& a, int n_sms, cudaStream_t s);

// MLP training (hand-written forward / backward / Adam), mlp.cu
struct MlpBatch {
  const float* feats;     // [n][kFeatDim]
  const float* target;    // [n] log(K-th distance / cell)
  uint32_t n;
};
cudaError_t launch_mlp_loss_grad(const float* params, const MlpBatch& b, float* grad,
                                 float* loss_sum, int n_sms, cudaStream_t s);
cudaError_t launch_mlp_adam(float* params, const float* grad, float* m, float* v, float lr,
                            float beta1, float beta2, float eps, uint32_t step, float scale,
                            cudaStream_t s);
cudaError_t launch_mlp_forward(const float* params, const float* feats, uint32_t n, float* y,
                               int n_sms, cudaStream_t s);
cudaError_t launch_kth_dist(const int32_t* rows, uint32_t n_queries, uint32_t k,
                            const float* points, const float* queries, float* kth_d,
                            cudaStream_t s);

}  // namespace rtnn
