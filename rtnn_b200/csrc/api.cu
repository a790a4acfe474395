// api.cu -- C ABI (include/rtnn.h) and the host side of the pipeline.
//
// The pipeline replaces the timed region of optixNSearch (src/optixNSearch/main.cpp:91-148):
//   uploadData/computeMinMax (optix.cpp:117-168)      -> k_bbox, k_grid_plan
//   sortParticles/gridSort (sort.cpp:500-692)         -> k_count, scan, k_scatter
//   query Hilbert order + partition (sort.cpp:393-498) -> k_query_keys, radix sort, k_widths
//   createGeometry/gasSortSearch/search (search.cpp)  -> k_search (+ fallback pass)
// Every step is issued on one stream with no host synchronisation, so the same code
// path is captured into a CUDA graph by rtnn_plan_execute. Sizes that are only known on
// the device (cells per cloud, fallback count) are read by the kernels themselves.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rtnn.h"
#include "../../include/rtnn_learn.h"
#include "kernels.h"

using namespace rtnn;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

cudaError_t ensure(DevBuf& b, size_t bytes) {
  if (bytes < 16) bytes = 16;
  if (b.cap >= bytes) return cudaSuccess;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  const size_t want = bytes + bytes / 8;
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) { cudaGetLastError(); b.p = nullptr; return e; }
    b.cap = bytes;
    return cudaSuccess;
  }
  b.cap = want;
  return cudaSuccess;
}

void release(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}

struct Workspace {
  DevBuf tables, grids, bbox, cells, rank, spts, keys0, keys1, vals0, vals1, sq, qwidth,
      qwidth_in, fbflag, fbnextw, fbpos[2], fbcloud[2], fbwidth[2], hist, scan_state, counters,
      in_pts, in_qs, out, kth, ppos, cellsz;
  bool order_in1 = false;   // the last query sort left its permutation in vals1 (else vals0)
  void release_all() {
    for (DevBuf* b : {&tables, &grids, &bbox, &cells, &rank, &spts, &keys0, &keys1, &vals0,
                      &vals1, &sq, &qwidth, &qwidth_in, &fbflag, &fbnextw, &fbpos[0], &fbpos[1],
                      &fbcloud[0], &fbcloud[1], &fbwidth[0], &fbwidth[1], &hist, &scan_state, &counters,
                      &in_pts, &in_qs, &out, &kth, &ppos, &cellsz})
      release(*b);
  }
};

struct Shapes {
  uint32_t n_clouds = 1;
  uint64_t N = 0, Q = 0;
  bool single = true;
  std::vector<uint32_t> tab;  // batched: point_off | query_off | chunk_base | qchunk_base |
                              // tile_base | lead_base
  uint32_t n_chunks = 0, n_qchunks = 0, n_tiles = 0;
  uint64_t max_cloud_q = 0;
  uint32_t order_bits = 1, key_bits = 8;
  bool key64 = false;
  float cell_budget = 8.f;
  uint64_t cell_capacity = 0;
};

struct Params {
  rtnn_mode mode;
  float radius;
  uint32_t k;
  uint32_t flags;
  uint32_t fb_passes;   // escalating fallback passes (partitioned searches)
  uint32_t width_model; // learned widths: 0 per query (before the sort), 1 per tile (in the search)
};

uint32_t ceil_log2(uint64_t x) {
  uint32_t b = 0;
  while ((1ull << b) < x) ++b;
  return b;
}

}  // namespace

struct rtnn_ctx {
  int device = 0;
  int n_sms = 148;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  rtnn_tuning tuning{0.5f, 0.0625f, 0.f, 16.f, 4u, 0u, 1.1f, 4u, 0.0f, 2.0f, 16u, 2u, 1.0f, 0u, 0u};
  Workspace ws;
  cudaEvent_t ev[6] = {};
  Counters* h_ctr = nullptr;   // pinned
  CloudGrid* h_grid = nullptr; // pinned
  DevBuf model;
  bool has_model = false;
  DevBuf train_grad, train_m, train_v, train_loss;
  // host-buffer batches in sub-batches (run_batched_overlapped): download and upload
  // streams, per sub-batch stage events (the five of issue() and the upload's), per
  // sub-batch counters
  cudaStream_t copy = nullptr, up = nullptr;
  cudaEvent_t sub_ev[32][6] = {};
  DevBuf sub_ctr;
  uint32_t* h_tab = nullptr;   // pinned: every sub-batch's cloud tables, uploaded async
  size_t h_tab_cap = 0;
  // the order of the last search in ws (rtnn_layout): valid after a one-batch search
  bool layout_valid = false;
  uint64_t layout_n = 0, layout_q = 0;
};

struct rtnn_plan {
  rtnn_ctx* ctx = nullptr;
  Shapes sh;
  Params pr{};
  Workspace ws;
  bool use_graph = false;
  bool keep_order = false;   // RTNN_FLAG_KEEP_ORDER
  bool have_order = false;   // a sort ran and its order is kept (until rtnn_plan_resort)
  // one graph per mode: [0] sorts the queries, [1] reuses the kept order
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  const float* g_pts[2] = {nullptr, nullptr};
  const float* g_qs[2] = {nullptr, nullptr};
  int32_t* g_out[2] = {nullptr, nullptr};
};

namespace {

rtnn_status fail(rtnn_ctx* c, rtnn_status st, const std::string& msg) {
  if (c) c->err = msg;
  return st;
}

rtnn_status cuda_fail(rtnn_ctx* c, cudaError_t e, const char* where) {
  const rtnn_status st = (e == cudaErrorMemoryAllocation) ? RTNN_ERR_OUT_OF_MEMORY : RTNN_ERR_CUDA;
  return fail(c, st, std::string(where) + ": " + cudaGetErrorString(e));
}

#define RTNN_CU(call, where)                                   \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, where);     \
  } while (0)

rtnn_status check_args(rtnn_ctx* c, uint64_t N, uint64_t Q, float radius, uint32_t k,
                       uint32_t flags, bool plan = false) {
  if (!(std::isfinite(radius) && radius >= 1e-30f))
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "radius must be a finite number > 0");
  if (!rtnn_k_supported(k))
    return fail(c, RTNN_ERR_UNSUPPORTED_K, "k must be in [1, " + std::to_string(RTNN_MAX_K) + "]");
  if (N >= (1ull << 31) || Q >= (1ull << 31))
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "at most 2^31 - 1 points and queries");
  const uint32_t known = RTNN_FLAG_DEVICE_POINTERS | RTNN_FLAG_PARTITION | RTNN_FLAG_LEARNED |
                         RTNN_FLAG_SORTED_ROWS | RTNN_FLAG_LOCAL_INDICES | RTNN_FLAG_ANY_K |
                         RTNN_FLAG_REF_LAYOUT;
  if ((flags & RTNN_FLAG_KEEP_ORDER) && !plan)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "RTNN_FLAG_KEEP_ORDER applies to plans only");
  if ((flags & RTNN_FLAG_REF_LAYOUT) && plan)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT,
                "RTNN_FLAG_REF_LAYOUT applies to rtnn_search and rtnn_search_batched only");
  if (flags & ~(known | RTNN_FLAG_KEEP_ORDER))
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "unknown flag bits");
  if ((flags & RTNN_FLAG_LEARNED) && !c->has_model)
    return fail(c, RTNN_ERR_NO_MODEL,
                "RTNN_FLAG_LEARNED needs a width model (rtnn_model_set or rtnn_model_train)");
  return RTNN_OK;
}

void finish_shapes(Shapes& sh, const rtnn_tuning& tu) {
  // Hilbert steps per axis: about 64 key cells per query of the largest cloud
  uint32_t mb = (ceil_log2(std::max<uint64_t>(sh.max_cloud_q, 2)) + 6 + 2) / 3;
  mb = std::max(1u, std::min(16u, mb));
  const uint32_t cb = ceil_log2(sh.n_clouds);
  if (cb + 3 * mb + 4 > 64) mb = (60 - cb) / 3;   // room for 4 density-bucket bits
  if (mb > 1 && cb + 3 * mb + 4 > 32 && cb + 3 * (mb - 1) + 4 <= 32) --mb;   // stay 32-bit
  sh.order_bits = mb;
  sh.key_bits = std::max(8u, cb + 3 * mb);
  sh.key64 = sh.key_bits > 32;
  // cells: each cloud gets max(64, budget * points); indices stay 32-bit
  double budget = std::max(0.01f, tu.cell_budget);
  const double limit = 4.0e9;
  if (budget * (double)sh.N + 64.0 * sh.n_clouds > limit)
    budget = std::max(0.01, (limit - 64.0 * sh.n_clouds) / std::max<double>(1.0, (double)sh.N));
  sh.cell_budget = (float)budget;
  sh.cell_capacity = (uint64_t)std::ceil(budget * (double)sh.N) + 64ull * sh.n_clouds + 64;
}

Shapes single_shapes(uint64_t N, uint64_t Q, const rtnn_tuning& tu) {
  Shapes sh;
  sh.n_clouds = 1;
  sh.N = N;
  sh.Q = Q;
  sh.single = true;
  sh.n_chunks = (uint32_t)((N + kChunk - 1) / kChunk);
  sh.n_qchunks = (uint32_t)((Q + kChunk - 1) / kChunk);
  sh.n_tiles = (uint32_t)((Q + kTile - 1) / kTile);
  sh.max_cloud_q = Q;
  finish_shapes(sh, tu);
  return sh;
}

rtnn_status batched_shapes(rtnn_ctx* c, const uint64_t* point_off, uint32_t n_clouds,
                           const uint64_t* query_off, const rtnn_tuning& tu, Shapes& sh) {
  if (n_clouds == 0) return fail(c, RTNN_ERR_INVALID_ARGUMENT, "n_clouds must be > 0");
  if (!point_off) return fail(c, RTNN_ERR_INVALID_ARGUMENT, "point_offsets is NULL");
  const uint64_t* qoff = query_off ? query_off : point_off;
  if (point_off[0] != 0 || qoff[0] != 0)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "offsets must start at 0");
  const uint32_t n1 = n_clouds + 1;
  sh.n_clouds = n_clouds;
  sh.single = false;
  sh.tab.assign(6ull * n1, 0u);
  uint32_t* po = sh.tab.data();
  uint32_t* qo = po + n1;
  uint32_t* cb = qo + n1;
  uint32_t* qb = cb + n1;
  uint32_t* tb = qb + n1;
  uint32_t* lb = tb + n1;
  uint64_t chunks = 0, qchunks = 0, tiles = 0, maxq = 0;
  for (uint32_t i = 0; i < n_clouds; ++i) {
    if (point_off[i + 1] < point_off[i] || qoff[i + 1] < qoff[i])
      return fail(c, RTNN_ERR_INVALID_ARGUMENT, "offsets must be non-decreasing");
    const uint64_t np = point_off[i + 1] - point_off[i], nq = qoff[i + 1] - qoff[i];
    po[i] = (uint32_t)point_off[i];
    qo[i] = (uint32_t)qoff[i];
    cb[i] = (uint32_t)chunks;
    qb[i] = (uint32_t)qchunks;
    tb[i] = (uint32_t)tiles;
    chunks += (np + kChunk - 1) / kChunk;
    qchunks += (nq + kChunk - 1) / kChunk;
    tiles += (nq + kTile - 1) / kTile;
    maxq = std::max(maxq, nq);
  }
  sh.N = point_off[n_clouds];
  sh.Q = qoff[n_clouds];
  if (sh.N >= (1ull << 31) || sh.Q >= (1ull << 31))
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "at most 2^31 - 1 points and queries");
  po[n_clouds] = (uint32_t)sh.N;
  qo[n_clouds] = (uint32_t)sh.Q;
  cb[n_clouds] = (uint32_t)chunks;
  qb[n_clouds] = (uint32_t)qchunks;
  tb[n_clouds] = (uint32_t)tiles;
  // lead tiles (common.cuh: main_tile) only for the clouds whose tiles start in the last
  // eighth of the pass: their long tiles would otherwise start near its end. The other
  // clouds keep plain cloud order (their widest tiles lead each cloud anyway), so that a
  // cloud's tiles run close together in time and share its candidates in L2.
  const uint64_t tail_from = tiles - (tiles >> kLeadShift);
  uint64_t leads = 0;
  for (uint32_t i = 0; i < n_clouds; ++i) {
    lb[i] = (uint32_t)leads;
    if (tb[i] >= tail_from) leads += lead_tiles(tb[i + 1] - tb[i]);
  }
  lb[n_clouds] = (uint32_t)leads;
  sh.n_chunks = (uint32_t)chunks;
  sh.n_qchunks = (uint32_t)qchunks;
  sh.n_tiles = (uint32_t)tiles;
  sh.max_cloud_q = maxq;
  finish_shapes(sh, tu);
  return RTNN_OK;
}

// learned widths, unless the tuning switched them off (width_model 2: the width model
// cannot pay on this workload, every query is searched at the full radius)
bool learned(const Params& p) { return (p.flags & RTNN_FLAG_LEARNED) != 0 && p.width_model != 2; }
// narrowed widths with escalation passes: the analytic partition or the learned widths
bool partitioned(const Params& p) { return (p.flags & RTNN_FLAG_PARTITION) != 0 || learned(p); }
// learned widths per 32-query tile, evaluated by the search kernel itself
bool tile_widths(const Params& p) { return learned(p) && p.width_model == 1; }
// a width per query before the sort: the analytic partition, or the per-query model
bool per_query_widths(const Params& p) { return partitioned(p) && !tile_widths(p); }
uint32_t level_bits_of(const Params& p) { return per_query_widths(p) ? 4u : 0u; }
uint32_t key_bits_of(const Shapes& sh, const Params& p) { return sh.key_bits + level_bits_of(p); }
bool key64_of(const Shapes& sh, const Params& p) { return key_bits_of(sh, p) > 32; }

uint32_t fallback_passes_of(const Params& p) { return p.fb_passes; }

rtnn_status reserve(rtnn_ctx* c, Workspace& ws, const Shapes& sh, const Params& pr) {
  const uint64_t n1 = sh.n_clouds + 1ull;
  const uint64_t N = std::max<uint64_t>(sh.N, 1), Q = std::max<uint64_t>(sh.Q, 1);
  const uint64_t rt = radix_tiles_for(Q);
  const uint64_t scan_n = std::max<uint64_t>(std::max<uint64_t>(sh.cell_capacity + 1, 256ull * rt), Q + 1);
  RTNN_CU(ensure(ws.tables, 6 * n1 * 4), "alloc tables");
  RTNN_CU(ensure(ws.grids, sh.n_clouds * sizeof(CloudGrid)), "alloc grids");
  RTNN_CU(ensure(ws.bbox, 6ull * sh.n_clouds * 4), "alloc bbox");
  RTNN_CU(ensure(ws.cells, (sh.cell_capacity + 1) * 4), "alloc cells");
  RTNN_CU(ensure(ws.rank, N * 4), "alloc rank");
  RTNN_CU(ensure(ws.spts, N * 16), "alloc sorted points");
  RTNN_CU(ensure(ws.keys0, Q * (key64_of(sh, pr) ? 8 : 4)), "alloc keys");
  RTNN_CU(ensure(ws.keys1, Q * (key64_of(sh, pr) ? 8 : 4)), "alloc keys");
  RTNN_CU(ensure(ws.vals0, Q * 4), "alloc vals");
  RTNN_CU(ensure(ws.vals1, Q * 4), "alloc vals");
  RTNN_CU(ensure(ws.sq, Q * 16), "alloc sorted queries");
  if (pr.flags & RTNN_FLAG_REF_LAYOUT) RTNN_CU(ensure(ws.ppos, N * 4), "alloc point positions");
  RTNN_CU(ensure(ws.qwidth_in, Q * 4), "alloc widths");   // also the training features' pass
  if (per_query_widths(pr)) RTNN_CU(ensure(ws.qwidth, Q * 4), "alloc widths");
  if (partitioned(pr)) {
    for (int i = 0; i < 2; ++i) {
      RTNN_CU(ensure(ws.fbpos[i], Q * 4), "alloc fallback list");
      RTNN_CU(ensure(ws.fbcloud[i], Q * 4), "alloc fallback list");
      RTNN_CU(ensure(ws.fbwidth[i], Q * 4), "alloc fallback list");
    }
    RTNN_CU(ensure(ws.fbflag, (Q + 1) * 4), "alloc fallback flags");
    RTNN_CU(ensure(ws.fbnextw, Q * 4), "alloc fallback widths");
  }
  RTNN_CU(ensure(ws.hist, 256 * rt * 4), "alloc radix histogram");
  RTNN_CU(ensure(ws.scan_state, scan_tiles_for(scan_n) * 8), "alloc scan state");
  RTNN_CU(ensure(ws.counters, sizeof(Counters)), "alloc counters");
  return RTNN_OK;
}

CloudTables tables_of(const Workspace& ws, uint32_t n_clouds) {
  const uint32_t* t = (const uint32_t*)ws.tables.p;
  const uint32_t n1 = n_clouds + 1;
  CloudTables ct;
  ct.point_off = t;
  ct.query_off = t + n1;
  ct.chunk_base = t + 2 * n1;
  ct.qchunk_base = t + 3 * n1;
  ct.tile_base = t + 4 * n1;
  ct.lead_base = t + 5 * n1;
  ct.n_clouds = n_clouds;
  return ct;
}

// Issues the whole pipeline on stream s. ev: 4 events (or nullptr) bracketing
// build | partition | search.
uint32_t launches_of(const Shapes& sh, const Params& pr, bool reuse_order = false) {
  const uint32_t passes = sh.Q ? (key_bits_of(sh, pr) + 7) / 8 : 0;
  // tables, build (6), query keys + sort (skipped when a kept order is reused), gather
  uint32_t n = (sh.single ? 1 : 0) + 6 + (reuse_order ? 0 : 1 + 3 * passes) + 1;
  if (per_query_widths(pr)) n += 1;                          // analytic widths
  // search passes; each flagging pass adds a flag scan and a compaction
  n += partitioned(pr) ? 3 * fallback_passes_of(pr) + 4 : 1;
  return n;
}

rtnn_status issue(rtnn_ctx* c, Workspace& ws, const Shapes& sh, const Params& pr,
                  const float* d_pts, const float* d_qs, int32_t* d_out, cudaStream_t s,
                  cudaEvent_t* ev, uint32_t index_base = 0, bool reuse_order = false,
                  float* width_out = nullptr, float* feats_out = nullptr,
                  float* cellsz_out = nullptr) {
  Counters* ctr = (Counters*)ws.counters.p;
  const bool knn = pr.mode == RTNN_MODE_KNN;
  const rtnn_tuning& tu = c->tuning;
  if (ev) RTNN_CU(cudaEventRecord(ev[0], s), "event");
  RTNN_CU(cudaMemsetAsync(ctr, 0, sizeof(Counters), s), "memset counters");
  if (sh.single)
    RTNN_CU(launch_single_tables((uint32_t*)ws.tables.p, (uint32_t)sh.N, (uint32_t)sh.Q, s), "tables");
  const CloudTables t = tables_of(ws, sh.n_clouds);
  const bool ap = ((uintptr_t)d_pts % 16) == 0, aq = ((uintptr_t)d_qs % 16) == 0;
  uint32_t* cells = (uint32_t*)ws.cells.p;
  CloudGrid* grids = (CloudGrid*)ws.grids.p;

  RTNN_CU(launch_bbox(d_pts, sh.N, ap, t, sh.n_chunks, (uint32_t*)ws.bbox.p, c->n_sms, s), "bbox");
  RTNN_CU(launch_grid_plan(t, (const uint32_t*)ws.bbox.p, pr.radius, tu.cell_ratio,
                           tu.min_cell_ratio, tu.points_per_cell, sh.cell_budget, sh.order_bits,
                           sh.cell_capacity, grids, ctr, s),
          "grid plan");
  RTNN_CU(launch_zero_cells(cells, ctr, c->n_sms, s), "zero cells");
  RTNN_CU(launch_count(d_pts, sh.N, ap, t, sh.n_chunks, grids, cells, (uint32_t*)ws.rank.p, ctr, s),
          "count");
  RTNN_CU(launch_scan_excl(cells, 0, &ctr->total_cells, 1, sh.cell_capacity + 1,
                           (uint64_t*)ws.scan_state.p, &ctr->scan_tiles[0], ctr, s),
          "scan cells");
  const bool ref_layout = (pr.flags & RTNN_FLAG_REF_LAYOUT) != 0;
  RTNN_CU(launch_scatter(d_pts, sh.N, ap, t, sh.n_chunks, grids, cells, (uint32_t*)ws.rank.p,
                         (float4*)ws.spts.p, ctr, s, ref_layout ? (uint32_t*)ws.ppos.p : nullptr),
          "scatter");
  if (ev) RTNN_CU(cudaEventRecord(ev[1], s), "event");

  // density buckets: a width per query (caller's order; analytic or the per-query model),
  // then the sort key cloud | bucket of the width | Hilbert index, so each 32-query tile
  // shares one width band. Per-tile learned widths come from the search kernel itself.
  // feats_out: the per-query model's features of every query (training samples).
  const bool part = partitioned(pr);
  const bool pqw = per_query_widths(pr);
  if (pqw || feats_out) {
    WidthArgs w{};
    w.t = t;
    w.grids = grids;
    w.cells = cells;
    w.xyz = d_qs;
    // self-search: queries taken in cell order (neighbours share their row reads); widths
    // and training features are still written at the caller's query index
    w.spts = d_qs == d_pts ? (const float4*)ws.spts.p : nullptr;
    w.total_cells = &ctr->total_cells;
    w.n_queries = (uint32_t)sh.Q;
    w.radius = pr.radius;
    w.need = pr.k + 1;
    w.alpha = 1.24f;   // equal-volume radius of a (2s+2)-cell cube, util.cpp:422-426
    w.model = (learned(pr) && !tile_widths(pr)) ? (const float*)c->model.p : nullptr;
    w.margin = tu.width_margin;
    w.qwidth = (float*)ws.qwidth_in.p;
    w.feats = feats_out;
    w.cellsz = cellsz_out;
    RTNN_CU(launch_widths(w, c->n_sms, s), "widths");
  }
  // reuse_order (a RTNN_FLAG_KEEP_ORDER plan after its first execute): the permutation of
  // the last sort is still in vals0/vals1 and only the gather below runs; any order that
  // keeps each cloud's queries together gives the same rows
  if (!reuse_order) {
    const bool key64 = key64_of(sh, pr);
    RTNN_CU(launch_query_keys(d_qs, sh.Q, aq, t, sh.n_qchunks, grids, sh.order_bits,
                              pqw ? (const float*)ws.qwidth_in.p : nullptr, pr.radius,
                              level_bits_of(pr), tu.buckets_per_halving, key64, ws.keys0.p, s),
            "query keys");
    bool in1 = false;
    RTNN_CU(radix_sort_pairs(key64, ws.keys0.p, (uint32_t*)ws.vals0.p, ws.keys1.p,
                             (uint32_t*)ws.vals1.p, (uint32_t)sh.Q, key_bits_of(sh, pr), true,
                             (uint32_t*)ws.hist.p, (uint64_t*)ws.scan_state.p, &ctr->scan_tiles[1],
                             ctr, &in1, s),
            "radix sort");
    ws.order_in1 = in1;
  }
  const uint32_t* order = (const uint32_t*)(ws.order_in1 ? ws.vals1.p : ws.vals0.p);
  RTNN_CU(launch_gather_queries(d_qs, order, (uint32_t)sh.Q, (float4*)ws.sq.p,
                                pqw ? (const float*)ws.qwidth_in.p : nullptr,
                                pqw ? (float*)ws.qwidth.p : nullptr, c->n_sms, s),
          "gather queries");
  if (ev) RTNN_CU(cudaEventRecord(ev[2], s), "event");

  SearchArgs a{};
  a.t = t;
  a.grids = grids;
  a.cells = cells;
  a.spts = (const float4*)ws.spts.p;
  a.sq = (const float4*)ws.sq.p;
  a.qwidth = pqw ? (const float*)ws.qwidth.p : nullptr;
  a.model = tile_widths(pr) ? (const float*)c->model.p : nullptr;
  a.margin = tu.width_margin;
  a.width_out = width_out;
  a.out = d_out;
  a.ctr = ctr;
  a.n_tiles = sh.n_tiles;
  a.radius = pr.radius;
  a.r2 = pr.radius * pr.radius;
  a.k = pr.k;
  a.index_base = index_base;
  a.ref_ppos = ref_layout ? (const uint32_t*)ws.ppos.p : nullptr;
  a.lane_walk_ratio = tu.lane_walk_ratio;
  a.width_clip = tu.width_clip;
  a.gap_ratio = tu.gap_ratio;
  a.flags = ((pr.flags & RTNN_FLAG_SORTED_ROWS) ? kSearchSortedRows : 0u) |
            ((pr.flags & RTNN_FLAG_LOCAL_INDICES) ? kSearchLocalIndices : 0u) |
            ((pr.flags & RTNN_FLAG_ANY_K) ? kSearchAnyK : 0u);
  int wpb = 4;
  fit_search_shape(pr.k, tu.pending_slots, (int)tu.warps_per_block, &a.pending, &wpb);
  a.qcap = search_q_cap(pr.k);   // 0: k too large for one warp's hit buffer
  // kernel per pass: the tile walk, the lane walk or one warp per query (query_warps 1:
  // one warp per query in every pass; 2: tiles for the first pass, one warp per query for
  // the escalation passes, whose short queries are scattered over the clouds; 3: the lane
  // walk for the first pass, one warp per query for the escalation passes; 4: the lane
  // walk in every pass)
  const bool q_main = tu.query_warps == 1 && a.qcap != 0;
  const bool q_fallback = (tu.query_warps >= 1 && tu.query_warps <= 3) && a.qcap != 0;
  const bool l_main = tu.query_warps == 3 || tu.query_warps == 4;
  const bool l_fallback = tu.query_warps == 4;
  const int wpb_q = (int)std::max(1u, std::min(8u, tu.warps_per_block));
  auto grid_for = [&](bool per_query, bool lanes, int w) {
    int bps = per_query ? search_q_blocks_per_sm(knn, pr.k, w)
                        : search_blocks_per_sm(knn, pr.k, a.pending, w, lanes);
    if (tu.blocks_per_sm > 0) bps = std::min(bps, (int)tu.blocks_per_sm);
    const uint64_t persistent = (uint64_t)c->n_sms * bps;
    const uint64_t need_blocks = (sh.n_tiles + w - 1) / w;
    return (unsigned)std::max<uint64_t>(1, std::min(persistent, need_blocks));
  };
  const unsigned blocks_tile = grid_for(false, false, wpb);
  const unsigned blocks_lane = grid_for(false, true, wpb);
  const unsigned blocks_q = a.qcap != 0 ? grid_for(true, false, wpb_q) : 1u;
  // pass 0: every query at its partition width; each pass flags its short queries, an
  // order-preserving compaction (scan of the flags) turns them into list p%2 at a wider
  // width (grown by the density each query saw, at most doubled), and escalation pass p
  // reads list (p-1)%2; the final pass searches what
  // is left at the full radius. Lists stay in (cloud, bucket, Hilbert) order, so fallback
  // tiles remain spatially coherent.
  const int n_fb = part ? (int)fallback_passes_of(pr) : 0;
  uint32_t* flags = (uint32_t*)ws.fbflag.p;
  for (int p = 0; p <= (part ? n_fb + 1 : 0); ++p) {
    if (p == 1 && ev) RTNN_CU(cudaEventRecord(ev[3], s), "event");
    a.pass = p == 0 ? kPassMain : (p <= n_fb ? kPassEscalate : kPassFinal);
    a.work = &ctr->work[p];
    const int in = (p + 1) & 1, outl = p & 1;
    a.fb_in_pos = (const uint32_t*)ws.fbpos[in].p;
    a.fb_in_cloud = (const uint32_t*)ws.fbcloud[in].p;
    a.fb_in_width = (const float*)ws.fbwidth[in].p;
    a.fb_in_count = p > 0 ? &ctr->fb_count[p - 1] : nullptr;
    const bool flagging = part && a.pass != kPassFinal;
    a.fb_flag = flagging ? flags : nullptr;
    a.fb_next_w = flagging ? (float*)ws.fbnextw.p : nullptr;
    if (flagging) RTNN_CU(cudaMemsetAsync(flags, 0, (sh.Q + 1) * 4, s), "memset flags");
    const bool per_query = p == 0 ? q_main : q_fallback;
    const bool lanes = p == 0 ? l_main : l_fallback;
    RTNN_CU(per_query ? launch_search_q(knn, a, blocks_q, wpb_q, s)
                      : launch_search(knn, a, lanes ? blocks_lane : blocks_tile, wpb, lanes, s),
            p == 0 ? "search" : "fallback search");
    if (flagging) {
      const uint32_t* n_dev = p > 0 ? &ctr->fb_count[p - 1] : nullptr;
      RTNN_CU(launch_scan_excl(flags, sh.Q + 1, n_dev, 1, sh.Q + 1, (uint64_t*)ws.scan_state.p,
                               &ctr->scan_tiles[12 + p], ctr, s),
              "scan flags");
      RTNN_CU(launch_compact_fallback(flags, (uint32_t)sh.Q, n_dev, t,
                                      p > 0 ? a.fb_in_pos : nullptr, p > 0 ? a.fb_in_cloud : nullptr,
                                      (const float*)ws.fbnextw.p, (uint32_t*)ws.fbpos[outl].p,
                                      (uint32_t*)ws.fbcloud[outl].p, (float*)ws.fbwidth[outl].p,
                                      &ctr->fb_count[p], c->n_sms, s),
              "compact fallback");
    }
  }
  if (ev) {
    if (!part) RTNN_CU(cudaEventRecord(ev[3], s), "event");
    RTNN_CU(cudaEventRecord(ev[4], s), "event");
  }
  return RTNN_OK;
}

rtnn_status read_back(rtnn_ctx* c, Workspace& ws, cudaStream_t s, const Shapes& sh,
                      const Params& pr, rtnn_stats* stats, bool timed, bool reuse_order = false) {
  RTNN_CU(cudaMemcpyAsync(c->h_ctr, ws.counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, s),
          "read counters");
  RTNN_CU(cudaMemcpyAsync(c->h_grid, ws.grids.p, sizeof(CloudGrid), cudaMemcpyDeviceToHost, s),
          "read grid");
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  const Counters& h = *c->h_ctr;
  if (h.error == kErrScanTimeout)
    return fail(c, RTNN_ERR_DEVICE_TIMEOUT,
                "scan look-back gave up waiting on tile " + std::to_string(h.error_info));
  if (h.error == kErrCellCapacity)
    return fail(c, RTNN_ERR_INTERNAL,
                "grid plan exceeded its cell capacity (cloud " + std::to_string(h.error_info) + ")");
  if (h.error == kErrIndexRange)
    return fail(c, RTNN_ERR_INTERNAL,
                "device index check failed (element " + std::to_string(h.error_info) + ")");
  if (h.error != 0) return fail(c, RTNN_ERR_INTERNAL, "device error " + std::to_string(h.error));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->n_points = sh.N;
    stats->n_queries = sh.Q;
    stats->n_clouds = sh.n_clouds;
    stats->n_buckets = partitioned(pr) ? 2 : 1;
    stats->n_fallback = partitioned(pr) ? h.fb_count[0] : 0;
    stats->n_tiles = sh.n_tiles;
    stats->n_cells = h.total_cells;
    stats->cell_size = c->h_grid->cell;
    stats->grid_dims[0] = (uint32_t)c->h_grid->dx;
    stats->grid_dims[1] = (uint32_t)c->h_grid->dy;
    stats->grid_dims[2] = (uint32_t)c->h_grid->dz;
    stats->n_launches = launches_of(sh, pr, reuse_order);
    stats->n_loaded = h.n_loaded;
    stats->n_tested = h.n_tested;
    if (timed) {
      cudaEventElapsedTime(&stats->ms_build, c->ev[0], c->ev[1]);
      cudaEventElapsedTime(&stats->ms_partition, c->ev[1], c->ev[2]);
      cudaEventElapsedTime(&stats->ms_search, c->ev[2], c->ev[4]);
      cudaEventElapsedTime(&stats->ms_fallback, c->ev[3], c->ev[4]);
      cudaEventElapsedTime(&stats->ms_total, c->ev[0], c->ev[4]);
    }
  }
  return RTNN_OK;
}

cudaStream_t stream_of(rtnn_ctx* c) { return c->stream ? c->stream : c->own; }

// Full search with optional host staging. width_out (device, optional): the main-pass
// search width of every query.
rtnn_status run_search(rtnn_ctx* c, const Shapes& sh, const Params& pr, const float* points,
                       const float* queries, int32_t* out, rtnn_stats* stats,
                       float* width_out = nullptr, float* feats = nullptr,
                       float* cellsz = nullptr) {
  cudaStream_t s = stream_of(c);
  const bool dev = (pr.flags & RTNN_FLAG_DEVICE_POINTERS) != 0;
  const bool same = (queries == nullptr);
  if (sh.Q == 0) return RTNN_OK;
  rtnn_status st = reserve(c, c->ws, sh, pr);
  if (st != RTNN_OK) return st;
  const float* d_pts = points;
  const float* d_qs = same ? points : queries;
  int32_t* d_out = out;
  const size_t out_bytes = (size_t)sh.Q * pr.k * sizeof(int32_t);
  c->layout_valid = false;
  if (!dev) {
    RTNN_CU(ensure(c->ws.in_pts, std::max<uint64_t>(sh.N, 1) * 12), "alloc points");
    RTNN_CU(cudaMemcpyAsync(c->ws.in_pts.p, points, sh.N * 12, cudaMemcpyHostToDevice, s), "copy points");
    d_pts = (const float*)c->ws.in_pts.p;
    if (same) {
      d_qs = d_pts;
    } else {
      RTNN_CU(ensure(c->ws.in_qs, sh.Q * 12), "alloc queries");
      RTNN_CU(cudaMemcpyAsync(c->ws.in_qs.p, queries, sh.Q * 12, cudaMemcpyHostToDevice, s), "copy queries");
      d_qs = (const float*)c->ws.in_qs.p;
    }
    RTNN_CU(ensure(c->ws.out, out_bytes), "alloc output");
    d_out = (int32_t*)c->ws.out.p;
  }
  if (sh.N == 0) {
    RTNN_CU(cudaMemsetAsync(d_out, 0xff, out_bytes, s), "fill output");
  } else {
    st = issue(c, c->ws, sh, pr, d_pts, d_qs, d_out, s, c->ev, 0, false, width_out, feats,
               cellsz);
    if (st != RTNN_OK) return st;
  }
  if (!dev) RTNN_CU(cudaMemcpyAsync(out, d_out, out_bytes, cudaMemcpyDeviceToHost, s), "copy output");
  if (sh.N == 0) {
    RTNN_CU(cudaStreamSynchronize(s), "synchronize");
    if (stats) {
      std::memset(stats, 0, sizeof(*stats));
      stats->n_queries = sh.Q;
      stats->n_clouds = sh.n_clouds;
    }
    return RTNN_OK;
  }
  st = read_back(c, c->ws, s, sh, pr, stats, true);
  if (st == RTNN_OK) {
    c->layout_valid = true;
    c->layout_n = sh.N;
    c->layout_q = sh.Q;
  }
  return st;
}

// Host buffers, many clouds: the batch runs as sub-batches of whole clouds (about equal
// query counts) on the context's stream; a second stream uploads each sub-batch's points
// (and queries) ahead of its search, and a third downloads each sub-batch's rows as soon
// as it is done -- the rows of consecutive clouds are contiguous and clouds are
// independent -- so the uploads, the searches and the result download (4 K bytes per
// query, the bound of the call) all overlap; only the first sub-batch's upload and search
// and the last one's download are exposed, hence many small sub-batches. Every upload and
// sub-batch is enqueued before any download, so the host never waits on a download while
// work is still to be issued (a copy to or from pageable memory returns only once done).
// Same rows as one batch; stats are summed.
constexpr uint32_t kMaxSub = 10;
constexpr uint64_t kOverlapMinBytes = 256ull << 20;   // smaller outputs: one batch
constexpr uint64_t kSubRowBytes = 128ull << 20;       // rows per sub-batch (about)

uint32_t overlap_sub_batches(uint64_t out_bytes, uint32_t n_clouds) {
  if (out_bytes < kOverlapMinBytes || n_clouds < 2) return 1;
  return (uint32_t)std::min<uint64_t>(
      {kMaxSub, n_clouds, std::max<uint64_t>(2, out_bytes / kSubRowBytes)});
}

rtnn_status run_batched_overlapped(rtnn_ctx* c, const uint64_t* point_off, uint32_t n_clouds,
                                   const float* points, const float* queries,
                                   const uint64_t* query_off, const Params& pr, int32_t* out,
                                   rtnn_stats* stats, uint32_t n_sub) {
  const uint64_t* qoff = queries ? query_off : point_off;
  const uint64_t N = point_off[n_clouds], Q = qoff[n_clouds];
  c->layout_valid = false;   // the workspace ends up holding only the last sub-batch
  // cloud boundaries: sub-batch g starts at the first cloud holding query Q * g / n_sub
  std::vector<uint32_t> cut{0};
  for (uint32_t g = 1; g < n_sub; ++g) {
    const uint64_t target = Q * g / n_sub;
    uint32_t ci = (uint32_t)(std::upper_bound(qoff, qoff + n_clouds + 1, target) - qoff);
    ci = std::min(ci, n_clouds);
    if (ci > cut.back() && ci < n_clouds) cut.push_back(ci);
  }
  cut.push_back(n_clouds);
  const uint32_t G = (uint32_t)cut.size() - 1;
  std::vector<Shapes> shs(G);
  std::vector<uint64_t> po, qo;
  for (uint32_t g = 0; g < G; ++g) {
    const uint32_t c0 = cut[g], nc = cut[g + 1] - cut[g];
    po.assign(point_off + c0, point_off + c0 + nc + 1);
    for (auto& v : po) v -= point_off[c0];
    if (queries) {
      qo.assign(query_off + c0, query_off + c0 + nc + 1);
      for (auto& v : qo) v -= query_off[c0];
    }
    rtnn_status st = batched_shapes(c, po.data(), nc, queries ? qo.data() : nullptr, c->tuning, shs[g]);
    if (st != RTNN_OK) return st;
    st = reserve(c, c->ws, shs[g], pr);   // grows the workspace to the largest sub-batch
    if (st != RTNN_OK) return st;
  }
  cudaStream_t s = stream_of(c);
  if (!c->copy) RTNN_CU(cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking), "create stream");
  if (!c->up) RTNN_CU(cudaStreamCreateWithFlags(&c->up, cudaStreamNonBlocking), "create stream");
  for (auto& row : c->sub_ev)
    for (auto& e : row)
      if (!e) RTNN_CU(cudaEventCreateWithFlags(&e, cudaEventDefault), "create event");
  const size_t out_bytes = (size_t)Q * pr.k * sizeof(int32_t);
  RTNN_CU(ensure(c->ws.in_pts, std::max<uint64_t>(N, 1) * 12), "alloc points");
  RTNN_CU(ensure(c->ws.out, out_bytes), "alloc output");
  RTNN_CU(ensure(c->sub_ctr, (size_t)kMaxSub * sizeof(Counters)), "alloc counters");
  const float* d_pts = (const float*)c->ws.in_pts.p;
  const float* d_qs = d_pts;
  if (queries) {
    RTNN_CU(ensure(c->ws.in_qs, Q * 12), "alloc queries");
    d_qs = (const float*)c->ws.in_qs.p;
  }
  // uploads on their own stream, in sub-batch order, after the work already on the
  // context's stream (which may still read these buffers)
  RTNN_CU(cudaEventRecord(c->sub_ev[0][5], s), "event");
  RTNN_CU(cudaStreamWaitEvent(c->up, c->sub_ev[0][5], 0), "wait");
  for (uint32_t g = 0; g < G; ++g) {
    const uint64_t p0 = point_off[cut[g]], np = point_off[cut[g + 1]] - p0;
    if (np)
      RTNN_CU(cudaMemcpyAsync((char*)c->ws.in_pts.p + p0 * 12, points + 3 * p0, np * 12,
                              cudaMemcpyHostToDevice, c->up),
              "copy points");
    if (queries) {
      const uint64_t q0 = qoff[cut[g]], nq = qoff[cut[g + 1]] - q0;
      if (nq)
        RTNN_CU(cudaMemcpyAsync((char*)c->ws.in_qs.p + q0 * 12, queries + 3 * q0, nq * 12,
                                cudaMemcpyHostToDevice, c->up),
                "copy queries");
    }
    RTNN_CU(cudaEventRecord(c->sub_ev[g][5], c->up), "event");
  }
  int32_t* d_out = (int32_t*)c->ws.out.p;
  Counters* d_sub = (Counters*)c->sub_ctr.p;
  // the cloud tables of every sub-batch in pinned memory, so that their uploads never make
  // the host wait for the stream (a copy from pageable memory may)
  size_t tab_words = 0;
  for (const Shapes& sh : shs) tab_words += sh.tab.size();
  if (tab_words > c->h_tab_cap) {
    if (c->h_tab) cudaFreeHost(c->h_tab);
    c->h_tab = nullptr;
    c->h_tab_cap = 0;
    RTNN_CU(cudaMallocHost((void**)&c->h_tab, tab_words * 4), "alloc pinned tables");
    c->h_tab_cap = tab_words;
  }
  // downloads into page-locked memory are asynchronous: each is enqueued right after its
  // sub-batch; into pageable memory after the last sub-batch (such a download returns only
  // once done, and the host must first have issued all the work)
  cudaPointerAttributes oattr{};
  const bool out_pinned = cudaPointerGetAttributes(&oattr, out) == cudaSuccess &&
                          oattr.type == cudaMemoryTypeHost;
  cudaGetLastError();   // clear a failed attribute query of pageable memory
  auto download = [&](uint32_t g) -> rtnn_status {
    RTNN_CU(cudaStreamWaitEvent(c->copy, c->sub_ev[g][4], 0), "wait");
    const uint64_t q0 = qoff[cut[g]], nq = qoff[cut[g + 1]] - q0;
    if (nq)
      RTNN_CU(cudaMemcpyAsync(out + q0 * pr.k, d_out + q0 * pr.k, nq * pr.k * 4, cudaMemcpyDeviceToHost,
                              c->copy),
              "copy output");
    return RTNN_OK;
  };
  size_t tab_at = 0;
  for (uint32_t g = 0; g < G; ++g) {
    const Shapes& sh = shs[g];
    uint32_t* htab = c->h_tab + tab_at;
    tab_at += sh.tab.size();
    std::memcpy(htab, sh.tab.data(), sh.tab.size() * 4);
    RTNN_CU(cudaStreamWaitEvent(s, c->sub_ev[g][5], 0), "wait");
    RTNN_CU(cudaMemcpyAsync(c->ws.tables.p, htab, sh.tab.size() * 4, cudaMemcpyHostToDevice, s),
            "copy tables");
    if (sh.N == 0 || sh.Q == 0) {   // nothing to search: empty rows (if any), no counts
      if (sh.Q)
        RTNN_CU(cudaMemsetAsync(d_out + qoff[cut[g]] * pr.k, 0xff, sh.Q * pr.k * 4, s), "fill output");
      RTNN_CU(cudaMemsetAsync(d_sub + g, 0, sizeof(Counters), s), "clear counters");
      for (int i = 0; i < 5; ++i) RTNN_CU(cudaEventRecord(c->sub_ev[g][i], s), "event");
    } else {
      const rtnn_status st = issue(c, c->ws, sh, pr, d_pts + 3 * point_off[cut[g]],
                                   d_qs + 3 * qoff[cut[g]], d_out + qoff[cut[g]] * pr.k, s,
                                   c->sub_ev[g], (uint32_t)point_off[cut[g]]);
      if (st != RTNN_OK) return st;
      RTNN_CU(cudaMemcpyAsync(d_sub + g, c->ws.counters.p, sizeof(Counters), cudaMemcpyDeviceToDevice, s),
              "save counters");
    }
    if (out_pinned) {
      const rtnn_status st = download(g);
      if (st != RTNN_OK) return st;
    }
  }
  for (uint32_t g = 0; g < G && !out_pinned; ++g) {   // each after its sub-batch's last event
    const rtnn_status st = download(g);
    if (st != RTNN_OK) return st;
  }
  RTNN_CU(cudaStreamSynchronize(c->copy), "synchronize");
  std::vector<Counters> h(G);
  RTNN_CU(cudaMemcpyAsync(h.data(), d_sub, G * sizeof(Counters), cudaMemcpyDeviceToHost, s), "read counters");
  RTNN_CU(cudaMemcpyAsync(c->h_grid, c->ws.grids.p, sizeof(CloudGrid), cudaMemcpyDeviceToHost, s),
          "read grid");
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  for (uint32_t g = 0; g < G; ++g) {
    const Counters& hc = h[g];
    if (hc.error == kErrScanTimeout)
      return fail(c, RTNN_ERR_DEVICE_TIMEOUT,
                  "scan look-back gave up waiting on tile " + std::to_string(hc.error_info));
    if (hc.error == kErrCellCapacity)
      return fail(c, RTNN_ERR_INTERNAL, "grid plan exceeded its cell capacity (cloud " +
                                            std::to_string(cut[g] + hc.error_info) + ")");
    if (hc.error != 0) return fail(c, RTNN_ERR_INTERNAL, "device error " + std::to_string(hc.error));
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->n_points = N;
    stats->n_queries = Q;
    stats->n_clouds = n_clouds;
    stats->n_buckets = partitioned(pr) ? 2 : 1;
    stats->cell_size = c->h_grid->cell;
    stats->grid_dims[0] = (uint32_t)c->h_grid->dx;
    stats->grid_dims[1] = (uint32_t)c->h_grid->dy;
    stats->grid_dims[2] = (uint32_t)c->h_grid->dz;
    for (uint32_t g = 0; g < G; ++g) {
      const Shapes& sh = shs[g];
      if (partitioned(pr)) stats->n_fallback += h[g].fb_count[0];
      stats->n_tiles += sh.n_tiles;
      stats->n_cells += h[g].total_cells;
      stats->n_launches += (sh.N && sh.Q) ? launches_of(sh, pr) : 0;
      stats->n_loaded += h[g].n_loaded;
      stats->n_tested += h[g].n_tested;
      float t[5] = {0, 0, 0, 0, 0};
      if (sh.N && sh.Q) {
        cudaEventElapsedTime(&t[0], c->sub_ev[g][0], c->sub_ev[g][1]);
        cudaEventElapsedTime(&t[1], c->sub_ev[g][1], c->sub_ev[g][2]);
        cudaEventElapsedTime(&t[2], c->sub_ev[g][2], c->sub_ev[g][4]);
        cudaEventElapsedTime(&t[3], c->sub_ev[g][3], c->sub_ev[g][4]);
        cudaEventElapsedTime(&t[4], c->sub_ev[g][0], c->sub_ev[g][4]);
      }
      stats->ms_build += t[0];
      stats->ms_partition += t[1];
      stats->ms_search += t[2];
      stats->ms_fallback += t[3];
      stats->ms_total += t[4];
    }
  }
  return RTNN_OK;
}

}  // namespace

extern "C" {

const char* rtnn_version(void) { return "rtnn_b200 0.1.0 (sm_100a)"; }

int rtnn_k_supported(uint32_t k) { return (k >= 1 && k <= RTNN_MAX_K) ? 1 : 0; }

int rtnn_k_compiled(uint32_t k) { return search_compiled_k(k) != 0 ? 1 : 0; }

rtnn_status rtnn_create(rtnn_ctx** out, int device) {
  if (!out) return RTNN_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return RTNN_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) return RTNN_ERR_NO_DEVICE;
  rtnn_ctx* c = new rtnn_ctx();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->n_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
  for (int i = 0; i < 6 && e == cudaSuccess; ++i) e = cudaEventCreate(&c->ev[i]);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&c->h_ctr, sizeof(Counters));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&c->h_grid, sizeof(CloudGrid));
  if (e == cudaSuccess) e = search_prepare(device);
  if (e != cudaSuccess) {
    cudaGetLastError();
    rtnn_destroy(c);
    return RTNN_ERR_CUDA;
  }
  *out = c;
  return RTNN_OK;
}

rtnn_status rtnn_destroy(rtnn_ctx* c) {
  if (!c) return RTNN_OK;
  cudaSetDevice(c->device);
  if (c->own) cudaStreamSynchronize(c->own);
  c->ws.release_all();
  release(c->model);
  release(c->train_grad);
  release(c->train_m);
  release(c->train_v);
  release(c->train_loss);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto& row : c->sub_ev)
    for (auto& e : row)
      if (e) cudaEventDestroy(e);
  release(c->sub_ctr);
  if (c->copy) cudaStreamDestroy(c->copy);
  if (c->up) cudaStreamDestroy(c->up);
  if (c->h_tab) cudaFreeHost(c->h_tab);
  if (c->h_ctr) cudaFreeHost(c->h_ctr);
  if (c->h_grid) cudaFreeHost(c->h_grid);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
  return RTNN_OK;
}

const char* rtnn_last_error(const rtnn_ctx* c) { return c ? c->err.c_str() : "no context"; }

rtnn_status rtnn_set_stream(rtnn_ctx* c, void* stream) {
  if (!c) return RTNN_ERR_INVALID_ARGUMENT;
  c->stream = (cudaStream_t)stream;
  return RTNN_OK;
}

rtnn_status rtnn_get_tuning(const rtnn_ctx* c, rtnn_tuning* t) {
  if (!c || !t) return RTNN_ERR_INVALID_ARGUMENT;
  *t = c->tuning;
  return RTNN_OK;
}

rtnn_status rtnn_set_tuning(rtnn_ctx* c, const rtnn_tuning* t) {
  if (!c || !t) return RTNN_ERR_INVALID_ARGUMENT;
  if (!(t->cell_ratio > 0.f && t->cell_ratio <= 64.f) || !(t->cell_budget > 0.f) ||
      !(t->min_cell_ratio > 0.f && t->min_cell_ratio <= t->cell_ratio) ||
      !(t->points_per_cell >= 0.f) || t->fallback_passes > kMaxPasses - 2 ||
      t->warps_per_block < 1 || t->warps_per_block > 8 || !(t->width_margin > 0.f) ||
      !(t->lane_walk_ratio >= 0.f) || !(t->gap_ratio >= 0.f) || t->pending_slots < 8 ||
      t->pending_slots > 256 || t->query_warps > 4 ||
      !(t->buckets_per_halving >= 0.f && t->buckets_per_halving <= 8.f) || t->width_model > 2 ||
      t->width_clip > 16)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "tuning values out of range");
  c->tuning = *t;
  return RTNN_OK;
}

rtnn_status rtnn_search(rtnn_ctx* c, const float* points, uint64_t n_points, const float* queries,
                        uint64_t n_queries, rtnn_mode mode, float radius, uint32_t k,
                        uint32_t flags, int32_t* out, rtnn_stats* stats) {
  if (!c) return RTNN_ERR_INVALID_ARGUMENT;
  c->err.clear();
  if (mode != RTNN_MODE_RADIUS && mode != RTNN_MODE_KNN)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "mode must be RTNN_MODE_RADIUS or RTNN_MODE_KNN");
  if (queries == nullptr) n_queries = n_points;
  rtnn_status st = check_args(c, n_points, n_queries, radius, k, flags);
  if (st != RTNN_OK) return st;
  if (n_points > 0 && !points) return fail(c, RTNN_ERR_INVALID_ARGUMENT, "points is NULL");
  if (n_queries > 0 && !out) return fail(c, RTNN_ERR_INVALID_ARGUMENT, "out is NULL");
  if (flags & RTNN_FLAG_LOCAL_INDICES) flags &= ~RTNN_FLAG_LOCAL_INDICES;  // one cloud: same
  cudaSetDevice(c->device);
  const Shapes sh = single_shapes(n_points, n_queries, c->tuning);
  const Params pr{mode, radius, k, flags, c->tuning.fallback_passes, c->tuning.width_model};
  return run_search(c, sh, pr, points, queries, out, stats);
}

rtnn_status rtnn_search_batched(rtnn_ctx* c, const float* points, const uint64_t* point_offsets,
                                uint32_t n_clouds, const float* queries,
                                const uint64_t* query_offsets, rtnn_mode mode, float radius,
                                uint32_t k, uint32_t flags, int32_t* out, rtnn_stats* stats) {
  if (!c) return RTNN_ERR_INVALID_ARGUMENT;
  c->err.clear();
  if (mode != RTNN_MODE_RADIUS && mode != RTNN_MODE_KNN)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "mode must be RTNN_MODE_RADIUS or RTNN_MODE_KNN");
  Shapes sh;
  rtnn_status st = batched_shapes(c, point_offsets, n_clouds, queries ? query_offsets : nullptr,
                                  c->tuning, sh);
  if (st != RTNN_OK) return st;
  if (queries && !query_offsets) return fail(c, RTNN_ERR_INVALID_ARGUMENT, "query_offsets is NULL");
  st = check_args(c, sh.N, sh.Q, radius, k, flags);
  if (st != RTNN_OK) return st;
  if (sh.N > 0 && !points) return fail(c, RTNN_ERR_INVALID_ARGUMENT, "points is NULL");
  if (sh.Q > 0 && !out) return fail(c, RTNN_ERR_INVALID_ARGUMENT, "out is NULL");
  cudaSetDevice(c->device);
  const Params pr{mode, radius, k, flags, c->tuning.fallback_passes, c->tuning.width_model};
  st = reserve(c, c->ws, sh, pr);
  if (st != RTNN_OK) return st;
  const uint32_t n_sub = (flags & (RTNN_FLAG_DEVICE_POINTERS | RTNN_FLAG_REF_LAYOUT)) || sh.N == 0
                            ? 1u : overlap_sub_batches((uint64_t)sh.Q * k * 4, n_clouds);
  if (n_sub > 1)
    return run_batched_overlapped(c, point_offsets, n_clouds, points, queries, query_offsets, pr,
                                  out, stats, n_sub);
  cudaStream_t s = stream_of(c);
  RTNN_CU(cudaMemcpyAsync(c->ws.tables.p, sh.tab.data(), sh.tab.size() * 4, cudaMemcpyHostToDevice, s),
          "copy tables");
  return run_search(c, sh, pr, points, queries, out, stats);
}

// ---- plans (CUDA graph) ------------------------------------------------------------

rtnn_status rtnn_plan_create(rtnn_ctx* c, rtnn_plan** plan, const uint64_t* point_offsets,
                             uint32_t n_clouds, const uint64_t* query_offsets, rtnn_mode mode,
                             float radius, uint32_t k, uint32_t flags, int use_graph) {
  if (!c || !plan) return RTNN_ERR_INVALID_ARGUMENT;
  c->err.clear();
  *plan = nullptr;
  if (mode != RTNN_MODE_RADIUS && mode != RTNN_MODE_KNN)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "mode must be RTNN_MODE_RADIUS or RTNN_MODE_KNN");
  rtnn_plan* p = new rtnn_plan();
  p->ctx = c;
  rtnn_status st = batched_shapes(c, point_offsets, n_clouds, query_offsets, c->tuning, p->sh);
  if (st == RTNN_OK)
    st = check_args(c, p->sh.N, p->sh.Q, radius, k, flags | RTNN_FLAG_DEVICE_POINTERS, true);
  if (st == RTNN_OK && (p->sh.N == 0 || p->sh.Q == 0))
    st = fail(c, RTNN_ERR_INVALID_ARGUMENT, "a plan needs at least one point and one query");
  if (st != RTNN_OK) { delete p; return st; }
  p->pr = Params{mode, radius, k, flags | RTNN_FLAG_DEVICE_POINTERS, c->tuning.fallback_passes,
                 c->tuning.width_model};
  p->use_graph = use_graph != 0;
  p->keep_order = (flags & RTNN_FLAG_KEEP_ORDER) != 0;
  cudaSetDevice(c->device);
  st = reserve(c, p->ws, p->sh, p->pr);
  if (st == RTNN_OK) {
    cudaError_t e = cudaMemcpy(p->ws.tables.p, p->sh.tab.data(), p->sh.tab.size() * 4,
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) st = cuda_fail(c, e, "copy tables");
  }
  if (st != RTNN_OK) {
    p->ws.release_all();
    delete p;
    return st;
  }
  *plan = p;
  return RTNN_OK;
}

rtnn_status rtnn_plan_execute(rtnn_plan* p, const float* d_points, const float* d_queries,
                              int32_t* d_out, rtnn_stats* stats) {
  if (!p) return RTNN_ERR_INVALID_ARGUMENT;
  rtnn_ctx* c = p->ctx;
  c->err.clear();
  if (!d_points || !d_out) return fail(c, RTNN_ERR_INVALID_ARGUMENT, "NULL device pointer");
  if ((p->pr.flags & RTNN_FLAG_LEARNED) && !c->has_model)
    return fail(c, RTNN_ERR_NO_MODEL, "RTNN_FLAG_LEARNED needs a width model");
  cudaSetDevice(c->device);
  cudaStream_t s = stream_of(c);
  const float* d_qs = d_queries ? d_queries : d_points;
  const bool reuse = p->keep_order && p->have_order;
  if (!p->use_graph) {
    rtnn_status st = issue(c, p->ws, p->sh, p->pr, d_points, d_qs, d_out, s, c->ev, 0, reuse);
    if (st != RTNN_OK) return st;
    st = read_back(c, p->ws, s, p->sh, p->pr, stats, true, reuse);
    if (st == RTNN_OK && p->keep_order) p->have_order = true;
    return st;
  }
  const int m = reuse ? 1 : 0;
  if (!p->exec[m] || p->g_pts[m] != d_points || p->g_qs[m] != d_qs || p->g_out[m] != d_out) {
    if (p->exec[m]) { cudaGraphExecDestroy(p->exec[m]); p->exec[m] = nullptr; }
    if (p->graph[m]) { cudaGraphDestroy(p->graph[m]); p->graph[m] = nullptr; }
    RTNN_CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
    rtnn_status st = issue(c, p->ws, p->sh, p->pr, d_points, d_qs, d_out, s, nullptr, 0, reuse);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (st != RTNN_OK) { if (g) cudaGraphDestroy(g); return st; }
    if (e != cudaSuccess) return cuda_fail(c, e, "end capture");
    p->graph[m] = g;
    RTNN_CU(cudaGraphInstantiate(&p->exec[m], g, 0), "instantiate graph");
    p->g_pts[m] = d_points;
    p->g_qs[m] = d_qs;
    p->g_out[m] = d_out;
  }
  RTNN_CU(cudaEventRecord(c->ev[0], s), "event");
  RTNN_CU(cudaGraphLaunch(p->exec[m], s), "graph launch");
  RTNN_CU(cudaEventRecord(c->ev[4], s), "event");
  rtnn_status st = read_back(c, p->ws, s, p->sh, p->pr, stats, false, reuse);
  if (st == RTNN_OK && stats) cudaEventElapsedTime(&stats->ms_total, c->ev[0], c->ev[4]);
  if (st == RTNN_OK && p->keep_order) p->have_order = true;
  return st;
}

rtnn_status rtnn_plan_resort(rtnn_plan* p) {
  if (!p) return RTNN_ERR_INVALID_ARGUMENT;
  p->have_order = false;
  return RTNN_OK;
}

rtnn_status rtnn_plan_destroy(rtnn_plan* p) {
  if (!p) return RTNN_OK;
  cudaSetDevice(p->ctx->device);
  cudaStreamSynchronize(stream_of(p->ctx));
  for (int m = 0; m < 2; ++m) {
    if (p->exec[m]) cudaGraphExecDestroy(p->exec[m]);
    if (p->graph[m]) cudaGraphDestroy(p->graph[m]);
  }
  p->ws.release_all();
  delete p;
  return RTNN_OK;
}

// ---- learned widths -------------------------------------------------------------------

uint32_t rtnn_model_size(void) { return (uint32_t)kModelParams; }

rtnn_status rtnn_model_set(rtnn_ctx* c, const float* params, uint32_t n) {
  if (!c || !params) return RTNN_ERR_INVALID_ARGUMENT;
  if (n != (uint32_t)kModelParams)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "model must have rtnn_model_size() floats");
  cudaSetDevice(c->device);
  RTNN_CU(ensure(c->model, kModelParams * 4), "alloc model");
  RTNN_CU(cudaMemcpy(c->model.p, params, kModelParams * 4, cudaMemcpyHostToDevice), "copy model");
  c->has_model = true;
  return RTNN_OK;
}

rtnn_status rtnn_model_get(rtnn_ctx* c, float* params, uint32_t n) {
  if (!c || !params) return RTNN_ERR_INVALID_ARGUMENT;
  if (!c->has_model) return fail(c, RTNN_ERR_NO_MODEL, "no model loaded");
  if (n != (uint32_t)kModelParams)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "model must have rtnn_model_size() floats");
  cudaSetDevice(c->device);
  RTNN_CU(cudaMemcpy(params, c->model.p, kModelParams * 4, cudaMemcpyDeviceToHost), "copy model");
  return RTNN_OK;
}

rtnn_status rtnn_collect_training(rtnn_ctx* c, const float* d_points, uint64_t n_points,
                                  const float* d_queries, uint64_t n_queries, rtnn_mode mode,
                                  float radius, uint32_t k, float* d_feats, float* d_target,
                                  uint64_t* n_samples) {
  if (!c || !d_points || !d_feats || !d_target || !n_samples) return RTNN_ERR_INVALID_ARGUMENT;
  c->err.clear();
  *n_samples = 0;
  if (d_queries == nullptr) n_queries = n_points;
  const uint32_t flags = RTNN_FLAG_DEVICE_POINTERS | RTNN_FLAG_SORTED_ROWS;
  rtnn_status st = check_args(c, n_points, n_queries, radius, k, flags);
  if (st != RTNN_OK) return st;
  if (n_points == 0 || n_queries == 0) return RTNN_OK;
  cudaSetDevice(c->device);
  cudaStream_t s = stream_of(c);
  const bool per_tile = c->tuning.width_model == 1;
  RTNN_CU(ensure(c->ws.out, (size_t)n_queries * k * 4), "alloc rows");
  RTNN_CU(ensure(c->ws.kth, n_queries * 4), "alloc kth");
  const Shapes sh = single_shapes(n_points, n_queries, c->tuning);
  const Params pr{mode, radius, k, flags, c->tuning.fallback_passes, c->tuning.width_model};
  int32_t* rows = (int32_t*)c->ws.out.p;
  const float* qs = d_queries ? d_queries : d_points;
  if (per_tile) {
    // the plain search: exact rows, and the tiles (sorted queries) the learned search forms
    st = run_search(c, sh, pr, d_points, d_queries, rows, nullptr);
    if (st != RTNN_OK) return st;
    RTNN_CU(launch_kth_dist(rows, (uint32_t)n_queries, k, d_points, qs, (float*)c->ws.kth.p, s),
            "kth");
    TileSampleArgs a{};
    a.t = tables_of(c->ws, 1);
    a.grids = (const CloudGrid*)c->ws.grids.p;
    a.cells = (const uint32_t*)c->ws.cells.p;
    a.total_cells = &((const Counters*)c->ws.counters.p)->total_cells;
    a.sq = (const float4*)c->ws.sq.p;
    a.kth = (const float*)c->ws.kth.p;
    a.n_tiles = sh.n_tiles;
    a.need = k + 1;
    a.radius = radius;
    a.feats = d_feats;
    a.target = d_target;
    RTNN_CU(launch_tile_samples(a, c->n_sms, s), "tile samples");
    RTNN_CU(cudaStreamSynchronize(s), "synchronize");
    *n_samples = sh.n_tiles;
    return RTNN_OK;
  }
  // per query: the plain search writes every query's features and its cloud's cell edge
  RTNN_CU(ensure(c->ws.cellsz, n_queries * 4), "alloc cell sizes");
  st = run_search(c, sh, pr, d_points, d_queries, rows, nullptr, nullptr, d_feats,
                  (float*)c->ws.cellsz.p);
  if (st != RTNN_OK) return st;
  RTNN_CU(launch_kth_dist(rows, (uint32_t)n_queries, k, d_points, qs, (float*)c->ws.kth.p, s), "kth");
  // target = log(kth / cell); queries with < K neighbors inside r get log(1.5 r / cell)
  std::vector<float> kth(n_queries), cz(n_queries);
  RTNN_CU(cudaMemcpyAsync(kth.data(), c->ws.kth.p, n_queries * 4, cudaMemcpyDeviceToHost, s), "copy");
  RTNN_CU(cudaMemcpyAsync(cz.data(), c->ws.cellsz.p, n_queries * 4, cudaMemcpyDeviceToHost, s), "copy");
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  std::vector<float> tgt(n_queries);
  for (uint64_t i = 0; i < n_queries; ++i) {
    const float d = kth[i] >= 0.f ? std::max(kth[i], 1e-6f * radius) : 1.5f * radius;
    tgt[i] = std::log(d / cz[i]);
  }
  RTNN_CU(cudaMemcpyAsync(d_target, tgt.data(), n_queries * 4, cudaMemcpyHostToDevice, s), "copy");
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  *n_samples = n_queries;
  return RTNN_OK;
}

rtnn_status rtnn_query_widths(rtnn_ctx* c, const float* d_points, uint64_t n_points,
                              const float* d_queries, uint64_t n_queries, rtnn_mode mode,
                              float radius, uint32_t k, uint32_t flags, float* d_widths) {
  if (!c || !d_points || !d_widths) return RTNN_ERR_INVALID_ARGUMENT;
  c->err.clear();
  if (d_queries == nullptr) n_queries = n_points;
  flags = (flags & RTNN_FLAG_LEARNED) | RTNN_FLAG_PARTITION | RTNN_FLAG_DEVICE_POINTERS;
  // learned widths switched off by the tuning: the learned search takes every query at r
  if ((flags & RTNN_FLAG_LEARNED) && c->tuning.width_model == 2)
    flags = RTNN_FLAG_LEARNED | RTNN_FLAG_DEVICE_POINTERS;
  rtnn_status st = check_args(c, n_points, n_queries, radius, k, flags);
  if (st != RTNN_OK) return st;
  if (n_points == 0 || n_queries == 0) return RTNN_OK;
  cudaSetDevice(c->device);
  cudaStream_t s = stream_of(c);
  RTNN_CU(ensure(c->ws.out, (size_t)n_queries * k * 4), "alloc rows");
  const Shapes sh = single_shapes(n_points, n_queries, c->tuning);
  const Params pr{mode, radius, k, flags, c->tuning.fallback_passes, c->tuning.width_model};
  // the first search pass writes the width it searched each query at (per query for the
  // analytic partition, per tile for the learned widths)
  st = run_search(c, sh, pr, d_points, d_queries, (int32_t*)c->ws.out.p, nullptr, d_widths);
  if (st != RTNN_OK) return st;
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  return RTNN_OK;
}

rtnn_status rtnn_mlp_loss_grad(rtnn_ctx* c, const float* d_params, const float* d_feats,
                               const float* d_target, uint32_t n, float* d_grad, float* d_loss) {
  if (!c || !d_params || !d_feats || !d_target || !d_grad || !d_loss) return RTNN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  cudaStream_t s = stream_of(c);
  RTNN_CU(cudaMemsetAsync(d_grad, 0, kTrainParams * 4, s), "memset");
  RTNN_CU(cudaMemsetAsync(d_loss, 0, 4, s), "memset");
  MlpBatch b{d_feats, d_target, n};
  RTNN_CU(launch_mlp_loss_grad(d_params, b, d_grad, d_loss, c->n_sms, s), "loss/grad");
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  return RTNN_OK;
}

rtnn_status rtnn_mlp_forward(rtnn_ctx* c, const float* d_params, const float* d_feats, uint32_t n,
                             float* d_y) {
  if (!c || !d_params || !d_feats || !d_y) return RTNN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  cudaStream_t s = stream_of(c);
  RTNN_CU(launch_mlp_forward(d_params, d_feats, n, d_y, c->n_sms, s), "forward");
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  return RTNN_OK;
}

rtnn_status rtnn_mlp_adam_step(rtnn_ctx* c, float* d_params, const float* d_grad, float* d_m,
                               float* d_v, float lr, uint32_t step, float grad_scale) {
  if (!c || !d_params || !d_grad || !d_m || !d_v || step == 0) return RTNN_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  cudaStream_t s = stream_of(c);
  RTNN_CU(launch_mlp_adam(d_params, d_grad, d_m, d_v, lr, 0.9f, 0.999f, 1e-8f, step, grad_scale, s),
          "adam");
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  return RTNN_OK;
}

rtnn_status rtnn_layout(rtnn_ctx* c, uint32_t* point_order, uint64_t n_points,
                        uint32_t* query_order, uint64_t n_queries, uint32_t flags) {
  if (!c) return RTNN_ERR_INVALID_ARGUMENT;
  c->err.clear();
  if (!c->layout_valid)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT,
                "no search to describe: the last rtnn_search / rtnn_search_batched call on this "
                "context failed, had no points or queries, or ran in host sub-batches (use "
                "RTNN_FLAG_REF_LAYOUT, which keeps one batch)");
  if (flags & ~RTNN_FLAG_DEVICE_POINTERS)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "flags: only RTNN_FLAG_DEVICE_POINTERS");
  if ((point_order && n_points != c->layout_n) || (query_order && n_queries != c->layout_q))
    return fail(c, RTNN_ERR_INVALID_ARGUMENT,
                "n_points / n_queries must be those of the last search (" +
                    std::to_string(c->layout_n) + " / " + std::to_string(c->layout_q) + ")");
  cudaSetDevice(c->device);
  cudaStream_t s = stream_of(c);
  const cudaMemcpyKind kind = (flags & RTNN_FLAG_DEVICE_POINTERS) ? cudaMemcpyDeviceToDevice
                                                                  : cudaMemcpyDeviceToHost;
  // the fourth word of each sorted float4 {x, y, z, caller index}
  if (point_order && n_points)
    RTNN_CU(cudaMemcpy2DAsync(point_order, 4, (const char*)c->ws.spts.p + 12, 16, 4, n_points,
                              kind, s),
            "copy point order");
  if (query_order && n_queries)
    RTNN_CU(cudaMemcpy2DAsync(query_order, 4, (const char*)c->ws.sq.p + 12, 16, 4, n_queries,
                              kind, s),
            "copy query order");
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  return RTNN_OK;
}

rtnn_status rtnn_sort_pairs(rtnn_ctx* c, void* d_keys, uint32_t key_bytes, uint32_t* d_values,
                            uint64_t n, uint32_t key_bits) {
  if (!c) return RTNN_ERR_INVALID_ARGUMENT;
  c->err.clear();
  if (key_bytes != 4 && key_bytes != 8)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "key_bytes must be 4 or 8");
  if (key_bits == 0 || key_bits > 8 * key_bytes)
    return fail(c, RTNN_ERR_INVALID_ARGUMENT, "key_bits must be in [1, 8 * key_bytes]");
  if (n >= (1ull << 31)) return fail(c, RTNN_ERR_INVALID_ARGUMENT, "at most 2^31 - 1 pairs");
  if (n == 0) return RTNN_OK;
  if (!d_keys || !d_values) return fail(c, RTNN_ERR_INVALID_ARGUMENT, "NULL device pointer");
  cudaSetDevice(c->device);
  cudaStream_t s = stream_of(c);
  const bool key64 = key_bytes == 8;
  const uint64_t rt = radix_tiles_for(n);
  RTNN_CU(ensure(c->ws.keys1, n * key_bytes), "alloc keys");
  RTNN_CU(ensure(c->ws.vals1, n * 4), "alloc values");
  RTNN_CU(ensure(c->ws.hist, 256 * rt * 4), "alloc radix histogram");
  RTNN_CU(ensure(c->ws.scan_state, scan_tiles_for(256 * rt) * 8), "alloc scan state");
  RTNN_CU(ensure(c->ws.counters, sizeof(Counters)), "alloc counters");
  Counters* ctr = (Counters*)c->ws.counters.p;
  RTNN_CU(cudaMemsetAsync(ctr, 0, sizeof(Counters), s), "memset counters");
  bool in1 = false;
  RTNN_CU(radix_sort_pairs(key64, d_keys, d_values, c->ws.keys1.p, (uint32_t*)c->ws.vals1.p,
                           (uint32_t)n, key_bits, false, (uint32_t*)c->ws.hist.p,
                           (uint64_t*)c->ws.scan_state.p, &ctr->scan_tiles[0], ctr, &in1, s),
          "radix sort");
  if (in1) {   // an odd number of passes: the sorted pairs are in the context's buffers
    RTNN_CU(cudaMemcpyAsync(d_keys, c->ws.keys1.p, n * key_bytes, cudaMemcpyDeviceToDevice, s),
            "copy keys");
    RTNN_CU(cudaMemcpyAsync(d_values, c->ws.vals1.p, n * 4, cudaMemcpyDeviceToDevice, s),
            "copy values");
  }
  RTNN_CU(cudaMemcpyAsync(c->h_ctr, ctr, sizeof(Counters), cudaMemcpyDeviceToHost, s), "copy");
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  if (c->h_ctr->error == kErrScanTimeout)
    return fail(c, RTNN_ERR_DEVICE_TIMEOUT, "scan look-back gave up waiting on tile " +
                                                std::to_string(c->h_ctr->error_info));
  if (c->h_ctr->error != 0)
    return fail(c, RTNN_ERR_INTERNAL, "device error " + std::to_string(c->h_ctr->error));
  return RTNN_OK;
}

rtnn_status rtnn_selftest_wait_timeout(rtnn_ctx* c) {
  if (!c) return RTNN_ERR_INVALID_ARGUMENT;
  c->err.clear();
  cudaSetDevice(c->device);
  cudaStream_t s = stream_of(c);
  // two scan tiles; the tile counter starts at 1, so the only working block takes tile 1
  // and waits on tile 0, which no block ever publishes: the bounded look-back must give up
  const uint64_t n = 2ull * kScanTile;
  RTNN_CU(ensure(c->ws.cells, n * 4), "alloc");
  RTNN_CU(ensure(c->ws.scan_state, scan_tiles_for(n) * 8), "alloc");
  RTNN_CU(ensure(c->ws.counters, sizeof(Counters)), "alloc");
  Counters* ctr = (Counters*)c->ws.counters.p;
  static const uint32_t one = 1;
  RTNN_CU(cudaMemsetAsync(c->ws.cells.p, 0, n * 4, s), "memset");
  RTNN_CU(cudaMemsetAsync(ctr, 0, sizeof(Counters), s), "memset");
  RTNN_CU(cudaMemcpyAsync(&ctr->scan_tiles[0], &one, 4, cudaMemcpyHostToDevice, s), "copy");
  RTNN_CU(launch_scan_excl((uint32_t*)c->ws.cells.p, n, nullptr, 0, n,
                           (uint64_t*)c->ws.scan_state.p, &ctr->scan_tiles[0], ctr, s),
          "scan");
  RTNN_CU(cudaMemcpyAsync(c->h_ctr, ctr, sizeof(Counters), cudaMemcpyDeviceToHost, s), "copy");
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  if (c->h_ctr->error == kErrScanTimeout)
    return fail(c, RTNN_ERR_DEVICE_TIMEOUT, "scan look-back gave up waiting on tile " +
                                                std::to_string(c->h_ctr->error_info));
  return fail(c, RTNN_ERR_INTERNAL, "the bounded wait did not report a timeout");
}

rtnn_status rtnn_model_train(rtnn_ctx* c, const float* d_feats, const float* d_target,
                             uint64_t n, uint32_t epochs, uint32_t batch, float lr,
                             uint64_t seed, float* loss_per_epoch) {
  if (!c || !d_feats || !d_target || n == 0 || epochs == 0 || batch == 0)
    return RTNN_ERR_INVALID_ARGUMENT;
  c->err.clear();
  cudaSetDevice(c->device);
  cudaStream_t s = stream_of(c);
  // input / output normalisation from the data (host), He-initialised weights
  std::vector<float> f(n * kFeatDim), t(n);
  RTNN_CU(cudaMemcpyAsync(f.data(), d_feats, f.size() * 4, cudaMemcpyDeviceToHost, s), "copy");
  RTNN_CU(cudaMemcpyAsync(t.data(), d_target, t.size() * 4, cudaMemcpyDeviceToHost, s), "copy");
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  std::vector<float> P(kModelParams, 0.f);
  for (int j = 0; j < kFeatDim; ++j) {
    double m = 0, v = 0;
    for (uint64_t i = 0; i < n; ++i) m += f[i * kFeatDim + j];
    m /= (double)n;
    for (uint64_t i = 0; i < n; ++i) { const double d = f[i * kFeatDim + j] - m; v += d * d; }
    v /= (double)n;
    P[j] = (float)m;
    P[kFeatDim + j] = (float)(std::sqrt(v) < 1e-2 ? 1.0 : std::sqrt(v));   // constant feature: identity scale
  }
  {
    double m = 0, v = 0;
    for (uint64_t i = 0; i < n; ++i) m += t[i];
    m /= (double)n;
    for (uint64_t i = 0; i < n; ++i) { const double d = t[i] - m; v += d * d; }
    P[2 * kFeatDim] = (float)m;
    P[2 * kFeatDim + 1] = (float)std::max(std::sqrt(v / (double)n), 1e-3);
  }
  uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto unif = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return ((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
  };
  float* T = P.data() + kNormParams;
  const float s1 = std::sqrt(6.0f / kFeatDim), s2 = std::sqrt(6.0f / kHidden);
  for (int i = 0; i < kHidden * kFeatDim; ++i) T[i] = (float)(unif() * s1);
  float* W2 = T + kHidden * kFeatDim + kHidden;
  for (int i = 0; i < kHidden * kHidden; ++i) W2[i] = (float)(unif() * s2);
  float* W3 = W2 + kHidden * kHidden + kHidden;
  for (int i = 0; i < kHidden; ++i) W3[i] = (float)(unif() * s2 * 0.5f);
  RTNN_CU(ensure(c->model, kModelParams * 4), "alloc model");
  RTNN_CU(ensure(c->train_grad, kTrainParams * 4), "alloc grad");
  RTNN_CU(ensure(c->train_m, kTrainParams * 4), "alloc adam");
  RTNN_CU(ensure(c->train_v, kTrainParams * 4), "alloc adam");
  RTNN_CU(ensure(c->train_loss, 4 * epochs + 16), "alloc loss");
  float* dP = (float*)c->model.p;
  RTNN_CU(cudaMemcpyAsync(dP, P.data(), kModelParams * 4, cudaMemcpyHostToDevice, s), "copy");
  RTNN_CU(cudaMemsetAsync(c->train_m.p, 0, kTrainParams * 4, s), "memset");
  RTNN_CU(cudaMemsetAsync(c->train_v.p, 0, kTrainParams * 4, s), "memset");
  RTNN_CU(cudaMemsetAsync(c->train_loss.p, 0, 4 * epochs, s), "memset");
  float* dloss = (float*)c->train_loss.p;
  uint32_t step = 0;
  for (uint32_t ep = 0; ep < epochs; ++ep) {
    for (uint64_t b0 = 0; b0 < n; b0 += batch) {
      const uint32_t nb = (uint32_t)std::min<uint64_t>(batch, n - b0);
      RTNN_CU(cudaMemsetAsync(c->train_grad.p, 0, kTrainParams * 4, s), "memset");
      MlpBatch b{d_feats + b0 * kFeatDim, d_target + b0, nb};
      RTNN_CU(launch_mlp_loss_grad(dP, b, (float*)c->train_grad.p, dloss + ep, c->n_sms, s), "loss/grad");
      RTNN_CU(launch_mlp_adam(dP, (const float*)c->train_grad.p, (float*)c->train_m.p,
                              (float*)c->train_v.p, lr, 0.9f, 0.999f, 1e-8f, ++step, 1.0f / nb, s),
              "adam");
    }
  }
  if (loss_per_epoch) {
    RTNN_CU(cudaMemcpyAsync(loss_per_epoch, dloss, 4 * epochs, cudaMemcpyDeviceToHost, s), "copy");
  }
  RTNN_CU(cudaStreamSynchronize(s), "synchronize");
  if (loss_per_epoch)
    for (uint32_t ep = 0; ep < epochs; ++ep) loss_per_epoch[ep] /= (float)n;
  c->has_model = true;
  return RTNN_OK;
}

}  // extern "C"
