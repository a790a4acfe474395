/*
 * rtnn.h -- C ABI of the B200-native neighbor-search engine (librtnn_b200.so).
 *
 * The reference (horizon-research/rtnn) has no library API: its boundary is the
 * `optixNSearch` executable (src/optixNSearch/main.cpp:47-161). Each entry point
 * below replaces one step of that executable; the replaced reference code is cited
 * beside it. All calls return an rtnn_status and never throw across the ABI; the
 * message of the last failure on a context is available from rtnn_last_error().
 *
 * Output contract (src/optixNSearch/search.cpp:18, geometry.cu:72-83,
 * camera.cu:99-104): a row-major Q x K int32 buffer, row q holding the neighbors of
 * query q; unused slots hold -1 (the reference's UINT_MAX). Indices refer to the
 * caller's point order (the reference returns indices into its Morton-sorted copy).
 *
 * Predicates (distance d = ((dx*dx + dy*dy) + dz*dz) in FP32, each operation
 * rounded, no FMA: src/sutil/vec_math.h:527-530, check.cpp:36-37):
 *   RTNN_MODE_RADIUS: d < r*r, the query itself included (geometry.cu:61-66).
 *   RTNN_MODE_KNN:    0 < d < r*r, coincident points excluded (geometry.cu:187).
 * When more than K points qualify, the K smallest by (d, index) are returned, so the
 * neighbor set of every row is deterministic and exact.
 *
 * Threading: a context is not thread-safe; use one context per host thread. Calls on
 * a context are ordered on the context's CUDA stream.
 */
#ifndef RTNN_H_
#define RTNN_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rtnn_status {
  RTNN_OK = 0,
  RTNN_ERR_INVALID_ARGUMENT = 1,  /* bad pointer, size, radius or flag combination */
  RTNN_ERR_CUDA = 2,              /* a CUDA runtime call failed */
  RTNN_ERR_OUT_OF_MEMORY = 3,     /* device allocation failed */
  RTNN_ERR_UNSUPPORTED_K = 4,     /* K == 0 or K > RTNN_MAX_K */
  RTNN_ERR_DEVICE_TIMEOUT = 5,    /* a bounded device-side wait gave up */
  RTNN_ERR_NO_DEVICE = 6,         /* no CUDA device, or the device id is out of range */
  RTNN_ERR_NO_MODEL = 7,          /* RTNN_FLAG_LEARNED without a loaded width model */
  RTNN_ERR_INTERNAL = 8           /* a device-side consistency check failed */
} rtnn_status;

typedef enum rtnn_mode {
  RTNN_MODE_RADIUS = 0,           /* -sm radius (util.cpp:220-227) */
  RTNN_MODE_KNN = 1               /* -sm knn */
} rtnn_mode;

/* Largest K any search accepts (the reference bakes K in at compile time,
 * src/optixNSearch/CMakeLists.txt:58-61; here it is a run-time argument up to this). */
#define RTNN_MAX_K 128u

/* Flags for rtnn_search / rtnn_search_batched / rtnn_plan_create. */
#define RTNN_FLAG_DEVICE_POINTERS 0x1u  /* points, queries and out are device pointers */
#define RTNN_FLAG_PARTITION       0x2u  /* density buckets with analytic widths + exact fallback
                                           (replaces the query partitioning of sort.cpp:393-498) */
#define RTNN_FLAG_LEARNED         0x4u  /* density buckets with widths from the loaded MLP + exact
                                           fallback (replaces the analytic heuristic) */
#define RTNN_FLAG_SORTED_ROWS     0x8u  /* sort each output row by (distance, index) */
#define RTNN_FLAG_LOCAL_INDICES   0x10u /* batched: indices relative to the point's own cloud */
#define RTNN_FLAG_ANY_K           0x20u /* any K of the qualifying points (the first found),
                                           not the K nearest: the reference's radius-search
                                           semantics (geometry.cu:72-83), cheaper */
#define RTNN_FLAG_KEEP_ORDER      0x40u /* plans only (time stepping, points that move a little
                                           between executes): the first execute sorts the
                                           queries and keeps that order, later executes reuse it
                                           and skip the query keys and sort (the reference
                                           sorts the queries on every run, sort.cpp:393-498,
                                           751-797); rows stay exact, only tile coherence can
                                           age. See rtnn_plan_resort. */
#define RTNN_FLAG_REF_LAYOUT      0x80u /* rtnn_search / rtnn_search_batched: the output in the
                                           engine's own order, as the reference returns it
                                           (sort.cpp:378-386,612,626; search.cpp:43-53): row j
                                           belongs to the j-th query in the search's sorted
                                           order and every entry is a position in the engine's
                                           cell-sorted copy of the points. rtnn_layout gives the
                                           two permutations that map them back. */

/* Per-call statistics (all optional to read). Times are device times measured with
 * CUDA events on the context stream (graph replays report ms_total only). */
typedef struct rtnn_stats {
  uint64_t n_points;
  uint64_t n_queries;
  uint32_t n_clouds;
  uint32_t n_buckets;        /* distinct width levels used by the partition (1 when plain) */
  uint64_t n_fallback;       /* queries re-searched at the full radius */
  uint64_t n_tiles;          /* 32-query work items of the first search pass */
  uint64_t n_cells;          /* total grid cells over all clouds */
  float cell_size;           /* cell edge of the first cloud */
  uint32_t grid_dims[3];     /* grid dimensions of the first cloud */
  float ms_build;            /* bounds, per-cell counts, scan, scatter (grid build) */
  float ms_partition;        /* per-query widths and the query sort into buckets */
  float ms_search;           /* every search pass and the output write */
  float ms_total;            /* device time of the whole call (copies excluded) */
  uint32_t n_launches;       /* kernels of this library launched by the call */
  float ms_fallback;         /* the part of ms_search spent after the first pass */
  uint64_t n_loaded;         /* candidate points streamed from HBM/L2 by all search passes */
  uint64_t n_tested;         /* candidates distance-tested (each against 32 queries) */
} rtnn_stats;

typedef struct rtnn_ctx rtnn_ctx;
typedef struct rtnn_plan rtnn_plan;

/* Creates a context on CUDA device `device` (replaces setDevice, main.cpp:9-24).
 * The context owns one CUDA stream and a grow-only cache of device buffers. */
rtnn_status rtnn_create(rtnn_ctx** ctx, int device);

/* Frees every device buffer of the context (replaces cleanupState, optix.cpp:628-677). */
rtnn_status rtnn_destroy(rtnn_ctx* ctx);

/* Message of the last failed call on this context ("" when none). */
const char* rtnn_last_error(const rtnn_ctx* ctx);

/* Makes the context issue its work on `stream` (a cudaStream_t); NULL restores the
 * context's own stream. */
rtnn_status rtnn_set_stream(rtnn_ctx* ctx, void* stream);

/* Returns 1 when `k` is accepted by the searches, else 0. */
int rtnn_k_supported(uint32_t k);

/* Returns 1 when the searches have kernels with this K compiled in (the reference compiles
 * its one K into each build, src/optixNSearch/CMakeLists.txt:58-61, camera.cu:66-72; here a
 * fixed set: 5, 8, 16, 32, 50 and 64), else 0. Other K up to RTNN_MAX_K run kernels that
 * take K at run time, with the same results. */
int rtnn_k_compiled(uint32_t k);

/* Version string of the library. */
const char* rtnn_version(void);

/* One fixed-radius or KNN search of `n_queries` queries against `n_points` points.
 * Replaces the whole timed region of optixNSearch (main.cpp:91-148: sortParticles,
 * createGeometry, gasSortSearch, search) for `-f points -q queries -sm mode -r radius
 * -k k`. `queries` may be NULL: the points are then also the queries (util.cpp:371).
 * points/queries: xyz float triples (12 bytes each, AoS as read by util.cpp:101-135).
 * out: n_queries * k int32. Host pointers unless RTNN_FLAG_DEVICE_POINTERS. */
rtnn_status rtnn_search(rtnn_ctx* ctx,
                        const float* points, uint64_t n_points,
                        const float* queries, uint64_t n_queries,
                        rtnn_mode mode, float radius, uint32_t k, uint32_t flags,
                        int32_t* out, rtnn_stats* stats);

/* Many independent point clouds searched in one persistent launch (no counterpart in
 * the reference, which searches one cloud per process). Cloud c owns points
 * [point_offsets[c], point_offsets[c+1]) and queries [query_offsets[c],
 * query_offsets[c+1]); queries == NULL means every cloud's points are its queries.
 * point_offsets / query_offsets are HOST arrays of n_clouds + 1 entries. Row q of out
 * holds neighbors of query q from the query's own cloud only. */
rtnn_status rtnn_search_batched(rtnn_ctx* ctx,
                                const float* points, const uint64_t* point_offsets,
                                uint32_t n_clouds,
                                const float* queries, const uint64_t* query_offsets,
                                rtnn_mode mode, float radius, uint32_t k, uint32_t flags,
                                int32_t* out, rtnn_stats* stats);

/* A plan fixes the shapes of a (batched) search so that grid build and search can be
 * captured once in a CUDA graph and replayed on new point data of the same shape.
 * Device pointers only. use_graph = 0 issues the kernels directly on every execute. */
rtnn_status rtnn_plan_create(rtnn_ctx* ctx, rtnn_plan** plan,
                             const uint64_t* point_offsets, uint32_t n_clouds,
                             const uint64_t* query_offsets, /* NULL: queries are points */
                             rtnn_mode mode, float radius, uint32_t k, uint32_t flags,
                             int use_graph);
rtnn_status rtnn_plan_execute(rtnn_plan* plan, const float* d_points, const float* d_queries,
                              int32_t* d_out, rtnn_stats* stats);
rtnn_status rtnn_plan_destroy(rtnn_plan* plan);
/* RTNN_FLAG_KEEP_ORDER plans: the next execute sorts the queries again (for example every
 * few time steps, or after the points moved far) and keeps the new order. */
rtnn_status rtnn_plan_resort(rtnn_plan* plan);

/* Search-tuning knobs chosen by the autotuner (rtnn_b200/autotune.py caches them). */
typedef struct rtnn_tuning {
  float cell_ratio;       /* largest cell edge = radius * cell_ratio
                             (the reference's cellSize = radius / crRatio, sort.cpp:80) */
  float min_cell_ratio;   /* smallest cell edge = radius * min_cell_ratio */
  float points_per_cell;  /* > 0: a cloud's cell edge shrinks (down to the smallest) until
                             its bounding box holds about this many points per cell */
  float cell_budget;      /* max grid cells per point before the cell edge is grown */
  uint32_t warps_per_block;   /* search kernel block size in warps (1..8) */
  uint32_t blocks_per_sm;     /* persistent search grid = SMs * blocks_per_sm (0: occupancy) */
  float width_margin;     /* learned width = margin * predicted K-th distance */
  uint32_t fallback_passes;   /* partitioned search: passes that retry short queries at a wider
                                 width (grown from the density each saw, 1.15x to 2x) before
                                 the last pass at the full radius (0..6) */
  float lane_walk_ratio;      /* a 32-query tile whose extent exceeds ratio x its search width
                                 is searched lane by lane (each lane walks its own query's
                                 cells) instead of sharing one candidate stream; 0: never */
  float gap_ratio;            /* a tile is split into runs wherever two consecutive queries
                                 (sort order) are farther apart than ratio x its widest search
                                 width, so one candidate box never spans a jump of the Morton
                                 curve; 0: split only between clouds */
  uint32_t pending_slots;     /* per query, shared-memory slots for hits found since the last
                                 merge into its K kept neighbors (8..256); more slots mean
                                 fewer merges and fewer resident warps. Reduced when K +
                                 slots would not fit one warp's shared memory */
  uint32_t query_warps;       /* search kernel: 0: one warp per 32-query tile sharing one
                                 candidate stream (wide widths, coherent queries); 1: one
                                 warp per query -- each query walks only its own candidate
                                 box and keeps its hits with warp-wide sorts (narrow widths);
                                 2: tiles for the first pass, one warp per query for the
                                 escalation passes (scattered short queries); 3: the lane
                                 walk for the first pass -- each lane of a 32-query tile
                                 walks only the cells of its own query's box (dense clouds,
                                 narrow per-query widths) -- and one warp per query for the
                                 escalation passes; 4: the lane walk in every pass. K <= 64
                                 for the per-query kernel; larger K use the tiles there */
  float buckets_per_halving;  /* partitioned search: density buckets (sort-key levels) per
                                 halving of the search width (0..8; 0: all narrowed widths
                                 in one bucket). Fewer buckets keep tiles spatially tighter,
                                 more keep a tile's widths alike */
  uint32_t width_model;       /* RTNN_FLAG_LEARNED: 0: a width per query from the model before
                                 the query sort, queries bucketed by width (one more pass,
                                 tight boxes); 1: a width per 32-query tile, evaluated by the
                                 search kernel itself (no extra pass, one box per tile); 2:
                                 the widths are off -- a learned search takes every query at
                                 the full radius, exactly as the plain search does (the
                                 autotuner's choice where narrowed widths cannot pay: most
                                 K-th distances at r, or a grid already tight around them).
                                 The model is trained for one kind (rtnn_collect_training
                                 follows this setting; 2 collects per-query samples) */
  uint32_t width_clip;        /* partitioned search, tile walk: in each run of a tile the
                                 `width_clip` widest narrowed widths are clipped to the next
                                 widest, so one outlier does not grow the shared candidate box;
                                 a clipped query that finds fewer than K is escalated like any
                                 short one, so rows stay exact (0..16; 0: no clipping) */
} rtnn_tuning;

rtnn_status rtnn_get_tuning(const rtnn_ctx* ctx, rtnn_tuning* tuning);
rtnn_status rtnn_set_tuning(rtnn_ctx* ctx, const rtnn_tuning* tuning);

/* The order of the last successful rtnn_search / rtnn_search_batched on this context (the
 * reference keeps the same two orders: its points sorted in place, sort.cpp:612,626, and
 * the per-partition query arrays h_actQs, sort.cpp:378-386). point_order[i] = caller index
 * of the i-th point of the cell-sorted copy; query_order[j] = caller index of the query of
 * the j-th row in RTNN_FLAG_REF_LAYOUT output. So a reference-layout row j maps back as
 * caller_row[query_order[j]][s] = point_order[row[j][s]] (-1 stays -1). Either pointer may
 * be NULL; n_points / n_queries must equal the last search's. Host buffers unless flags
 * holds RTNN_FLAG_DEVICE_POINTERS. Unavailable after a host-buffer batch that ran in
 * sub-batches (a large result without RTNN_FLAG_REF_LAYOUT). */
rtnn_status rtnn_layout(rtnn_ctx* ctx, uint32_t* point_order, uint64_t n_points,
                        uint32_t* query_order, uint64_t n_queries, uint32_t flags);

/* The library's LSD radix sort on its own (replaces thrust::sort_by_key,
 * src/optixNSearch/thrust_helper.cu:13-43, which the reference calls at sort.cpp:415,
 * 487-488 and 612; here it orders the queries). Sorts n (key, value) pairs in place on the
 * device by the low key_bits bits of each key, stably (equal keys keep their input order).
 * d_keys: n keys of key_bytes (4 or 8) bytes; d_values: n uint32 values moved with their
 * keys. Device pointers, ordered on the context's stream; returns when done. */
rtnn_status rtnn_sort_pairs(rtnn_ctx* ctx, void* d_keys, uint32_t key_bytes, uint32_t* d_values,
                            uint64_t n, uint32_t key_bits);

/* Failure-detection self-test (no counterpart in the reference, which has no device-side
 * waits): runs the decoupled look-back scan with a predecessor tile that is never
 * published, so its bounded wait (about a second) gives up. Returns
 * RTNN_ERR_DEVICE_TIMEOUT when the limit works -- the expected result -- and leaves the
 * context usable; any other status means the wait did not report. */
rtnn_status rtnn_selftest_wait_timeout(rtnn_ctx* ctx);

/* Search for callers that cannot allocate device memory. It has no counterpart in the
 * reference. For hosts that own all device memory through
 * their own pool, real-time loops that cannot afford cudaMalloc's implicit synchronisation,
 * and code running while a CUDA graph is captured in global mode: this call makes no
 * cudaMalloc, cudaFree or other allocation, and needs no context.
 * Plain (unpartitioned) radius or KNN search, the same rows as rtnn_search with flags 0.
 * Device pointers only; `stream` is a cudaStream_t (NULL: the legacy default stream); the
 * call returns after the search has finished. While another thread captures a CUDA graph
 * in global mode, pass a stream created with cudaStreamNonBlocking: the legacy default
 * stream waits on every blocking stream, so work on it would break that capture.
 * d_queries == NULL searches the points themselves: n_queries is then ignored and the
 * output has n_points rows. Its scratch is one fixed array of
 * RTNN_NOALLOC_SCRATCH_BYTES in device memory, held by every GPU that loads the library
 * until the process exits, and shared by all calls: calls whose work overlaps on the GPU
 * race and must be serialised by the caller. Limits: at most RTNN_NOALLOC_MAX_POINTS points
 * and RTNN_NOALLOC_MAX_QUERIES queries (RTNN_ERR_INVALID_ARGUMENT otherwise). The first call
 * on a device looks up the array's device address, page-locks a small status block that
 * is part of the library and caches launch shapes, and should come before any stream
 * capture; these are kept for the life of the process, so cudaDeviceReset after the first
 * call on a device is not supported. Later calls do not synchronise the stream: the last
 * kernel writes the call's status to that block and the call waits for it (at most a
 * minute, then RTNN_ERR_DEVICE_TIMEOUT). errbuf (optional, errlen bytes) receives a
 * message when the call fails. */
#define RTNN_NOALLOC_SCRATCH_BYTES (16u << 20)
#define RTNN_NOALLOC_MAX_POINTS (1u << 18)
#define RTNN_NOALLOC_MAX_QUERIES (1u << 18)
rtnn_status rtnn_search_noalloc(const float* d_points, uint32_t n_points,
                                const float* d_queries, uint32_t n_queries, rtnn_mode mode,
                                float radius, uint32_t k, int32_t* d_out, void* stream,
                                char* errbuf, size_t errlen);

#ifdef __cplusplus
}
#endif

#endif /* RTNN_H_ */
