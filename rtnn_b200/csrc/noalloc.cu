// noalloc.cu -- the one search entry point that allocates no memory.
//
// Some callers cannot call cudaMalloc once they are running: hosts that hand out all
// device memory through their own pool and forbid allocations behind its back, real-time
// loops where cudaMalloc's implicit device synchronisation and unbounded latency are not
// acceptable, and code that runs while another thread captures a CUDA graph in global
// capture mode (where cudaMalloc is prohibited). rtnn_search_noalloc serves them: the
// caller passes device inputs and a device output, and every scratch buffer of the
// search (grid cells, ranks, cell-sorted points, sort keys, sorted queries, scan state,
// counters) is carved from one file-scope __device__ array of fixed size.
//
// That array is held by every GPU that loads the library until the process exits. It is
// shared by all calls and keeps the last call's contents, so this code clears everything
// that must start at zero on each call, and calls whose work overlaps on the GPU (two
// streams, or two host threads) race on it and must be serialised by the caller.
// In host code the array's name is only a host-side stand-in: its device address is
// looked up with cudaGetSymbolAddress once per device (with that device current) on the
// first call made on that device, which is why that first call should come before any
// stream capture begins. That first call also page-locks a small static status block in
// host memory (no allocation: the block is part of the library) and caches the search
// kernels' launch shapes, so that later calls make no call that synchronises the device or
// could join another thread's capture: the call enqueues its kernels and a last one that
// writes the device status and a sequence number into the mapped status block, and the
// host waits for that number (for at most a minute) instead of synchronising the stream.
// The addresses are cached for the life of the process, so a cudaDeviceReset after the
// first call on a device is not supported. Beside a global-mode capture on another thread
// the caller passes a non-blocking stream: the legacy default stream would wait on the
// capturing stream and break its capture.
#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>
#include <thread>

#include "../../include/rtnn.h"
#include "kernels.h"

using namespace rtnn;

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[RTNN_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};

// Completion status of the last call on each device, written by the device through the
// mapped (page-locked) host block: error and error_info, then seq.
struct alignas(64) NoallocStatus {
  volatile uint32_t seq;
  volatile uint32_t error;
  volatile uint32_t error_info;
  uint32_t pad[13];
};
alignas(4096) NoallocStatus g_status[kMaxDevices];   // one page
bool g_status_pinned = false;
NoallocStatus* g_status_dev[kMaxDevices] = {};   // device view of g_status[dev]
uint32_t g_seq[kMaxDevices] = {};
// search blocks per SM for every K (index k - 1) and mode, cached at set-up
int g_bps[kMaxDevices][2][RTNN_MAX_K] = {};
constexpr double kWaitSeconds = 60.0;

__global__ void k_noalloc_publish(const Counters* ctr, NoallocStatus* st, uint32_t seq) {
  st->error = ctr ? ctr->error : 0u;
  st->error_info = ctr ? ctr->error_info : 0u;
  __threadfence_system();
  st->seq = seq;
}

// Enqueues the status write and waits (bounded) for it to arrive in host memory.
cudaError_t publish_and_wait(int dev, const Counters* ctr, cudaStream_t s, bool* timed_out) {
  *timed_out = false;
  const uint32_t seq = ++g_seq[dev];
  k_noalloc_publish<<<1, 1, 0, s>>>(ctr, g_status_dev[dev], seq);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const auto t0 = std::chrono::steady_clock::now();
  while (g_status[dev].seq != seq) {
    std::this_thread::yield();
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > kWaitSeconds) {
      // a kernel that faulted never lets the status through: report its error if it did
      const cudaError_t q = cudaStreamQuery(s);
      if (q != cudaSuccess && q != cudaErrorNotReady) return q;
      *timed_out = true;
      return cudaSuccess;
    }
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  return cudaSuccess;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

void set_msg(char* buf, size_t len, const char* msg) {
  if (buf && len) {
    std::strncpy(buf, msg, len - 1);
    buf[len - 1] = '\0';
  }
}

}  // namespace

extern "C" rtnn_status rtnn_search_noalloc(const float* d_points, uint32_t n_points,
                                           const float* d_queries, uint32_t n_queries,
                                           rtnn_mode mode, float radius, uint32_t k,
                                           int32_t* d_out, void* stream, char* errbuf,
                                           size_t errlen) {
  set_msg(errbuf, errlen, "");
  if (d_queries == nullptr) n_queries = n_points;
  if (mode != RTNN_MODE_RADIUS && mode != RTNN_MODE_KNN) {
    set_msg(errbuf, errlen, "mode must be RTNN_MODE_RADIUS or RTNN_MODE_KNN");
    return RTNN_ERR_INVALID_ARGUMENT;
  }
  if (!(radius >= 1e-30f && radius < 3.0e38f)) {
    set_msg(errbuf, errlen, "radius must be a finite number > 0");
    return RTNN_ERR_INVALID_ARGUMENT;
  }
  if (k < 1 || k > RTNN_MAX_K) {
    set_msg(errbuf, errlen, "k must be in [1, RTNN_MAX_K]");
    return RTNN_ERR_UNSUPPORTED_K;
  }
  if (n_points > RTNN_NOALLOC_MAX_POINTS || n_queries > RTNN_NOALLOC_MAX_QUERIES) {
    set_msg(errbuf, errlen,
            "rtnn_search_noalloc: more than RTNN_NOALLOC_MAX_POINTS points or "
            "RTNN_NOALLOC_MAX_QUERIES queries; use rtnn_search");
    return RTNN_ERR_INVALID_ARGUMENT;
  }
  if ((n_points > 0 && !d_points) || (n_queries > 0 && !d_out)) {
    set_msg(errbuf, errlen, "NULL device pointer");
    return RTNN_ERR_INVALID_ARGUMENT;
  }
  if (n_queries == 0) return RTNN_OK;
  cudaStream_t s = (cudaStream_t)stream;

  // set-up, once per device: the scratch array's device address, SM count, kernel
  // attributes, the page-locked status block and the search kernels' launch shapes
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    set_msg(errbuf, errlen, "no current CUDA device");
    return RTNN_ERR_NO_DEVICE;
  }
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
      void* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev);
      if (e == cudaSuccess) e = search_prepare(dev);
      if (e == cudaSuccess && !g_status_pinned) {
        e = cudaHostRegister(g_status, sizeof(g_status),
                             cudaHostRegisterPortable | cudaHostRegisterMapped);
        if (e == cudaSuccess) g_status_pinned = true;
      }
      if (e == cudaSuccess) {
        void* dp = nullptr;
        e = cudaHostGetDevicePointer(&dp, &g_status[dev], 0);
        g_status_dev[dev] = (NoallocStatus*)dp;
      }
      for (int knn = 0; knn < 2 && e == cudaSuccess; ++knn)
        for (uint32_t kk = 1; kk <= RTNN_MAX_K; ++kk) {
          uint32_t pend = 16;
          int wpb = 4;
          fit_search_shape(kk, 16u, 4, &pend, &wpb);
          g_bps[dev][knn][kk - 1] = search_blocks_per_sm(knn != 0, kk, pend, wpb, false);
        }
      if (e != cudaSuccess || !ptr) {
        cudaGetLastError();
        set_msg(errbuf, errlen, e != cudaSuccess ? cudaGetErrorString(e) : "scratch address is NULL");
        return RTNN_ERR_CUDA;
      }
      g_scratch_ptr[dev] = ptr;
    }
    base = (unsigned char*)g_scratch_ptr[dev];
  }
  const int n_sms = g_sms[dev];
  bool timed_out = false;
  if (n_points == 0) {
    cudaError_t e = cudaMemsetAsync(d_out, 0xff, (size_t)n_queries * k * 4, s);
    if (e == cudaSuccess) e = publish_and_wait(dev, nullptr, s, &timed_out);
    if (e != cudaSuccess) { set_msg(errbuf, errlen, cudaGetErrorString(e)); return RTNN_ERR_CUDA; }
    if (timed_out) {
      set_msg(errbuf, errlen, "rtnn_search_noalloc: the device did not finish within a minute");
      return RTNN_ERR_DEVICE_TIMEOUT;
    }
    return RTNN_OK;
  }

  // fixed tuning: cell = r/2, at most 2 cells per point (+64), plain (no partition)
  const uint64_t N = n_points, Q = n_queries;
  const float cell_budget = 2.0f;
  const uint64_t cap = (uint64_t)(cell_budget * (double)N) + 64 + 64;
  uint32_t mb = 1;
  while (mb < 10 && (1ull << (3 * mb)) < Q) ++mb;
  const uint32_t key_bits = 3 * mb < 8 ? 8 : 3 * mb;
  const uint32_t rt = radix_tiles_for(Q);
  const uint64_t scan_n = (cap + 1 > 256ull * rt) ? cap + 1 : 256ull * rt;
  size_t off = 0;
  auto carve = [&](size_t bytes) { const size_t o = off; off += align256(bytes); return base + o; };
  Counters* ctr = (Counters*)carve(sizeof(Counters));
  uint32_t* tables = (uint32_t*)carve(12 * 4);
  CloudGrid* grids = (CloudGrid*)carve(sizeof(CloudGrid));
  uint32_t* bbox = (uint32_t*)carve(6 * 4);
  uint32_t* cells = (uint32_t*)carve((cap + 1) * 4);
  uint32_t* rank = (uint32_t*)carve(N * 4);
  float4* spts = (float4*)carve(N * 16);
  void* keys0 = carve(Q * 4);
  void* keys1 = carve(Q * 4);
  uint32_t* vals0 = (uint32_t*)carve(Q * 4);
  uint32_t* vals1 = (uint32_t*)carve(Q * 4);
  float4* sq = (float4*)carve(Q * 16);
  uint32_t* hist = (uint32_t*)carve(256ull * rt * 4);
  uint64_t* scan_state = (uint64_t*)carve(scan_tiles_for(scan_n) * 8);
  if (off > RTNN_NOALLOC_SCRATCH_BYTES) {
    set_msg(errbuf, errlen, "rtnn_search_noalloc: scratch layout exceeds RTNN_NOALLOC_SCRATCH_BYTES");
    return RTNN_ERR_INTERNAL;
  }

  const float* d_qs = d_queries ? d_queries : d_points;
  const bool ap = ((uintptr_t)d_points % 16) == 0, aq = ((uintptr_t)d_qs % 16) == 0;
  const uint32_t n_chunks = (uint32_t)((N + kChunk - 1) / kChunk);
  const uint32_t n_qchunks = (uint32_t)((Q + kChunk - 1) / kChunk);
  const uint32_t n_tiles = (uint32_t)((Q + kTile - 1) / kTile);
  CloudTables t;
  t.point_off = tables;
  t.query_off = tables + 2;
  t.chunk_base = tables + 4;
  t.qchunk_base = tables + 6;
  t.tile_base = tables + 8;
  t.lead_base = tables + 10;
  t.n_clouds = 1;
  const bool knn = mode == RTNN_MODE_KNN;
  bool in1 = false;
  cudaError_t e = cudaMemsetAsync(ctr, 0, sizeof(Counters), s);
  if (e == cudaSuccess) e = launch_single_tables(tables, (uint32_t)N, (uint32_t)Q, s);
  if (e == cudaSuccess) e = launch_bbox(d_points, N, ap, t, n_chunks, bbox, n_sms, s);
  if (e == cudaSuccess)
    e = launch_grid_plan(t, bbox, radius, 0.5f, 0.0625f, 0.f, cell_budget, mb, cap, grids, ctr, s);
  if (e == cudaSuccess) e = launch_zero_cells(cells, ctr, n_sms, s);
  if (e == cudaSuccess) e = launch_count(d_points, N, ap, t, n_chunks, grids, cells, rank, ctr, s);
  if (e == cudaSuccess)
    e = launch_scan_excl(cells, 0, &ctr->total_cells, 1, cap + 1, scan_state, &ctr->scan_tiles[0], ctr, s);
  if (e == cudaSuccess) e = launch_scatter(d_points, N, ap, t, n_chunks, grids, cells, rank, spts, ctr, s);
  if (e == cudaSuccess)
    e = launch_query_keys(d_qs, Q, aq, t, n_qchunks, grids, mb, nullptr, radius, 0, 0.f, false,
                          keys0, s);
  if (e == cudaSuccess)
    e = radix_sort_pairs(false, keys0, vals0, keys1, vals1, (uint32_t)Q, key_bits, true, hist,
                         scan_state, &ctr->scan_tiles[1], ctr, &in1, s);
  if (e == cudaSuccess)
    e = launch_gather_queries(d_qs, in1 ? vals1 : vals0, (uint32_t)Q, sq, nullptr, nullptr, n_sms, s);
  if (e == cudaSuccess) {
    SearchArgs a{};
    a.t = t;
    a.grids = grids;
    a.cells = cells;
    a.spts = spts;
    a.sq = sq;
    a.out = d_out;
    a.ctr = ctr;
    a.work = &ctr->work[0];
    a.n_tiles = n_tiles;
    a.radius = radius;
    a.r2 = radius * radius;
    a.k = k;
    a.pass = kPassMain;
    int wpb = 4;
    fit_search_shape(k, 16u, 4, &a.pending, &wpb);
    const uint64_t blocks = (uint64_t)n_sms * g_bps[dev][knn ? 1 : 0][k - 1];
    const uint64_t need = (n_tiles + wpb - 1) / wpb;
    e = launch_search(knn, a, (unsigned)(blocks < need ? blocks : need), wpb, false, s);
  }
  if (e == cudaSuccess) e = publish_and_wait(dev, ctr, s, &timed_out);
  if (e != cudaSuccess) {
    set_msg(errbuf, errlen, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? RTNN_ERR_OUT_OF_MEMORY : RTNN_ERR_CUDA;
  }
  if (timed_out) {
    set_msg(errbuf, errlen, "rtnn_search_noalloc: the device did not finish within a minute");
    return RTNN_ERR_DEVICE_TIMEOUT;
  }
  const uint32_t error = g_status[dev].error;
  if (error == kErrScanTimeout) {
    set_msg(errbuf, errlen, "scan look-back gave up waiting");
    return RTNN_ERR_DEVICE_TIMEOUT;
  }
  if (error != 0) {
    set_msg(errbuf, errlen, "device consistency check failed");
    return RTNN_ERR_INTERNAL;
  }
  return RTNN_OK;
}
