/*
 * oracle.c -- CPU restatement of the reference's neighbor-search semantics.
 *
 * TEST INFRASTRUCTURE ONLY: the parity tests, __graft_entry__.smoke() and the CPU
 * baseline of bench.py call this library to check results. The product (librtnn_b200.so)
 * never links or calls it.
 *
 * Semantics restated (paths relative to the reference project):
 *  - squared distance: dot(q - p, q - p) = dx*dx + dy*dy + dz*dz, left to right, each
 *    operation rounded to FP32 (src/sutil/vec_math.h:527-530; src/optixNSearch/check.cpp:36-37,
 *    117-118). Built with -ffp-contract=off so no FMA is formed.
 *  - radius search: a point is a neighbor when d < r*r (r*r rounded to FP32), the query
 *    itself included (geometry.cu:61-66, check.cpp:119).
 *  - KNN: a point is a candidate when 0 < d < r*r (geometry.cu:187, check.cpp:38), and
 *    the K smallest are kept (check.cpp:39-46 keeps a max-heap of K; equal distances keep
 *    the earlier index there, which is the (distance, index) order used here).
 *  - more than K radius neighbors: the K smallest by (distance, index) are returned
 *    (the reference returns the first K in traversal order, geometry.cu:72-83; the
 *    rebuilt library returns the nearest K, which its own reference check accepts).
 *  - output: row q holds the neighbors sorted by (distance, index), -1 after the last
 *    (UINT_MAX fill, search.cpp:18).
 * Pinned against the reference's own check.cpp (compiled from the reference sources by
 * oracle/Makefile into oracle/_ref/refcheck) and against the FP64 brute force below.
 */
#include <math.h>
#include <stdio.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static inline float d2_ref(const float* q, const float* p) {
  const float dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
  const float s = dx * dx + dy * dy;   /* (dx*dx + dy*dy) rounded, then + dz*dz */
  return s + dz * dz;
}

static inline uint64_t key_of(float d, uint32_t idx) {
  uint32_t b;
  memcpy(&b, &d, 4);
  return ((uint64_t)b << 32) | idx;
}

static int cmp_u64(const void* a, const void* b) {
  uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return (x > y) - (x < y);
}

typedef struct {
  uint64_t* v;
  size_t n, cap;
} KeyVec;

static int kv_push(KeyVec* kv, uint64_t x) {
  if (kv->n == kv->cap) {
    size_t nc = kv->cap ? 2 * kv->cap : 256;
    uint64_t* nv = (uint64_t*)realloc(kv->v, nc * sizeof(uint64_t));
    if (!nv) return -1;
    kv->v = nv;
    kv->cap = nc;
  }
  kv->v[kv->n++] = x;
  return 0;
}

static inline int accept(float d, float r2, int knn) {
  return knn ? (d > 0.0f && d < r2) : (d < r2);
}

static void write_row(KeyVec* kv, uint32_t k, int32_t* row, uint32_t idx_base) {
  qsort(kv->v, kv->n, sizeof(uint64_t), cmp_u64);
  for (uint32_t j = 0; j < k; ++j)
    row[j] = (j < kv->n) ? (int32_t)((uint32_t)kv->v[j] - idx_base) : -1;
}

/* O(N*Q) brute force. mode 0 = radius, 1 = knn. Returns 0 on success. */
int oracle_bruteforce(const float* pts, uint64_t n, const float* qs, uint64_t nq, int mode,
                      float r, uint32_t k, int32_t* out, int threads) {
  const float r2 = r * r;
  int err = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
#endif
  {
    KeyVec kv = {0, 0, 0};
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
      kv.n = 0;
      for (uint64_t p = 0; p < n; ++p) {
        const float d = d2_ref(qs + 3 * q, pts + 3 * p);
        if (accept(d, r2, mode)) {
          if (kv_push(&kv, key_of(d, (uint32_t)p))) err = 1;
        }
      }
      write_row(&kv, k, out + (uint64_t)q * k, 0);
    }
    free(kv.v);
  }
  return err;
}

/* Uniform-grid exact search (same results as the brute force, fast enough for 1e7).
 * idx_base is subtracted from written indices (for per-cloud local indices). */
static int grid_search_range(const float* pts, uint64_t n, const float* qs, uint64_t nq,
                             int mode, float r, uint32_t k, int32_t* out, uint32_t idx_offset,
                             int local) {
  const float r2 = r * r;
  if (n == 0) {
    for (uint64_t i = 0; i < nq * k; ++i) out[i] = -1;
    return 0;
  }
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint64_t p = 0; p < n; ++p)
    for (int a = 0; a < 3; ++a) {
      const float v = pts[3 * p + a];
      if (isfinite(v)) {
        if (v < mn[a]) mn[a] = v;
        if (v > mx[a]) mx[a] = v;
      }
    }
  for (int a = 0; a < 3; ++a)
    if (!(mn[a] <= mx[a])) { mn[a] = 0; mx[a] = 0; }
  double cell = r;
  int64_t d[3];
  for (;;) {
    double tot = 1;
    for (int a = 0; a < 3; ++a) {
      d[a] = (int64_t)floor((mx[a] - mn[a]) / cell) + 1;
      tot *= (double)d[a];
    }
    if (tot <= 4.0 * (double)n + 64) break;
    cell *= 1.3;
  }
  const uint64_t ncell = (uint64_t)(d[0] * d[1] * d[2]);
  uint32_t* start = (uint32_t*)calloc(ncell + 1, sizeof(uint32_t));
  uint32_t* order = (uint32_t*)malloc(n * sizeof(uint32_t));
  uint64_t* pc = (uint64_t*)malloc(n * sizeof(uint64_t));
  if (!start || !order || !pc) { free(start); free(order); free(pc); return 1; }
  for (uint64_t p = 0; p < n; ++p) {
    int64_t c[3];
    for (int a = 0; a < 3; ++a) {
      double f = floor(((double)pts[3 * p + a] - mn[a]) / cell);
      if (!(f >= 0)) f = 0;
      if (f > (double)(d[a] - 1)) f = (double)(d[a] - 1);
      c[a] = (int64_t)f;
    }
    pc[p] = (uint64_t)((c[2] * d[1] + c[1]) * d[0] + c[0]);
    start[pc[p] + 1]++;
  }
  for (uint64_t i = 0; i < ncell; ++i) start[i + 1] += start[i];
  {
    uint32_t* fill = (uint32_t*)malloc(ncell * sizeof(uint32_t));
    if (!fill) { free(start); free(order); free(pc); return 1; }
    memcpy(fill, start, ncell * sizeof(uint32_t));
    for (uint64_t p = 0; p < n; ++p) order[fill[pc[p]]++] = (uint32_t)p;
    free(fill);
  }
  free(pc);
  const double rr = (double)r * (1.0 + 1e-5);
  int err = 0;
#ifdef _OPENMP
#pragma omp parallel
#endif
  {
    KeyVec kv = {0, 0, 0};
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 256)
#endif
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
      kv.n = 0;
      const float* qq = qs + 3 * q;
      int64_t lo[3], hi[3];
      int empty = !(isfinite(qq[0]) && isfinite(qq[1]) && isfinite(qq[2]));
      for (int a = 0; a < 3 && !empty; ++a) {
        double fl = floor(((double)qq[a] - rr - mn[a]) / cell);
        double fh = floor(((double)qq[a] + rr - mn[a]) / cell);
        if (fh < 0 || fl > (double)(d[a] - 1)) empty = 1;
        lo[a] = fl < 0 ? 0 : (int64_t)fl;
        hi[a] = fh > (double)(d[a] - 1) ? d[a] - 1 : (int64_t)fh;
      }
      if (!empty) {
        for (int64_t z = lo[2]; z <= hi[2]; ++z)
          for (int64_t y = lo[1]; y <= hi[1]; ++y) {
            const uint64_t row = (uint64_t)((z * d[1] + y) * d[0]);
            for (uint32_t i = start[row + lo[0]]; i < start[row + hi[0] + 1]; ++i) {
              const uint32_t p = order[i];
              const float dd = d2_ref(qq, pts + 3ull * p);
              if (accept(dd, r2, mode))
                if (kv_push(&kv, key_of(dd, p + idx_offset))) err = 1;
            }
          }
      }
      write_row(&kv, k, out + (uint64_t)q * k, local ? idx_offset : 0);
    }
    free(kv.v);
  }
  free(start);
  free(order);
  return err;
}

int oracle_grid_search(const float* pts, uint64_t n, const float* qs, uint64_t nq, int mode,
                       float r, uint32_t k, int32_t* out, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  return grid_search_range(pts, n, qs, nq, mode, r, k, out, 0, 0);
}

/* Many clouds: cloud c's queries see only cloud c's points. Offsets have n_clouds+1
 * entries; qs == NULL means each cloud's points are its queries. Indices are global
 * (into pts) unless local != 0. */
int oracle_grid_search_batched(const float* pts, const uint64_t* point_off, uint32_t n_clouds,
                               const float* qs, const uint64_t* query_off, int mode, float r,
                               uint32_t k, int local, int32_t* out, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  const uint64_t* qo = qs ? query_off : point_off;
  const float* qb = qs ? qs : pts;
  for (uint32_t c = 0; c < n_clouds; ++c) {
    const uint64_t p0 = point_off[c], p1 = point_off[c + 1], q0 = qo[c], q1 = qo[c + 1];
    int e = grid_search_range(pts + 3 * p0, p1 - p0, qb + 3 * q0, q1 - q0, mode, r, k,
                              out + q0 * k, (uint32_t)p0, local);
    if (e) return e;
  }
  return 0;
}

/* Pairs (query, point) whose FP32 classification (d32 < fl(r*r)) differs from the FP64
 * one (d64 < r*r with r widened to double): the points within about 1 ulp of r. For
 * KNN, d == 0 pairs are outside in both. Returns the number of pairs found (at most
 * max_pairs are written as [q, p] int64 pairs). */
int64_t oracle_boundary_pairs(const float* pts, uint64_t n, const float* qs, uint64_t nq,
                              int mode, float r, int64_t* pairs, int64_t max_pairs) {
  const float r2 = r * r;
  const double r64 = (double)r;
  int64_t cnt = 0;
  for (uint64_t q = 0; q < nq; ++q)
    for (uint64_t p = 0; p < n; ++p) {
      const float d32 = d2_ref(qs + 3 * q, pts + 3 * p);
      const double dx = (double)qs[3 * q] - pts[3 * p];
      const double dy = (double)qs[3 * q + 1] - pts[3 * p + 1];
      const double dz = (double)qs[3 * q + 2] - pts[3 * p + 2];
      const double d64 = dx * dx + dy * dy + dz * dz;
      const int in32 = accept(d32, r2, mode);
      const int in64 = mode ? (d64 > 0.0 && d64 < r64 * r64) : (d64 < r64 * r64);
      if (in32 != in64) {
        if (cnt < max_pairs) {
          pairs[2 * cnt] = (int64_t)q;
          pairs[2 * cnt + 1] = (int64_t)p;
        }
        ++cnt;
      }
    }
  return cnt;
}

/* FP64 brute force with the same selection rule (distance, index), for comparing the
 * FP32 results against exact arithmetic. */
int oracle_bruteforce_fp64(const float* pts, uint64_t n, const float* qs, uint64_t nq, int mode,
                           float r, uint32_t k, int32_t* out, int threads) {
  const double r2 = (double)r * (double)r;
  int err = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
#endif
  {
    double* dv = NULL;
    uint32_t* iv = NULL;
    size_t cap = 0;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
      size_t m = 0;
      for (uint64_t p = 0; p < n; ++p) {
        const double dx = (double)qs[3 * q] - pts[3 * p];
        const double dy = (double)qs[3 * q + 1] - pts[3 * p + 1];
        const double dz = (double)qs[3 * q + 2] - pts[3 * p + 2];
        const double d = dx * dx + dy * dy + dz * dz;
        const int ok = mode ? (d > 0.0 && d < r2) : (d < r2);
        if (!ok) continue;
        if (m == cap) {
          cap = cap ? 2 * cap : 256;
          dv = (double*)realloc(dv, cap * sizeof(double));
          iv = (uint32_t*)realloc(iv, cap * sizeof(uint32_t));
          if (!dv || !iv) { err = 1; break; }
        }
        dv[m] = d;
        iv[m] = (uint32_t)p;
        ++m;
      }
      /* selection sort of the k smallest by (d, idx) */
      int32_t* row = out + (uint64_t)q * k;
      for (uint32_t j = 0; j < k; ++j) {
        size_t best = m;
        for (size_t i = j; i < m; ++i)
          if (best == m || dv[i] < dv[best] || (dv[i] == dv[best] && iv[i] < iv[best])) best = i;
        if (best == m) { row[j] = -1; continue; }
        double td = dv[j]; dv[j] = dv[best]; dv[best] = td;
        uint32_t ti = iv[j]; iv[j] = iv[best]; iv[best] = ti;
        row[j] = (int32_t)iv[j];
      }
    }
    free(dv);
    free(iv);
  }
  return err;
}

/* Box counts N_s (s = 0..S-1) of the cells around (cx, cy, cz) in a raster grid of
 * per-cell counts (x fastest): the quantity the reference's calcSearchSize grows shell
 * by shell (grid.cu:84-211). */
void oracle_box_counts(const uint32_t* counts, int dx, int dy, int dz, int cx, int cy, int cz,
                       int S, uint32_t* N) {
  for (int s = 0; s < S; ++s) {
    uint32_t t = 0;
    for (int z = cz - s; z <= cz + s; ++z)
      for (int y = cy - s; y <= cy + s; ++y)
        for (int x = cx - s; x <= cx + s; ++x)
          if (x >= 0 && y >= 0 && z >= 0 && x < dx && y < dy && z < dz)
            t += counts[((uint64_t)z * dy + y) * dx + x];
    N[s] = t;
  }
}

/* The reference's shell walk of calcSearchSize (grid.cu:84-211), restated: start from
 * the centre cell; each iteration adds the six faces of the next shell and its eight
 * corners -- the twelve edge lines of the shell are never added -- and stops at the
 * first iteration whose count reaches knn + 1 or whose width (2*iter + 2) * cell
 * (getWidthFromIter, grid.cu:33-44) exceeds max_width. counts: raster, x fastest. */
int oracle_ref_shell_mask(const uint32_t* counts, int dx, int dy, int dz, int cx, int cy, int cz,
                          float cell, float max_width, uint32_t knn) {
#define CNT(x, y, z) (((x) >= 0 && (y) >= 0 && (z) >= 0 && (x) < dx && (y) < dy && (z) < dz) \
                          ? counts[((uint64_t)(z) * dy + (y)) * dx + (x)] : 0u)
  int iter = 0;
  uint32_t count = CNT(cx, cy, cz);
  int x0 = cx, x1 = cx, y0 = cy, y1 = cy, z0 = cz, z1 = cz;
  for (;;) {
    const float width = (float)(iter * 2 + 2) * cell;
    if (width > max_width) return iter;
    if (count >= knn + 1) return iter;
    ++iter;
    for (int x = x0; x <= x1; ++x)
      for (int y = y0; y <= y1; ++y) count += CNT(x, y, z0 - 1) + CNT(x, y, z1 + 1);
    for (int y = y0; y <= y1; ++y)
      for (int z = z0; z <= z1; ++z) count += CNT(x0 - 1, y, z) + CNT(x1 + 1, y, z);
    for (int x = x0; x <= x1; ++x)
      for (int z = z0; z <= z1; ++z) count += CNT(x, y0 - 1, z) + CNT(x, y1 + 1, z);
    --x0; ++x1; --y0; ++y1; --z0; ++z1;
    count += CNT(x0, y0, z0) + CNT(x0, y0, z1) + CNT(x0, y1, z0) + CNT(x0, y1, z1) +
             CNT(x1, y0, z0) + CNT(x1, y0, z1) + CNT(x1, y1, z0) + CNT(x1, y1, z1);
  }
#undef CNT
}

/* Point-cloud text reader as the reference's read_pc_data (src/optixNSearch/util.cpp:
 * 100-135): lines are read into a 1024-byte buffer (std::istream::getline: at most 1023
 * characters; a longer line, or a line of 1023 characters not followed by its '\n',
 * ends the read, and a last line without '\n' still counts), and each line goes through
 * sscanf("%lf,%lf,%lf\n") with the doubles cast to float. A field sscanf does not assign
 * is 0 here (the reference leaves it unset). Writes up to `cap` points into xyz and
 * returns the number of points in the file, or -1 when it cannot be opened. */
int64_t oracle_read_pc(const char* path, float* xyz, uint64_t cap) {
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  char line[1024];
  int64_t n = 0;
  for (;;) {
    size_t len = 0;
    int c, got_delim = 0, any = 0;
    while ((c = fgetc(f)) != EOF) {
      any = 1;
      if (c == '\n') { got_delim = 1; break; }
      if (len == 1023) { len = 1024; break; }  /* getline: n-1 stored, no delimiter */
      line[len++] = (char)c;
    }
    if (len == 1024 || !any) break;          /* failbit: the read ends */
    (void)got_delim;
    line[len] = '\0';
    double x = 0, y = 0, z = 0;
    sscanf(line, "%lf,%lf,%lf\n", &x, &y, &z);
    if ((uint64_t)n < cap) {
      xyz[3 * n + 0] = (float)x;
      xyz[3 * n + 1] = (float)y;
      xyz[3 * n + 2] = (float)z;
    }
    ++n;
  }
  fclose(f);
  return n;
}
