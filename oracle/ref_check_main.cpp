// ref_check_main.cpp -- runs the reference's own host-side check (check.cpp, compiled
// from the reference sources by oracle/Makefile) on a result buffer written to disk.
// TEST INFRASTRUCTURE ONLY.
//
//   refcheck POINTS QUERIES|- ROWS radius|knn R K [Q_BEGIN Q_END]
//
// POINTS / QUERIES: raw float32 xyz triples; ROWS: raw int32 [Q][K] (-1 == UINT_MAX).
// radius: sanityCheckRadius (check.cpp:103-139) over every query; it exits 1 on the
// first neighbor farther than R. knn: sanityCheckKNN (check.cpp:20-101) once per query
// in [Q_BEGIN, Q_END), each time with a one-query view so that its random pick
// (rand() % numQueries, check.cpp:23) is that query; it exits 1 when the set of
// neighbor distances differs from its brute-force priority queue.
// Prints "REFCHECK OK" and exits 0 when every check passed.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include "state.h"

void sanityCheckKNN(RTNNState& state, int batch_id);
void sanityCheckRadius(RTNNState& state, int batch_id);

static std::vector<char> slurp(const char* path) {
  std::vector<char> buf;
  FILE* f = std::fopen(path, "rb");
  if (!f) { std::fprintf(stderr, "cannot open %s\n", path); std::exit(2); }
  char tmp[1 << 16];
  size_t n;
  while ((n = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + n);
  std::fclose(f);
  return buf;
}

int main(int argc, char** argv) {
  if (argc < 7) {
    std::fprintf(stderr, "usage: %s POINTS QUERIES|- ROWS radius|knn R K [Q_BEGIN Q_END]\n", argv[0]);
    return 2;
  }
  std::vector<char> pb = slurp(argv[1]);
  std::vector<char> qb = std::string(argv[2]) == "-" ? pb : slurp(argv[2]);
  std::vector<char> rb = slurp(argv[3]);
  const std::string mode = argv[4];
  const float r = std::strtof(argv[5], nullptr);
  const unsigned k = (unsigned)std::strtoul(argv[6], nullptr, 10);
  const unsigned np = (unsigned)(pb.size() / sizeof(float3));
  const unsigned nq = (unsigned)(qb.size() / sizeof(float3));
  if (rb.size() != (size_t)nq * k * 4) { std::fprintf(stderr, "ROWS size mismatch\n"); return 2; }
  float3* pts = reinterpret_cast<float3*>(pb.data());
  float3* qs = reinterpret_cast<float3*>(qb.data());
  unsigned* rows = reinterpret_cast<unsigned*>(rb.data());

  RTNNState st;
  st.h_points = pts;
  st.numPoints = np;
  st.gRadius = r;
  st.radius = r;
  st.knn = k;
  st.searchMode = mode;
  void* res[1];
  st.h_res = res;
  if (mode == "radius") {
    st.h_queries = qs;
    st.numQueries = nq;
    res[0] = rows;
    sanityCheckRadius(st, 0);
  } else if (mode == "knn") {
    unsigned q0 = 0, q1 = nq;
    if (argc >= 9) {
      q0 = (unsigned)std::strtoul(argv[7], nullptr, 10);
      q1 = (unsigned)std::strtoul(argv[8], nullptr, 10);
      if (q1 > nq) q1 = nq;
    }
    for (unsigned q = q0; q < q1; ++q) {
      st.h_queries = qs + q;
      st.numQueries = 1;
      res[0] = rows + (size_t)q * k;
      sanityCheckKNN(st, 0);
    }
  } else {
    std::fprintf(stderr, "mode must be radius or knn\n");
    return 2;
  }
  std::printf("REFCHECK OK\n");
  return 0;
}
