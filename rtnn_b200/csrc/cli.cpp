// cli.cpp -- optixNSearch rebuilt on the C ABI (include/rtnn.h).
//
// Same flags and defaults as the reference executable (src/optixNSearch/util.cpp:137-383):
//   -f/--pfile, -q/--qfile, -sm/--searchmode radius|knn, -r/--radius (2), -k/--knn (50),
//   -d/--device (0), -c/--check (0), -p/--partition (1).
// The reference's OptiX and sorting knobs (-i -m -df -fq -nb -ab -ac -s -ps -qs -cr -gmu
// -egs -g -a -sg -mc -crs) are accepted and ignored with a warning. As in the reference,
// the KNN K is fixed when the binary is built (RTNN_KNN, default 5) and -k only applies to
// radius search (util.cpp:367-369). Input files hold one "x,y,z" point per line, read as
// double and cast to float (util.cpp:101-135).
// Points files ending in .bin or .f32 hold raw float32 x,y,z triples; text files are parsed
// on all host threads (pointio.cpp).
// Extra flags: -o FILE (write the int32 result rows), -lm FILE (learned width model,
// raw float32), --parse-only (print the parsed points' count and checksum and exit),
// --convert FILE (write the parsed points as raw float32 and exit), --threads N (text
// parser threads, 0 = all).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <queue>
#include <random>
#include <set>
#include <string>
#include <vector>

#include "pointio.h"
#include "rtnn.h"
#include "rtnn_learn.h"

#ifndef RTNN_KNN
#define RTNN_KNN 5
#endif

namespace {

struct Options {
  std::string pfile, qfile, search_mode = "radius", out_file, model_file, convert_file;
  unsigned threads = 0;
  float radius = 2.0f;
  unsigned knn = 50;
  int device = 0;
  bool check = false, partition = true, parse_only = false;
};

void usage(const char* argv0) {
  std::fprintf(stderr,
               "Usage: %s [options]\n"
               "  --pfile      | -f   File for search points (also the queries unless -q).\n"
               "  --qfile      | -q   File for queries.\n"
               "  --searchmode | -sm  \"knn\" or \"radius\" (default radius).\n"
               "  --radius     | -r   Search radius (default 2).\n"
               "  --knn        | -k   Max K returned in radius search (default 50); knn uses K=%d.\n"
               "  --device     | -d   GPU id (default 0).\n"
               "  --check      | -c   Sanity check the result (default 0).\n"
               "  --partition  | -p   Density-bucket partitioning (default 1).\n"
               "  -o FILE  write the result rows (int32, -1 = none); -lm FILE learned model;\n"
               "  --parse-only  print the parsed points and exit; --convert FILE write them as\n"
               "  raw float32 (*.f32 / *.bin, read back by -f/-q) and exit; --threads N parser\n"
               "  threads (0 = all).\n",
               argv0, RTNN_KNN);
  std::exit(0);
}

Options parse(int argc, char** argv) {
  Options o;
  static const std::set<std::string> ignored = {
      "-i", "--interleave", "-m", "--msr", "-df", "--deferFree", "-fq", "--filterQueries",
      "-nb", "--numbatch", "-ab", "--autobatch", "-ac", "--autocrratio", "-s", "--gassort",
      "-ps", "--pointsort", "-qs", "--querysort", "-cr", "--crratio", "-gmu", "--gpumemused",
      "-egs", "--estgassize", "-g", "--gather", "-a", "--approx", "-sg", "--gsrRatio",
      "-mc", "--metacellScale", "-crs", "--crStep"};
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i >= argc - 1) usage(argv[0]);
      return argv[++i];
    };
    if (a == "-h" || a == "--help") usage(argv[0]);
    else if (a == "-f" || a == "--pfile") o.pfile = next();
    else if (a == "-q" || a == "--qfile") o.qfile = next();
    else if (a == "-k" || a == "--knn") o.knn = (unsigned)std::atoi(next().c_str());
    else if (a == "-sm" || a == "--searchmode") {
      o.search_mode = next();
      if (o.search_mode != "knn" && o.search_mode != "radius") usage(argv[0]);
    } else if (a == "-r" || a == "--radius") o.radius = std::stof(next());
    else if (a == "-d" || a == "--device") o.device = std::atoi(next().c_str());
    else if (a == "-c" || a == "--check") o.check = std::atoi(next().c_str()) != 0;
    else if (a == "-p" || a == "--partition") o.partition = std::atoi(next().c_str()) != 0;
    else if (a == "-o") o.out_file = next();
    else if (a == "-lm") o.model_file = next();
    else if (a == "--parse-only") o.parse_only = true;
    else if (a == "--convert") o.convert_file = next();
    else if (a == "--threads") o.threads = (unsigned)std::atoi(next().c_str());
    else if (ignored.count(a)) {
      const std::string v = next();
      std::fprintf(stderr, "warning: %s %s has no effect (accepted for compatibility)\n",
                   a.c_str(), v.c_str());
    } else {
      std::fprintf(stderr, "Unknown option '%s'\n", a.c_str());
      usage(argv[0]);
    }
  }
  if (o.search_mode == "knn") o.knn = RTNN_KNN;
  if (o.pfile.empty()) usage(argv[0]);
  return o;
}

std::vector<float> read_points(const std::string& path, unsigned threads) {
  std::vector<float> xyz;
  std::string err;
  if (!rtnn::read_points_file(path, threads, &xyz, &err)) {
    std::fprintf(stderr, "Could not read the frame data (%s)\n", err.c_str());
    std::exit(1);
  }
  return xyz;
}

float d2(const float* a, const float* b) {
  const float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  const float s = dx * dx + dy * dy;
  return s + dz * dz;
}

// Soundness of every returned neighbor and, for KNN, the distance set of 5 random queries
// against a brute force (the checks of check.cpp:20-139).
bool sanity_check(const Options& o, const std::vector<float>& P, const std::vector<float>& Q,
                  const std::vector<int32_t>& res) {
  const size_t nq = Q.size() / 3, np = P.size() / 3, K = o.knn;
  const float r2 = o.radius * o.radius;
  size_t total = 0;
  for (size_t q = 0; q < nq; ++q)
    for (size_t n = 0; n < K; ++n) {
      const int32_t p = res[q * K + n];
      if (p < 0) break;
      ++total;
      if (!(d2(&P[3 * (size_t)p], &Q[3 * q]) < r2)) {
        std::printf("Point %d is not a neighbor of query %zu\n", p, q);
        return false;
      }
    }
  std::fprintf(stderr, "Avg neighbor/query: %f\n", nq ? (double)total / nq : 0.0);
  if (o.search_mode != "knn") return true;
  std::mt19937 rng(12345);
  for (int t = 0; t < 5 && nq; ++t) {
    const size_t q = rng() % nq;
    std::priority_queue<float> top;
    for (size_t p = 0; p < np; ++p) {
      const float d = d2(&Q[3 * q], &P[3 * p]);
      if (d > 0 && d < r2) {
        if (top.size() < K) top.push(d);
        else if (d < top.top()) { top.pop(); top.push(d); }
      }
    }
    std::multiset<float> gt, got;
    while (!top.empty()) { gt.insert(top.top()); top.pop(); }
    for (size_t n = 0; n < K && res[q * K + n] >= 0; ++n)
      got.insert(d2(&Q[3 * q], &P[3 * (size_t)res[q * K + n]]));
    if (gt != got) {
      std::printf("Incorrect query [%zu]\n", q);
      return false;
    }
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  const Options o = parse(argc, argv);
  std::vector<float> P = read_points(o.pfile, o.threads);
  const bool same = o.qfile.empty() || o.qfile == o.pfile;
  std::vector<float> Qv = same ? std::vector<float>() : read_points(o.qfile, o.threads);
  const std::vector<float>& Q = same ? P : Qv;
  const uint64_t np = P.size() / 3, nq = Q.size() / 3;
  if (!o.convert_file.empty()) {
    std::string err;
    if (!rtnn::write_points_f32(o.convert_file, P, &err)) {
      std::fprintf(stderr, "%s\n", err.c_str());
      return 1;
    }
    std::printf("points %llu written to %s\n", (unsigned long long)np, o.convert_file.c_str());
    return 0;
  }
  if (o.parse_only) {
    double sum = 0;
    for (float v : P) sum += v;
    std::printf("points %llu checksum %.17g\n", (unsigned long long)np, sum);
    return 0;
  }
  if (np == 0 || nq == 0) {
    std::printf("empty query and/or points\n");
    return 0;
  }
  std::printf("========================================\n");
  std::printf("numPoints: %llu\nnumQueries: %llu\nsearchMode: %s\nradius: %g\nK: %u\n",
              (unsigned long long)np, (unsigned long long)nq, o.search_mode.c_str(), o.radius, o.knn);
  std::printf("Query partition? %s\n", o.partition ? "true" : "false");
  std::printf("========================================\n");
  rtnn_ctx* ctx = nullptr;
  if (rtnn_create(&ctx, o.device) != RTNN_OK) {
    std::fprintf(stderr, "Caught exception: no CUDA device %d\n", o.device);
    return 1;
  }
  uint32_t flags = o.partition ? RTNN_FLAG_PARTITION : 0u;
  if (!o.model_file.empty()) {
    std::vector<float> m(rtnn_model_size());
    std::ifstream mf(o.model_file, std::ios::binary);
    mf.read(reinterpret_cast<char*>(m.data()), (std::streamsize)(m.size() * 4));
    if (!mf || rtnn_model_set(ctx, m.data(), (uint32_t)m.size()) != RTNN_OK) {
      std::fprintf(stderr, "Caught exception: bad model file %s\n", o.model_file.c_str());
      return 1;
    }
    flags |= RTNN_FLAG_LEARNED;
  }
  const rtnn_mode mode = o.search_mode == "knn" ? RTNN_MODE_KNN : RTNN_MODE_RADIUS;
  std::vector<int32_t> res((size_t)nq * o.knn);
  rtnn_stats st{};
  const auto t0 = std::chrono::steady_clock::now();
  const rtnn_status s = rtnn_search(ctx, P.data(), np, same ? nullptr : Q.data(), nq, mode,
                                    o.radius, o.knn, flags, res.data(), &st);
  const auto t1 = std::chrono::steady_clock::now();
  if (s != RTNN_OK) {
    std::fprintf(stderr, "Caught exception: %s\n", rtnn_last_error(ctx));
    rtnn_destroy(ctx);
    return 1;
  }
  std::printf("time total search time: %.3f ms (device %.3f ms: build %.3f, partition %.3f, search %.3f)\n",
              std::chrono::duration<double, std::milli>(t1 - t0).count(), st.ms_total, st.ms_build,
              st.ms_partition, st.ms_search);
  std::printf("\tfallback queries: %llu, cells: %llu, cell size: %g\n",
              (unsigned long long)st.n_fallback, (unsigned long long)st.n_cells, st.cell_size);
  if (!o.out_file.empty()) {
    std::ofstream of(o.out_file, std::ios::binary);
    of.write(reinterpret_cast<const char*>(res.data()), (std::streamsize)(res.size() * 4));
  }
  int rc = 0;
  if (o.check) {
    if (sanity_check(o, P, Q, res)) std::fprintf(stderr, "Sanity check done.\n");
    else rc = 1;
  }
  rtnn_destroy(ctx);
  return rc;
}
