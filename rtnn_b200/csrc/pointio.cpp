// pointio.cpp -- point-cloud files for the optixNSearch CLI: a multithreaded text reader
// with the reference's per-line semantics, and raw float32 files.
//
// Text: the file is mapped, cut into one byte range per thread at line boundaries, each
// thread counts its lines ('\n'-terminated; a last line without '\n' counts too, as
// std::istream::getline does), an exclusive scan over the counts gives each thread its
// first row, and the threads parse their lines into place. A field is what sscanf's "%lf"
// takes (util.cpp:125): leading white space skipped, then a strtod number. The common
// decimal forms go through std::from_chars (correctly rounded, as glibc's strtod is); hex
// floats and out-of-range values go through strtod itself, so every field gets strtod's
// double. The cast to float rounds to nearest, as the reference's make_float3(x, y, z).
// The reference reads lines into a 1024-byte buffer and stops at the first longer line;
// this reader takes lines of any length.
#include "pointio.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>

namespace rtnn {
namespace {

bool is_space(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

// scanf reads the longest prefix of a number: an exponent marker with no digits after it
// ("1e", "2e+") is consumed along with the number [b, q), whose value is the mantissa's.
const char* take_bare_exponent(const char* b, const char* q, const char* e, bool hex) {
  if (q == e) return q;
  const char lo = hex ? 'p' : 'e', up = hex ? 'P' : 'E';
  if (*q != lo && *q != up) return q;
  const char* m = (*b == '+' || *b == '-') ? b + 1 : b;
  if (std::isalpha((unsigned char)*m)) return q;  // inf / nan take no exponent
  for (const char* c = m; c < q; ++c)
    if (*c == lo || *c == up) return q;  // already has an exponent
  const char* r = q + 1;
  if (r < e && (*r == '+' || *r == '-')) ++r;
  return (r < e && *r >= '0' && *r <= '9') ? q : r;
}

// One "%lf" conversion of [p, e) as glibc's scanf makes it: the end of the consumed
// characters, or nullptr when no number parses.
const char* parse_double(const char* p, const char* e, double* out) {
  while (p < e && is_space(*p)) ++p;
  if (p == e) return nullptr;
  const char* s = p;
  if (*s == '+') {
    ++s;
    if (s == e || *s == '+' || *s == '-') return nullptr;
  }
  const char* m = (s < e && *s == '-') ? s + 1 : s;
  const bool hex = (e - m >= 2) && m[0] == '0' && (m[1] == 'x' || m[1] == 'X');
  if (!hex) {
    double d;
    const std::from_chars_result r = std::from_chars(s, e, d, std::chars_format::general);
    if (r.ec == std::errc()) {
      *out = d;
      return take_bare_exponent(s, r.ptr, e, false);
    }
    if (r.ec == std::errc::invalid_argument) return nullptr;
  }
  // strtod for the rest: hex floats, overflow to +-inf, underflow to subnormals or 0
  char buf[512];
  const size_t n = std::min<size_t>((size_t)(e - p), sizeof(buf) - 1);
  std::memcpy(buf, p, n);
  buf[n] = '\0';
  char* end = nullptr;
  const double d = std::strtod(buf, &end);
  if (end == buf) return nullptr;
  *out = d;
  return take_bare_exponent(p, p + (end - buf), e, hex);
}

// One line of text into xyz[0..2] (fields that do not parse stay 0).
void parse_line(const char* p, const char* e, float* xyz) {
  double v[3] = {0.0, 0.0, 0.0};
  for (int f = 0; f < 3; ++f) {
    if (f > 0) {
      if (p == e || *p != ',') break;
      ++p;
    }
    double d;
    const char* q = parse_double(p, e, &d);
    if (!q) break;
    v[f] = d;
    p = q;
  }
  xyz[0] = (float)v[0];
  xyz[1] = (float)v[1];
  xyz[2] = (float)v[2];
}

uint64_t count_lines(const char* p, const char* e) {
  uint64_t n = 0;
  while (p < e) {
    const void* nl = std::memchr(p, '\n', (size_t)(e - p));
    if (!nl) break;
    ++n;
    p = static_cast<const char*>(nl) + 1;
  }
  return n;
}

void parse_range(const char* p, const char* e, float* xyz) {
  while (p < e) {
    const void* nl = std::memchr(p, '\n', (size_t)(e - p));
    const char* le = nl ? static_cast<const char*>(nl) : e;
    parse_line(p, le, xyz);
    xyz += 3;
    p = le + 1;
  }
}

bool ends_with(const std::string& s, const char* suffix) {
  const size_t n = std::strlen(suffix);
  return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

bool read_binary(const std::string& path, std::vector<float>* xyz, std::string* err) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    *err = "cannot open " + path;
    return false;
  }
  std::fseek(f, 0, SEEK_END);
  const long size = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (size < 0 || size % 12 != 0) {
    std::fclose(f);
    *err = path + ": size is not a whole number of float32 x,y,z triples";
    return false;
  }
  xyz->resize((size_t)size / 4);
  const size_t got = size ? std::fread(xyz->data(), 4, xyz->size(), f) : 0;
  std::fclose(f);
  if (got != xyz->size()) {
    *err = "short read of " + path;
    return false;
  }
  return true;
}

}  // namespace

bool is_binary_points_name(const std::string& path) {
  return ends_with(path, ".bin") || ends_with(path, ".f32");
}

bool read_points_file(const std::string& path, unsigned threads, std::vector<float>* xyz,
                      std::string* err) {
  xyz->clear();
  if (is_binary_points_name(path)) return read_binary(path, xyz, err);
  const int fd = ::open(path.c_str(), O_RDONLY);
  if (fd < 0) {
    *err = "cannot open " + path;
    return false;
  }
  struct stat st;
  if (::fstat(fd, &st) != 0) {
    ::close(fd);
    *err = "cannot stat " + path;
    return false;
  }
  const size_t size = (size_t)st.st_size;
  if (size == 0) {
    ::close(fd);
    return true;
  }
  void* map = ::mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
  ::close(fd);
  if (map == MAP_FAILED) {
    *err = "cannot map " + path;
    return false;
  }
  ::madvise(map, size, MADV_SEQUENTIAL);
  const char* base = static_cast<const char*>(map);

  unsigned t_n = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
  t_n = (unsigned)std::max<size_t>(1, std::min<size_t>(t_n, size / (256u << 10) + 1));
  // range t is [cut[t], cut[t + 1]): whole lines, the first starting after a '\n'
  std::vector<size_t> cut(t_n + 1, size);
  cut[0] = 0;
  for (unsigned t = 1; t < t_n; ++t) {
    const size_t nominal = std::max(cut[t - 1], size * t / t_n);
    const void* nl = nominal ? std::memchr(base + nominal - 1, '\n', size - nominal + 1) : base;
    cut[t] = nominal == 0 ? 0 : (nl ? (size_t)(static_cast<const char*>(nl) - base) + 1 : size);
  }
  std::vector<uint64_t> first(t_n + 1, 0);
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < t_n; ++t)
    pool.emplace_back([&, t] { first[t + 1] = count_lines(base + cut[t], base + cut[t + 1]); });
  for (auto& th : pool) th.join();
  pool.clear();
  if (base[size - 1] != '\n') first[t_n] += 1;  // a last line without its '\n'
  for (unsigned t = 0; t < t_n; ++t) first[t + 1] += first[t];
  xyz->resize((size_t)first[t_n] * 3);
  float* out = xyz->data();
  for (unsigned t = 0; t < t_n; ++t)
    pool.emplace_back([&, t] { parse_range(base + cut[t], base + cut[t + 1], out + 3 * first[t]); });
  for (auto& th : pool) th.join();
  ::munmap(map, size);
  return true;
}

bool write_points_f32(const std::string& path, const std::vector<float>& xyz, std::string* err) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    *err = "cannot create " + path;
    return false;
  }
  const size_t put = xyz.empty() ? 0 : std::fwrite(xyz.data(), 4, xyz.size(), f);
  const bool ok = std::fclose(f) == 0 && put == xyz.size();
  if (!ok) *err = "short write of " + path;
  return ok;
}

}  // namespace rtnn
