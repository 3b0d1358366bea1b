// Matrix Market reader / writer (host code; no device work).  The format: a banner line
// "%%MatrixMarket matrix <array|coordinate> <real|integer|pattern> <general|symmetric|
// skew-symmetric>", comment lines starting with '%', a size line ("m n" for array, "m n entries"
// for coordinate), then the values -- column by column for array (the lower triangle only for
// symmetric storage), "i j [value]" triplets with 1-based indices for coordinate.
#include "mtx.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "runtime.h"

namespace isvdb {
namespace {

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// Read-only mapping of a whole file.
struct Mapped {
  const char *p = nullptr;
  size_t n = 0;
  int fd = -1;
  explicit Mapped(const char *path) {
    fd = open(path, O_RDONLY);
    if (fd < 0) fail(kErrArgument, "%s: cannot open (%s)", path, strerror(errno));
    struct stat st;
    if (fstat(fd, &st) != 0) {
      const int e = errno;
      close(fd);
      fail(kErrArgument, "%s: cannot stat (%s)", path, strerror(e));
    }
    n = (size_t)st.st_size;
    if (n) {
      void *m = mmap(nullptr, n, PROT_READ, MAP_PRIVATE, fd, 0);
      if (m == MAP_FAILED) {
        const int e = errno;
        close(fd);
        fail(kErrArgument, "%s: cannot map (%s)", path, strerror(e));
      }
      p = static_cast<const char *>(m);
      madvise(m, n, MADV_SEQUENTIAL);
    }
  }
  ~Mapped() {
    if (p) munmap(const_cast<char *>(p), n);
    if (fd >= 0) close(fd);
  }
  Mapped(const Mapped &) = delete;
  Mapped &operator=(const Mapped &) = delete;
};

// The next line [b, e) (without its line break) from p; false at the end of the data.
bool next_line(const char *&p, const char *end, const char *&b, const char *&e) {
  if (p >= end) return false;
  b = p;
  const char *nl = static_cast<const char *>(memchr(p, '\n', (size_t)(end - p)));
  e = nl ? nl : end;
  p = nl ? nl + 1 : end;
  if (e > b && e[-1] == '\r') --e;
  return true;
}

std::vector<std::string> split(const char *b, const char *e) {
  std::vector<std::string> out;
  while (b < e) {
    while (b < e && is_space(*b)) ++b;
    const char *s = b;
    while (b < e && !is_space(*b)) ++b;
    if (b > s) out.emplace_back(s, b);
  }
  return out;
}

std::string lower(std::string s) {
  for (char &c : s) c = (char)tolower((unsigned char)c);
  return s;
}

long long parse_size(const std::string &tok, const char *path) {
  long long v = 0;
  const auto r = std::from_chars(tok.data(), tok.data() + tok.size(), v);
  if (r.ec != std::errc() || r.ptr != tok.data() + tok.size() || v < 0)
    fail(kErrArgument, "%s: bad size '%s'", path, tok.c_str());
  return v;
}

MtxInfo parse_header(const char *path, const char *&p, const char *end) {
  const char *b, *e;
  if (!next_line(p, end, b, e)) fail(kErrArgument, "%s: empty file", path);
  std::vector<std::string> t = split(b, e);
  if (t.size() < 5 || t[0] != "%%MatrixMarket") fail(kErrArgument, "%s: no %%%%MatrixMarket banner", path);
  for (int i = 1; i < 5; ++i) t[i] = lower(t[i]);
  if (t[1] != "matrix") fail(kErrArgument, "%s: object '%s' is not a matrix", path, t[1].c_str());
  MtxInfo h;
  if (t[2] == "coordinate") h.coordinate = true;
  else if (t[2] != "array") fail(kErrArgument, "%s: unknown format '%s'", path, t[2].c_str());
  if (t[3] == "real" || t[3] == "double") h.field = 0;
  else if (t[3] == "integer") h.field = 1;
  else if (t[3] == "pattern") h.field = 2;
  else fail(kErrArgument, "%s: unsupported field '%s' (real, integer or pattern)", path, t[3].c_str());
  if (t[4] == "general") h.symmetry = 0;
  else if (t[4] == "symmetric") h.symmetry = 1;
  else if (t[4] == "skew-symmetric") h.symmetry = 2;
  else fail(kErrArgument, "%s: unsupported symmetry '%s'", path, t[4].c_str());
  if (!h.coordinate && h.field == 2) fail(kErrArgument, "%s: pattern field in array format", path);
  for (;;) {  // comments and blank lines, then the size line
    if (!next_line(p, end, b, e)) fail(kErrArgument, "%s: no size line", path);
    const char *q = b;
    while (q < e && is_space(*q)) ++q;
    if (q == e || *q == '%') continue;
    const std::vector<std::string> s = split(b, e);
    if (s.size() != (h.coordinate ? 3u : 2u)) fail(kErrArgument, "%s: bad size line", path);
    h.m = parse_size(s[0], path);
    h.n = parse_size(s[1], path);
    if (h.coordinate) h.entries = parse_size(s[2], path);
    break;
  }
  if (h.symmetry && h.m != h.n) fail(kErrArgument, "%s: symmetric storage of a non-square matrix", path);
  if (!h.coordinate)
    h.entries = h.symmetry == 0 ? h.m * h.n : h.symmetry == 1 ? h.n * (h.n + 1) / 2 : h.n * (h.n - 1) / 2;
  return h;
}

template <class T>
bool parse_value(const char *b, const char *e, T *v) {
  if (b < e && *b == '+') ++b;
  const auto r = std::from_chars(b, e, *v);
  return r.ec == std::errc() && r.ptr == e;
}

// Next token [b, e) from p; false at the end.
inline bool next_token(const char *&p, const char *end, const char *&b, const char *&e) {
  while (p < end && is_space(*p)) ++p;
  if (p >= end) return false;
  b = p;
  while (p < end && !is_space(*p)) ++p;
  e = p;
  return true;
}

[[noreturn]] void bad_value(const char *path, long long k, const char *b, const char *e) {
  const std::string tok(b, std::min<size_t>((size_t)(e - b), 40));
  fail(kErrArgument, "%s: value %lld ('%s') is not a number", path, k + 1, tok.c_str());
}

// Dense general values: tokens split over host threads at whitespace boundaries, counted, then
// parsed into their column-major positions.
template <class T>
void read_array_general(const char *path, const MtxInfo &h, const char *p, const char *end, T *a, long long lda,
                        char ordera) {
  const size_t bytes = (size_t)(end - p);
  unsigned hw = std::thread::hardware_concurrency();
  int nt = (int)std::min<size_t>(std::max(1u, std::min(hw, 64u)), std::max<size_t>(1, bytes >> 22));
  std::vector<const char *> cut(nt + 1);
  cut[0] = p;
  for (int t = 1; t < nt; ++t) {
    const char *c = std::max(p + bytes * t / nt, cut[t - 1]);
    while (c < end && !is_space(*c)) ++c;  // a chunk starts at whitespace: no token is split
    cut[t] = c;
  }
  cut[nt] = end;
  std::vector<long long> count(nt + 1, 0);
  auto run = [&](auto &&body) {
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(body, t);
    body(0);
    for (auto &x : th) x.join();
  };
  run([&](int t) {
    long long c = 0;
    for (const char *q = cut[t]; q < cut[t + 1]; ++q)
      if (!is_space(*q) && (q == cut[t] || is_space(q[-1]))) ++c;
    count[t + 1] = c;
  });
  for (int t = 0; t < nt; ++t) count[t + 1] += count[t];
  if (count[nt] != h.entries)
    fail(kErrArgument, "%s: %lld values for a %lld x %lld array", path, count[nt], h.m, h.n);
  std::atomic<long long> bad{-1};
  run([&](int t) {
    long long k = count[t];
    const char *q = cut[t], *b, *e;
    while (next_token(q, cut[t + 1], b, e)) {
      const long long i = k % h.m, j = k / h.m;
      T v;
      if (!parse_value(b, e, &v)) {
        long long none = -1;
        bad.compare_exchange_strong(none, k);
        return;
      }
      a[ordera == 'C' ? i + j * lda : i * lda + j] = v;
      ++k;
    }
  });
  if (bad.load() >= 0) {  // report the first bad token from a sequential pass
    const char *q = p, *b, *e;
    for (long long k = 0; next_token(q, end, b, e); ++k) {
      T v;
      if (!parse_value(b, e, &v)) bad_value(path, k, b, e);
    }
  }
}

template <class T>
void zero(T *a, long long m, long long n, long long lda, char ordera) {
  const long long outer = ordera == 'C' ? n : m, inner = ordera == 'C' ? m : n;
  for (long long o = 0; o < outer; ++o) std::fill(a + o * lda, a + o * lda + inner, T(0));
}

}  // namespace

template <class T>
MtxInfo mtx_read(const char *path, T *a, long long lda, char ordera) {
  if (!path) fail(kErrArgument, "Matrix Market read: path is NULL");
  Mapped f(path);
  const char *p = f.p, *end = f.p + f.n;
  const MtxInfo h = parse_header(path, p, end);
  if (!a) return h;
  if (ordera != 'C' && ordera != 'R') fail(kErrArgument, "Matrix Market read: ordera must be 'C' or 'R'");
  if (lda < (ordera == 'C' ? h.m : h.n) || lda < 1) fail(kErrArgument, "Matrix Market read: lda too small");
  auto at = [&](long long i, long long j) -> T & { return a[ordera == 'C' ? i + j * lda : i * lda + j]; };
  if (!h.coordinate && h.symmetry == 0) {
    read_array_general<T>(path, h, p, end, a, lda, ordera);
    return h;
  }
  const char *b, *e;
  if (!h.coordinate) {  // symmetric / skew-symmetric: the lower triangle column by column
    const long long d = h.symmetry == 2 ? 1 : 0;
    long long k = 0;
    if (h.symmetry == 2)
      for (long long i = 0; i < h.n; ++i) at(i, i) = T(0);
    for (long long j = 0; j < h.n; ++j)
      for (long long i = j + d; i < h.n; ++i, ++k) {
        T v;
        if (!next_token(p, end, b, e)) fail(kErrArgument, "%s: %lld values, %lld expected", path, k, h.entries);
        if (!parse_value(b, e, &v)) bad_value(path, k, b, e);
        at(i, j) = v;
        at(j, i) = h.symmetry == 2 ? -v : v;
      }
    return h;
  }
  zero(a, h.m, h.n, lda, ordera);
  for (long long k = 0; k < h.entries; ++k) {
    long long ij[2];
    for (int c = 0; c < 2; ++c) {
      if (!next_token(p, end, b, e)) fail(kErrArgument, "%s: %lld entries, %lld expected", path, k, h.entries);
      const auto r = std::from_chars(b, e, ij[c]);
      if (r.ec != std::errc() || r.ptr != e) bad_value(path, k, b, e);
    }
    const long long i = ij[0] - 1, j = ij[1] - 1;
    if (i < 0 || i >= h.m || j < 0 || j >= h.n)
      fail(kErrArgument, "%s: entry %lld at (%lld, %lld) outside %lld x %lld", path, k + 1, ij[0], ij[1], h.m, h.n);
    T v = T(1);
    if (h.field != 2) {
      if (!next_token(p, end, b, e)) fail(kErrArgument, "%s: entry %lld has no value", path, k + 1);
      if (!parse_value(b, e, &v)) bad_value(path, k, b, e);
    }
    at(i, j) = v;
    if (h.symmetry && i != j) at(j, i) = h.symmetry == 2 ? -v : v;
  }
  return h;
}

template <class T>
void mtx_write(const char *path, long long m, long long n, const T *a, long long lda, char ordera) {
  if (!path || (!a && m * n > 0)) fail(kErrArgument, "Matrix Market write: NULL argument");
  if (m < 0 || n < 0) fail(kErrArgument, "Matrix Market write: negative size");
  if (ordera != 'C' && ordera != 'R') fail(kErrArgument, "Matrix Market write: ordera must be 'C' or 'R'");
  if (m * n > 0 && lda < (ordera == 'C' ? m : n)) fail(kErrArgument, "Matrix Market write: lda too small");
  FILE *f = fopen(path, "w");
  if (!f) fail(kErrArgument, "%s: cannot create (%s)", path, strerror(errno));
  std::string buf = "%%MatrixMarket matrix array real general\n" + std::to_string(m) + " " + std::to_string(n) + "\n";
  bool ok = true;
  char tmp[64];
  for (long long j = 0; j < n && ok; ++j)
    for (long long i = 0; i < m; ++i) {
      const T v = a[ordera == 'C' ? i + j * lda : i * lda + j];
      const auto r = std::to_chars(tmp, tmp + sizeof(tmp), v);  // shortest form that reads back exactly
      buf.append(tmp, r.ptr);
      buf.push_back('\n');
      if (buf.size() >= (1u << 20)) {
        ok = fwrite(buf.data(), 1, buf.size(), f) == buf.size();
        buf.clear();
        if (!ok) break;
      }
    }
  if (ok && !buf.empty()) ok = fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  if (fclose(f) != 0) ok = false;
  if (!ok) fail(kErrArgument, "%s: write failed", path);
}

template MtxInfo mtx_read<float>(const char *, float *, long long, char);
template MtxInfo mtx_read<double>(const char *, double *, long long, char);
template void mtx_write<float>(const char *, long long, long long, const float *, long long, char);
template void mtx_write<double>(const char *, long long, long long, const double *, long long, char);

}  // namespace isvdb
