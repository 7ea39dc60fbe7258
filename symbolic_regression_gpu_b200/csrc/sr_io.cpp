// sr_io.cpp — parallel loaders of the reference's dataset and population
// text files.
//
// shared_data.txt (reference load_data_file, src/utils/utils.cpp:235-300):
//   one datapoint per line, num_vars + 1 numbers (x0 .. x_{V-1}, y).  The
//   reference parses every number with strtod into a double and the evolution
//   loop narrows it to float (src/cleaned/cl_sr_system.cpp:98-104); here each
//   number is parsed with std::from_chars (correctly rounded, like strtod) and
//   narrowed the same way, so the floats are identical.
// gen_N.txt (reference parse_input_info, utils.cpp:122-233):
//   <num_exprs>, then per expression four lines: "<num_vars> <num_dps>
//   <num_tokens>", the tokens, the values (doubles), the data file name.
//
// The file is memory-mapped, cut into line-aligned chunks, and the chunks are
// parsed by host threads (one pass to count, one to fill), so loading scales
// with the cores instead of one operator>> / strtod stream.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <charconv>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "sr_eval.h"

namespace {

struct Mapped {
  const char *p = nullptr;
  size_t n = 0;
  int fd = -1;
  ~Mapped() {
    if (p && n) munmap(const_cast<char *>(p), n);
    if (fd >= 0) close(fd);
  }
  bool open(const char *path) {
    fd = ::open(path, O_RDONLY);
    if (fd < 0) return false;
    struct stat st;
    if (fstat(fd, &st) != 0) return false;
    n = static_cast<size_t>(st.st_size);
    if (n == 0) return true;
    void *m = mmap(nullptr, n, PROT_READ, MAP_PRIVATE, fd, 0);
    if (m == MAP_FAILED) {
      n = 0;
      return false;
    }
    madvise(m, n, MADV_SEQUENTIAL);
    p = static_cast<const char *>(m);
    return true;
  }
};

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f'; }

inline const char *skip_inline_space(const char *s, const char *e) {
  while (s < e && (*s == ' ' || *s == '\t' || *s == '\r' || *s == '\v' || *s == '\f')) ++s;
  return s;
}

// One number of a line; false at the end of the line or on a parse error.
inline bool next_double(const char *&s, const char *e, double *out) {
  s = skip_inline_space(s, e);
  if (s >= e) return false;
  const char *b = s;
  if (*b == '+') ++b;  // strtod accepts a leading '+', from_chars does not
  const auto r = std::from_chars(b, e, *out);
  if (r.ec != std::errc() && r.ec != std::errc::result_out_of_range) return false;
  if (r.ec == std::errc::result_out_of_range) {
    // strtod's behaviour: +-HUGE_VAL on overflow, a denormal / 0 on underflow.
    *out = std::strtod(std::string(s, r.ptr).c_str(), nullptr);
  }
  s = r.ptr;
  return true;
}

inline bool next_long(const char *&s, const char *e, long long *out) {
  s = skip_inline_space(s, e);
  if (s >= e) return false;
  const char *b = s;
  if (*b == '+') ++b;
  const auto r = std::from_chars(b, e, *out);
  if (r.ec != std::errc()) return false;
  s = r.ptr;
  return true;
}

int thread_count(int requested) {
  const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  return requested > 0 ? std::min(requested, 256) : hw;
}

// Start of every line of [p, p+n) that holds a non-blank character,
// found in parallel.
std::vector<const char *> data_lines(const char *p, size_t n, int threads) {
  const int T = std::max(1, std::min<int>(threads, static_cast<int>(n / (1 << 16)) + 1));
  std::vector<std::vector<const char *>> parts(static_cast<size_t>(T));
  std::vector<std::thread> pool;
  for (int t = 0; t < T; ++t) {
    pool.emplace_back([&, t] {
      size_t a = n * t / T, b = n * (t + 1) / T;
      // a line belongs to the chunk its first character falls in
      if (t > 0)
        while (a < b && p[a - 1] != '\n') ++a;
      auto &out = parts[static_cast<size_t>(t)];
      size_t i = a;
      while (i < b) {
        const char *nl = static_cast<const char *>(std::memchr(p + i, '\n', n - i));
        const size_t end = nl ? static_cast<size_t>(nl - p) : n;
        bool blank = true;
        for (size_t k = i; k < end && blank; ++k) blank = is_space(p[k]);
        if (!blank) out.push_back(p + i);
        i = end + 1;
      }
    });
  }
  for (auto &th : pool) th.join();
  std::vector<const char *> lines;
  for (auto &v : parts) lines.insert(lines.end(), v.begin(), v.end());
  return lines;
}

inline const char *line_end(const char *s, const char *e) {
  const char *nl = static_cast<const char *>(std::memchr(s, '\n', static_cast<size_t>(e - s)));
  return nl ? nl : e;
}

}  // namespace

extern "C" {

sr_status sr_load_shared_data(const char *path, int32_t num_vars, int64_t max_dps, float *X,
                              int64_t ld, int64_t *num_dps, int32_t threads) {
  if (!path || !num_dps || num_vars < 0 || num_vars > SR_MAX_VARS) return SR_ERR_INVALID_ARGUMENT;
  Mapped m;
  if (!m.open(path)) return SR_ERR_INVALID_ARGUMENT;
  const std::vector<const char *> lines = data_lines(m.p, m.n, thread_count(threads));
  int64_t N = static_cast<int64_t>(lines.size());
  if (max_dps >= 0) N = std::min<int64_t>(N, max_dps);
  *num_dps = N;
  if (!X) return SR_OK;  // size query
  if (ld < N) return SR_ERR_INVALID_ARGUMENT;
  const int cols = num_vars + 1;
  const int T = std::max(1, std::min<int>(thread_count(threads), static_cast<int>(N / 4096) + 1));
  std::atomic<int> bad{0};
  std::vector<std::thread> pool;
  const char *fe = m.p + m.n;
  for (int t = 0; t < T; ++t) {
    pool.emplace_back([&, t] {
      const int64_t a = N * t / T, b = N * (t + 1) / T;
      for (int64_t j = a; j < b && !bad.load(std::memory_order_relaxed); ++j) {
        const char *s = lines[static_cast<size_t>(j)];
        const char *e = line_end(s, fe);
        for (int v = 0; v < cols; ++v) {
          double d;
          if (!next_double(s, e, &d)) {
            bad.store(1);
            return;
          }
          X[static_cast<int64_t>(v) * ld + j] = static_cast<float>(d);
        }
        if (skip_inline_space(s, e) != e) {  // more numbers than num_vars + 1
          bad.store(1);
          return;
        }
      }
    });
  }
  for (auto &th : pool) th.join();
  return bad.load() ? SR_ERR_MALFORMED_EXPRESSION : SR_OK;
}

sr_status sr_load_population(const char *path, int32_t *num_exprs, int64_t *num_tokens,
                             int32_t *tokens, double *values, int64_t *offsets,
                             int32_t *num_vars, int32_t *num_dps, char *data_file,
                             int32_t data_file_cap, int32_t threads) {
  if (!path || !num_exprs || !num_tokens) return SR_ERR_INVALID_ARGUMENT;
  Mapped m;
  if (!m.open(path)) return SR_ERR_INVALID_ARGUMENT;
  const char *fe = m.p + m.n;
  // First line: the expression count; then 4 lines per expression (the data
  // file name may be blank, so lines are split without dropping blanks).
  std::vector<const char *> lines;
  lines.reserve(1024);
  for (const char *s = m.p; s < fe;) {
    lines.push_back(s);
    const char *e = line_end(s, fe);
    s = e + 1;
  }
  size_t first = 0;
  while (first < lines.size()) {  // skip leading blank lines
    const char *s = skip_inline_space(lines[first], line_end(lines[first], fe));
    if (s != line_end(lines[first], fe)) break;
    ++first;
  }
  if (first >= lines.size()) return SR_ERR_MALFORMED_EXPRESSION;
  long long E = 0;
  {
    const char *s = lines[first];
    if (!next_long(s, line_end(s, fe), &E) || E <= 0 || E > (1ll << 30))
      return SR_ERR_MALFORMED_EXPRESSION;
  }
  if (lines.size() < first + 1 + 4 * static_cast<size_t>(E)) return SR_ERR_MALFORMED_EXPRESSION;
  auto rec = [&](long long i, int k) { return lines[first + 1 + 4 * static_cast<size_t>(i) + k]; };
  // Pass 1: metadata (token counts) of every expression, in parallel.
  std::vector<long long> meta(static_cast<size_t>(3 * E));
  const int T = std::max(1, std::min<int>(thread_count(threads), static_cast<int>(E / 256) + 1));
  std::atomic<int> bad{0};
  auto run = [&](auto &&body) {
    std::vector<std::thread> pool;
    for (int t = 0; t < T; ++t)
      pool.emplace_back([&, t] {
        const long long a = E * t / T, b = E * (t + 1) / T;
        for (long long i = a; i < b && !bad.load(std::memory_order_relaxed); ++i)
          if (!body(i)) bad.store(1);
      });
    for (auto &th : pool) th.join();
  };
  run([&](long long i) {
    const char *s = rec(i, 0);
    const char *e = line_end(s, fe);
    long long *mm = &meta[static_cast<size_t>(3 * i)];
    return next_long(s, e, &mm[0]) && next_long(s, e, &mm[1]) && next_long(s, e, &mm[2]) &&
           mm[2] >= 0 && mm[2] <= SR_MAX_TOKENS;
  });
  if (bad.load()) return SR_ERR_MALFORMED_EXPRESSION;
  int64_t total = 0;
  for (long long i = 0; i < E; ++i) total += meta[static_cast<size_t>(3 * i + 2)];
  *num_exprs = static_cast<int32_t>(E);
  *num_tokens = total;
  if (!tokens || !values || !offsets) return SR_OK;  // size query
  offsets[0] = 0;
  for (long long i = 0; i < E; ++i) offsets[i + 1] = offsets[i] + meta[static_cast<size_t>(3 * i + 2)];
  // Pass 2: tokens and values.
  run([&](long long i) {
    const int64_t o = offsets[i];
    const long long L = meta[static_cast<size_t>(3 * i + 2)];
    if (num_vars) num_vars[i] = static_cast<int32_t>(meta[static_cast<size_t>(3 * i)]);
    if (num_dps) num_dps[i] = static_cast<int32_t>(meta[static_cast<size_t>(3 * i + 1)]);
    const char *s = rec(i, 1);
    const char *e = line_end(s, fe);
    for (long long k = 0; k < L; ++k) {
      long long t;
      if (!next_long(s, e, &t)) return false;
      tokens[o + k] = static_cast<int32_t>(t);
    }
    s = rec(i, 2);
    e = line_end(s, fe);
    for (long long k = 0; k < L; ++k)
      if (!next_double(s, e, &values[o + k])) return false;
    return true;
  });
  if (bad.load()) return SR_ERR_MALFORMED_EXPRESSION;
  if (data_file && data_file_cap > 0) {
    const char *s = rec(0, 3);
    const char *e = line_end(s, fe);
    // the reference keeps the line as read by getline; drop a trailing '\r'
    if (e > s && e[-1] == '\r') --e;
    const size_t n = std::min<size_t>(static_cast<size_t>(e - s), static_cast<size_t>(data_file_cap - 1));
    std::memcpy(data_file, s, n);
    data_file[n] = '\0';
  }
  return SR_OK;
}

}  // extern "C"
