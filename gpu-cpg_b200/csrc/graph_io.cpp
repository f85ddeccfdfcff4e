// Host-side graph ingestion and the seeded DAG generator.
//
// Text format: the reference's CpGen::read_input (gpucpg/gpucpg.cu:453-548):
//   line 1: vertex count N
//   N lines of vertex names (ignored)
//   one edge per line: "u" -> "v"[, w];   (the delay defaults to 1.0 and is
//   ignored when ignore_wgts is set)
// Rows of the CSR keep edges in file order per tail vertex, as the reference's
// unordered_map<int, vector<pair<int,double>>> does (gpucpg.cu:500-541).
#include "cpg_internal.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <unordered_set>
#include <vector>

namespace cpg {

namespace {

// Parses an integer after optional blanks; returns false if none.
bool parse_long(const char*& p, const char* end, long& out) {
  while (p < end && (*p == ' ' || *p == '\t')) ++p;
  bool neg = false;
  if (p < end && (*p == '-' || *p == '+')) neg = (*p++ == '-');
  if (p >= end || *p < '0' || *p > '9') return false;
  long v = 0;
  while (p < end && *p >= '0' && *p <= '9') {
    v = v * 10 + (*p - '0');
    if (v > (1L << 40)) return false;
    ++p;
  }
  out = neg ? -v : v;
  return true;
}

// strtof on the text of [s, le): the fallback of parse_delay.
float strtof_bounded(const char* s, const char* le) {
  const std::string tok(s, le);
  return std::strtof(tok.c_str(), nullptr);
}

bool is_digit(char c) { return c >= '0' && c <= '9'; }

// The delay token of an edge line, rounded exactly as strtof rounds it (the
// reference converts it with std::stof).  A plain decimal of at most 19
// significant digits whose value is m * 10^e with m <= 2^53 and |e| <= 22
// takes Clinger's fast path: m and 10^e are exact doubles, so one IEEE
// multiply or divide gives q = the double nearest the decimal.  Rounding q to
// float then gives the float nearest the decimal unless q lies exactly
// halfway between two floats (every such midpoint is itself a double, so no
// midpoint can lie strictly between the decimal and q); that case, and every
// other form strtof accepts (hex, inf, nan, long mantissas, large exponents),
// goes to strtof itself.  The scan never passes the end of the line.
float parse_delay(const char* s, const char* le) {
  static const double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,
                                    1e8,  1e9,  1e10, 1e11, 1e12, 1e13, 1e14, 1e15,
                                    1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};
  const char* p = s;
  while (p < le && (*p == ' ' || *p == '\t')) ++p;
  if (p == le) return 0.0f;  // nothing to convert: strtof returns 0
  bool neg = false;
  if (*p == '-' || *p == '+') neg = (*p++ == '-');
  uint64_t m = 0;
  int digits = 0, frac = 0;
  bool any = false;
  while (p < le && is_digit(*p)) {
    any = true;
    if (m != 0 || *p != '0') {
      if (++digits > 19) return strtof_bounded(s, le);
      m = m * 10 + static_cast<uint64_t>(*p - '0');
    }
    ++p;
  }
  if (p < le && *p == '.') {
    ++p;
    while (p < le && is_digit(*p)) {
      any = true;
      if (m != 0 || *p != '0') {
        if (++digits > 19) return strtof_bounded(s, le);
        m = m * 10 + static_cast<uint64_t>(*p - '0');
      }
      ++frac;
      ++p;
    }
  }
  if (!any) return strtof_bounded(s, le);
  long e10 = -frac;
  if (p < le && (*p == 'e' || *p == 'E')) {
    const char* x = p + 1;
    bool eneg = false;
    if (x < le && (*x == '-' || *x == '+')) eneg = (*x++ == '-');
    if (x >= le || !is_digit(*x)) return strtof_bounded(s, le);
    long ev = 0;
    while (x < le && is_digit(*x)) {
      if (ev < 100000) ev = ev * 10 + (*x - '0');
      ++x;
    }
    e10 += eneg ? -ev : ev;
    p = x;
  }
  // a letter, digit or point right after the number: not a plain decimal
  if (p < le && (is_digit(*p) || *p == '.' || *p == '_' || ((*p | 0x20) >= 'a' && (*p | 0x20) <= 'z')))
    return strtof_bounded(s, le);
  if (m == 0) return neg ? -0.0f : 0.0f;
  if (m > (uint64_t{1} << 53) || e10 < -22 || e10 > 22) return strtof_bounded(s, le);
  const double md = static_cast<double>(m);
  const double q = e10 < 0 ? md / kPow10[-e10] : md * kPow10[e10];
  if (!(q <= 3.4028234663852886e38)) return strtof_bounded(s, le);
  const float f = static_cast<float>(q);
  const double fd = static_cast<double>(f);
  if (fd != q) {
    const float g = std::nextafter(f, fd < q ? INFINITY : 0.0f);
    if ((fd + static_cast<double>(g)) * 0.5 == q) return strtof_bounded(s, le);
  }
  return neg ? -f : f;
}

// One edge line: "u" -> "v"[, w]; returns 0 for an edge, 1 for a blank
// line, -1 for a malformed one.
int parse_edge_line(const char* ls, const char* le, long n, bool ignore_wgts, int32_t& u_out,
                    int32_t& v_out, float& w_out) {
  const char* q1 = static_cast<const char*>(std::memchr(ls, '"', le - ls));
  if (!q1) {
    for (const char* c = ls; c < le; ++c)
      if (*c != ' ' && *c != '\t' && *c != '\r') return -1;
    return 1;
  }
  const char* q2 = static_cast<const char*>(std::memchr(q1 + 1, '"', le - q1 - 1));
  const char* q3 = q2 ? static_cast<const char*>(std::memchr(q2 + 1, '"', le - q2 - 1)) : nullptr;
  const char* q4 = q3 ? static_cast<const char*>(std::memchr(q3 + 1, '"', le - q3 - 1)) : nullptr;
  long u = 0, v = 0;
  const char* a = q1 + 1;
  const char* b = q3 ? q3 + 1 : nullptr;
  if (!q4 || !parse_long(a, q2, u) || !parse_long(b, q4, v) || u < 0 || u >= n || v < 0 ||
      v >= n)
    return -1;
  float w = 1.0f;
  if (!ignore_wgts) {
    // the delay after the comma that follows the second name
    const char* c = static_cast<const char*>(std::memchr(q4 + 1, ',', le - q4 - 1));
    if (c) w = parse_delay(c + 1, le);
  }
  u_out = static_cast<int32_t>(u);
  v_out = static_cast<int32_t>(v);
  w_out = w;
  return 0;
}

// Reads len bytes at file offset off into dst on the host threads, in 16 MB
// slices, each thread through its own stream.  Returns false on a short read.
bool read_range(const char* path, long off, char* dst, size_t len, int threads) {
  const size_t slice = size_t{16} << 20;
  const long n_slices = static_cast<long>((len + slice - 1) / slice);
  int fail = 0;
#pragma omp parallel num_threads(threads) reduction(| : fail)
  {
    FILE* g = std::fopen(path, "rb");
    if (!g) {
      fail = 1;
    } else {
#pragma omp for schedule(dynamic, 1)
      for (long k = 0; k < n_slices; ++k) {
        const size_t at = static_cast<size_t>(k) * slice;
        const size_t l = std::min(slice, len - at);
        if (std::fseek(g, off + static_cast<long>(at), SEEK_SET) != 0 ||
            std::fread(dst + at, 1, l, g) != l)
          fail = 1;
      }
      std::fclose(g);
    }
  }
  return fail == 0;
}

// Size of a file in bytes, or -1.
long file_size(const char* path) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return -1;
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fclose(f);
  return sz;
}

int io_threads(long bytes) {
#ifdef _OPENMP
  if (bytes > (1L << 22)) return std::max(1, std::min(32, omp_get_max_threads()));
#endif
  (void)bytes;
  return 1;
}

// Number of '\n' in [p, e).
size_t count_lines(const char* p, const char* e) {
  size_t c = 0;
  while (p < e) {
    const char* nl = static_cast<const char*>(std::memchr(p, '\n', e - p));
    if (!nl) break;
    ++c;
    p = nl + 1;
  }
  return c;
}

}  // namespace

// The file is read and parsed on the host threads.  The edge section is
// split at line boundaries into one piece per thread; each piece first counts
// its lines, then parses straight into the output at its line offset, and the
// slots of blank lines are squeezed out afterwards, so the result (and the
// first error reported) is the sequential parse's.
Status read_text_graph(const char* path, bool ignore_wgts, EdgeList& out,
                       std::string& err) {
  const long sz = file_size(path);
  if (sz < 0) {
    err = std::string("cannot open ") + path + ": " + std::strerror(errno);
    return CPG_ERR_IO;
  }
  const int threads = io_threads(sz);
  // a newline and a NUL after the text (left uninitialised otherwise: every
  // byte is read from the file)
  std::unique_ptr<char[]> buf(new (std::nothrow) char[static_cast<size_t>(sz) + 2]);
  if (!buf) {
    err = "cannot hold the input file in host memory";
    return CPG_ERR_OOM;
  }
  if (!read_range(path, 0, buf.get(), static_cast<size_t>(sz), threads)) {
    err = std::string("short read of ") + path;
    return CPG_ERR_IO;
  }
  const size_t got = static_cast<size_t>(sz);
  buf[got] = '\n';
  buf[got + 1] = '\0';
  const char* p = buf.get();
  const char* const text_end = buf.get() + got;  // last byte of the file + 1
  auto next_line = [&](const char*& ls, const char*& le) -> bool {
    if (p >= text_end) return false;
    ls = p;
    le = static_cast<const char*>(std::memchr(p, '\n', text_end + 1 - p));
    p = le + 1;
    return true;
  };
  const char *ls, *le;
  if (!next_line(ls, le)) {
    err = "empty input";
    return CPG_ERR_IO;
  }
  long n = 0;
  const char* q = ls;
  if (!parse_long(q, le, n) || n < 0 || n > (1L << 31) - 4) {
    err = "bad vertex count line";
    return CPG_ERR_IO;
  }
  for (long i = 0; i < n; ++i) {
    if (!next_line(ls, le)) {
      err = "missing vertex name lines";
      return CPG_ERR_IO;
    }
  }
  out.n = static_cast<int32_t>(n);
  const long first_line = n + 2;  // line number of the first edge line
  const char* body = p < text_end ? p : text_end;
  const size_t body_len = static_cast<size_t>(text_end - body);
  // piece boundaries at line starts
  std::vector<const char*> cut(static_cast<size_t>(threads) + 1);
  cut[0] = body;
  cut[threads] = text_end;
  for (int t = 1; t < threads; ++t) {
    const char* c = std::max(body + body_len * t / threads, cut[t - 1]);
    const char* nl = static_cast<const char*>(std::memchr(c, '\n', text_end + 1 - c));
    cut[t] = std::min(nl + 1, text_end);
  }
  // lines per piece (the last piece's final line may lack its newline)
  std::vector<size_t> lines(static_cast<size_t>(threads) + 1, 0);
#pragma omp parallel for num_threads(threads) schedule(static, 1)
  for (int t = 0; t < threads; ++t) {
    size_t c = count_lines(cut[t], cut[t + 1]);
    if (t == threads - 1 && cut[t + 1] > cut[t] && cut[t + 1][-1] != '\n') ++c;
    lines[t + 1] = c;
  }
  for (int t = 0; t < threads; ++t) lines[t + 1] += lines[t];
  const size_t total = lines[threads];
  out.src.resize(total);
  out.dst.resize(total);
  out.w.resize(total);
  std::vector<size_t> edges(static_cast<size_t>(threads), 0);
  std::vector<long> bad(static_cast<size_t>(threads), -1);
#pragma omp parallel for num_threads(threads) schedule(static, 1)
  for (int t = 0; t < threads; ++t) {
    const char* c = cut[t];
    const char* const end = cut[t + 1];
    int32_t* src = out.src.data() + lines[t];
    int32_t* dst = out.dst.data() + lines[t];
    float* w = out.w.data() + lines[t];
    size_t ln = 0, e = 0;
    while (c < end) {
      const char* nl = static_cast<const char*>(std::memchr(c, '\n', end - c));
      const char* eol = nl ? nl : end;
      const int r = parse_edge_line(c, eol, n, ignore_wgts, src[e], dst[e], w[e]);
      if (r < 0) {
        bad[t] = static_cast<long>(ln);
        break;
      }
      e += (r == 0);
      ++ln;
      c = eol + 1;
    }
    edges[t] = e;
  }
  for (int t = 0; t < threads; ++t) {
    if (bad[t] >= 0) {
      err = "malformed edge line " +
            std::to_string(first_line + static_cast<long>(lines[t]) + bad[t]);
      return CPG_ERR_IO;
    }
  }
  // squeeze out the slots that blank lines left unused
  size_t at = edges[0];
  for (int t = 1; t < threads; ++t) {
    if (at != lines[t] && edges[t] > 0) {
      std::memmove(out.src.data() + at, out.src.data() + lines[t], edges[t] * 4);
      std::memmove(out.dst.data() + at, out.dst.data() + lines[t], edges[t] * 4);
      std::memmove(out.w.data() + at, out.w.data() + lines[t], edges[t] * 4);
    }
    at += edges[t];
  }
  out.src.resize(at);
  out.dst.resize(at);
  out.w.resize(at);
  return CPG_OK;
}

// Fan-out CSR of an edge list; each row keeps the list's order (the
// reference's unordered_map of vectors, gpucpg.cu:500-541).  Runs on the host
// threads.  A list already grouped by tail (a text file written row by row) is
// taken as it is: only the offsets are computed and, when `grouped` is given,
// the heads and delays are left in the list for the caller to use.  Otherwise
// each thread counts the tails of its contiguous slice, per-thread row offsets
// follow from the counts, and each thread scatters its slice in order, so
// every row stays in list order.
Status edges_to_csr(const EdgeList& el, HostGraph& g, std::string& err, bool* grouped) {
  const int64_t n = el.n;
  const int64_t m = static_cast<int64_t>(el.src.size());
  if (m > INT32_MAX - 1) {
    err = "too many edges for 32-bit CSR offsets";
    return CPG_ERR_INVALID;
  }
  if (grouped) *grouped = false;
  g.n = el.n;
  g.m = static_cast<int32_t>(m);
  int threads = io_threads(m * 12);
  const int32_t* src = el.src.data();
  const int32_t* dst = el.dst.data();
  int64_t bad = INT64_MAX;
  int unsorted = 0;
#pragma omp parallel for num_threads(threads) reduction(min : bad) reduction(| : unsorted)
  for (int64_t e = 0; e < m; ++e) {
    if (src[e] < 0 || src[e] >= n || dst[e] < 0 || dst[e] >= n) bad = std::min(bad, e);
    if (e > 0 && src[e] < src[e - 1]) unsorted = 1;
  }
  if (bad != INT64_MAX) {
    err = "edge endpoint out of range at edge " + std::to_string(bad);
    return CPG_ERR_INVALID;
  }
  g.adjp.assign(static_cast<size_t>(n) + 1, 0);
  int32_t* adjp = g.adjp.data();
  if (!unsorted) {
    // row ends where the tail changes; rows with no edges take the next end
#pragma omp parallel for num_threads(threads)
    for (int64_t e = 0; e < m; ++e)
      if (e == m - 1 || src[e] != src[e + 1]) adjp[src[e] + 1] = static_cast<int32_t>(e + 1);
    for (int64_t v = 0; v < n; ++v) adjp[v + 1] = std::max(adjp[v + 1], adjp[v]);
    if (grouped) {
      *grouped = true;
      g.adj.clear();
      g.w.clear();
    } else {
      g.adj = el.dst;
      g.w = el.w;
    }
    return CPG_OK;
  }
  // per-thread counts: at most 2^28 counters in all
  if (n > 0) threads = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(threads, (int64_t{1} << 28) / n)));
  std::vector<int32_t> cnt(static_cast<size_t>(threads) * static_cast<size_t>(n));
  auto slice = [&](int t, int64_t& b, int64_t& e) {
    b = m * t / threads;
    e = m * (t + 1) / threads;
  };
#pragma omp parallel for num_threads(threads) schedule(static, 1)
  for (int t = 0; t < threads; ++t) {
    int32_t* c = cnt.data() + static_cast<size_t>(t) * n;
    std::fill(c, c + n, 0);
    int64_t b, e;
    slice(t, b, e);
    for (int64_t x = b; x < e; ++x) ++c[src[x]];
  }
  // cnt[t][v] becomes thread t's offset inside row v; adjp[v + 1] the degree
#pragma omp parallel for num_threads(threads) schedule(static)
  for (int64_t v = 0; v < n; ++v) {
    int32_t run = 0;
    for (int t = 0; t < threads; ++t) {
      int32_t& c = cnt[static_cast<size_t>(t) * n + v];
      const int32_t k = c;
      c = run;
      run += k;
    }
    adjp[v + 1] = run;
  }
  for (int64_t v = 0; v < n; ++v) adjp[v + 1] += adjp[v];
  g.adj.resize(static_cast<size_t>(m));
  g.w.resize(static_cast<size_t>(m));
#pragma omp parallel for num_threads(threads) schedule(static, 1)
  for (int t = 0; t < threads; ++t) {
    int32_t* c = cnt.data() + static_cast<size_t>(t) * n;
    int64_t b, e;
    slice(t, b, e);
    for (int64_t x = b; x < e; ++x) {
      const int32_t v = src[x];
      const int32_t p = adjp[v] + c[v]++;
      g.adj[p] = dst[x];
      g.w[p] = el.w[x];
    }
  }
  return CPG_OK;
}

// ------------------------------------------------------------------ generator

namespace {

struct Rng {
  std::mt19937_64 eng;
  explicit Rng(uint64_t s) : eng(s) {}
  double uniform() { return (eng() >> 11) * (1.0 / 9007199254740992.0); }
  int64_t below(int64_t n) {  // uniform in [0, n)
    return static_cast<int64_t>(uniform() * static_cast<double>(n)) % n;
  }
};

}  // namespace

Status generate_dag(const cpg_gen_params& p, EdgeList& out, std::string& err) {
  if (p.n_levels < 2 || p.n_first < 1 || p.n_last < 1 ||
      p.n_pins < p.n_first + p.n_last + (p.n_levels - 2) || p.level_span < 1) {
    err = "generator: need n_levels >= 2 and at least one pin per level";
    return CPG_ERR_INVALID;
  }
  if (p.degree_kind == 0 && (p.deg_lo < 1 || p.deg_hi < p.deg_lo)) {
    err = "generator: bad uniform degree range";
    return CPG_ERR_INVALID;
  }
  if (p.degree_kind == 1 && (p.deg_mean < 1.0 || p.deg_cap < 1)) {
    err = "generator: bad geometric degree";
    return CPG_ERR_INVALID;
  }
  Rng rng(p.seed);
  const int32_t L = p.n_levels;
  std::vector<int64_t> lstart(L + 1, 0);
  const int64_t mid = static_cast<int64_t>(p.n_pins) - p.n_first - p.n_last;
  for (int32_t l = 0; l < L; ++l) {
    int64_t sz;
    if (l == 0) sz = p.n_first;
    else if (l == L - 1) sz = p.n_last;
    else sz = mid / (L - 2) + ((l - 1) < (mid % (L - 2)) ? 1 : 0);
    lstart[l + 1] = lstart[l] + sz;
  }
  // pin id of the i-th pin in level order: a seeded permutation, so vertex ids
  // carry no level locality
  const int32_t np = p.n_pins;
  std::vector<int32_t> perm(np);
  for (int32_t i = 0; i < np; ++i) perm[i] = i;
  for (int32_t i = np - 1; i > 0; --i) {
    int32_t j = static_cast<int32_t>(rng.below(i + 1));
    std::swap(perm[i], perm[j]);
  }
  auto sample_degree = [&]() -> int32_t {
    if (p.degree_kind == 0)
      return p.deg_lo + static_cast<int32_t>(rng.below(p.deg_hi - p.deg_lo + 1));
    const double q = 1.0 - 1.0 / p.deg_mean;
    if (q <= 0.0) return 1;
    double u = rng.uniform();
    if (u <= 0.0) u = 1e-300;
    int64_t k = 1 + static_cast<int64_t>(std::floor(std::log(u) / std::log(q)));
    if (k > p.deg_cap) k = p.deg_cap;
    return static_cast<int32_t>(k);
  };
  auto sample_weight = [&]() -> float {
    if (p.weight_kind == 1)
      return static_cast<float>(p.iw_lo + rng.below(p.iw_hi - p.iw_lo + 1));
    return p.w_lo + (p.w_hi - p.w_lo) * static_cast<float>(rng.uniform());
  };
  out.n = np + (p.add_virtual ? 2 : 0);
  out.src.clear();
  out.dst.clear();
  out.w.clear();
  std::vector<uint8_t> has_in(np, 0);
  std::vector<int32_t> chosen;
  std::unordered_set<int32_t> chosen_set;
  for (int32_t l = 0; l + 1 < L; ++l) {
    const int32_t lmax = std::min(L - 1, l + p.level_span);
    const int64_t span_pins = lstart[lmax + 1] - lstart[l + 1];
    for (int64_t i = lstart[l]; i < lstart[l + 1]; ++i) {
      const int32_t u = perm[i];
      int32_t deg = sample_degree();
      if (deg > span_pins) deg = static_cast<int32_t>(span_pins);
      chosen.clear();
      chosen_set.clear();
      for (int32_t k = 0; k < deg; ++k) {
        for (int attempt = 0; attempt < 64; ++attempt) {
          const int32_t tl = l + 1 + static_cast<int32_t>(rng.below(lmax - l));
          const int64_t sz = lstart[tl + 1] - lstart[tl];
          const int32_t v = perm[lstart[tl] + rng.below(sz)];
          if (chosen_set.insert(v).second) {
            chosen.push_back(v);
            break;
          }
        }
      }
      for (int32_t v : chosen) {
        out.src.push_back(u);
        out.dst.push_back(v);
        out.w.push_back(sample_weight());
        has_in[v] = 1;
      }
    }
  }
  // repair: every pin above level 0 gets at least one in-edge from level-1
  for (int32_t l = 1; l < L; ++l) {
    for (int64_t i = lstart[l]; i < lstart[l + 1]; ++i) {
      const int32_t v = perm[i];
      if (has_in[v]) continue;
      const int64_t sz = lstart[l] - lstart[l - 1];
      const int32_t u = perm[lstart[l - 1] + rng.below(sz)];
      out.src.push_back(u);
      out.dst.push_back(v);
      out.w.push_back(sample_weight());
      has_in[v] = 1;
    }
  }
  if (p.add_virtual) {
    const int32_t S = np, T = np + 1;
    for (int64_t i = lstart[0]; i < lstart[1]; ++i) {
      out.src.push_back(S);
      out.dst.push_back(perm[i]);
      out.w.push_back(0.0f);
    }
    for (int64_t i = lstart[L - 1]; i < lstart[L]; ++i) {
      out.src.push_back(perm[i]);
      out.dst.push_back(T);
      out.w.push_back(0.0f);
    }
  }
  return CPG_OK;
}

Status write_text_graph(const EdgeList& el, const char* path, std::string& err) {
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    err = std::string("cannot open ") + path + " for writing";
    return CPG_ERR_IO;
  }
  std::vector<char> iobuf(1 << 22);
  std::setvbuf(f, iobuf.data(), _IOFBF, iobuf.size());
  std::fprintf(f, "%d\n", el.n);
  for (int32_t i = 0; i < el.n; ++i) std::fprintf(f, "\"%d\";\n", i);
  for (size_t e = 0; e < el.src.size(); ++e)
    std::fprintf(f, "\"%d\" -> \"%d\", %.9g;\n", el.src[e], el.dst[e],
                 static_cast<double>(el.w[e]));
  if (std::fclose(f) != 0) {
    err = "write failed";
    return CPG_ERR_IO;
  }
  return CPG_OK;
}

// Binary CSR file, the layout of the reference's Graph::write_to_bin and
// read_from_bin (gpucpg/graph.h:24-56): int32 N, int32 M, int32 adjp[N+1],
// int32 adjncy[M], float w[M], host byte order, no padding.
Status write_csr_bin(int32_t n, int32_t m, const int32_t* adjp, const int32_t* adj,
                     const float* w, const char* path, std::string& err) {
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    err = std::string("cannot open ") + path + " for writing";
    return CPG_ERR_IO;
  }
  const size_t nn = static_cast<size_t>(n) + 1, mm = static_cast<size_t>(m);
  bool ok = std::fwrite(&n, 4, 1, f) == 1 && std::fwrite(&m, 4, 1, f) == 1 &&
            std::fwrite(adjp, 4, nn, f) == nn && (mm == 0 || (std::fwrite(adj, 4, mm, f) == mm &&
                                                              std::fwrite(w, 4, mm, f) == mm));
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    err = std::string("write failed: ") + path;
    return CPG_ERR_IO;
  }
  return CPG_OK;
}

// Reads and checks a binary CSR file: the size must match the header, the
// offsets must rise from 0 to M, and every head must lie in 0..N-1.
Status read_csr_bin(const char* path, HostGraph& g, std::string& err) {
  const long sz = file_size(path);
  if (sz < 0) {
    err = std::string("cannot open ") + path + ": " + std::strerror(errno);
    return CPG_ERR_IO;
  }
  int32_t hdr[2] = {-1, -1};
  if (sz < 8 || !read_range(path, 0, reinterpret_cast<char*>(hdr), 8, 1)) {
    err = "binary CSR file shorter than its header";
    return CPG_ERR_IO;
  }
  const int64_t n = hdr[0], m = hdr[1];
  if (n < 0 || m < 0 || n > INT32_MAX - 2 || sz != 8 + 4 * (n + 1) + 8 * m) {
    err = "binary CSR file size does not match its header (N=" + std::to_string(n) +
          ", M=" + std::to_string(m) + ", " + std::to_string(sz) + " bytes)";
    return CPG_ERR_IO;
  }
  const int threads = io_threads(sz);
  g.n = static_cast<int32_t>(n);
  g.m = static_cast<int32_t>(m);
  g.adjp.resize(static_cast<size_t>(n) + 1);
  g.adj.resize(static_cast<size_t>(m));
  g.w.resize(static_cast<size_t>(m));
  const long off_adj = 8 + 4 * (n + 1), off_w = off_adj + 4 * m;
  if (!read_range(path, 8, reinterpret_cast<char*>(g.adjp.data()), 4 * (n + 1), threads) ||
      (m > 0 && (!read_range(path, off_adj, reinterpret_cast<char*>(g.adj.data()), 4 * m, threads) ||
                 !read_range(path, off_w, reinterpret_cast<char*>(g.w.data()), 4 * m, threads)))) {
    err = std::string("short read of ") + path;
    return CPG_ERR_IO;
  }
  if (g.adjp[0] != 0 || g.adjp[n] != m) {
    err = "binary CSR offsets must start at 0 and end at M";
    return CPG_ERR_IO;
  }
  int64_t bad_row = INT64_MAX, bad_edge = INT64_MAX;
#pragma omp parallel for num_threads(threads) reduction(min : bad_row)
  for (int64_t v = 0; v < n; ++v)
    if (g.adjp[v + 1] < g.adjp[v]) bad_row = std::min(bad_row, v);
#pragma omp parallel for num_threads(threads) reduction(min : bad_edge)
  for (int64_t e = 0; e < m; ++e)
    if (g.adj[e] < 0 || g.adj[e] >= n) bad_edge = std::min(bad_edge, e);
  if (bad_row != INT64_MAX) {
    err = "binary CSR offsets fall at row " + std::to_string(bad_row);
    return CPG_ERR_IO;
  }
  if (bad_edge != INT64_MAX) {
    err = "binary CSR head out of range at edge " + std::to_string(bad_edge);
    return CPG_ERR_IO;
  }
  return CPG_OK;
}

}  // namespace cpg
