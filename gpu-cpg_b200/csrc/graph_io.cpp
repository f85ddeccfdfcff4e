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

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
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

}  // namespace

Status read_text_graph(const char* path, bool ignore_wgts, EdgeList& out,
                       std::string& err) {
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    err = std::string("cannot open ") + path + ": " + std::strerror(errno);
    return CPG_ERR_IO;
  }
  std::fseek(f, 0, SEEK_END);
  long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz < 0) {
    std::fclose(f);
    err = "cannot size input file";
    return CPG_ERR_IO;
  }
  std::vector<char> buf(static_cast<size_t>(sz) + 1);
  size_t got = std::fread(buf.data(), 1, static_cast<size_t>(sz), f);
  std::fclose(f);
  if (got != static_cast<size_t>(sz)) {
    err = "short read";
    return CPG_ERR_IO;
  }
  buf[got] = '\n';
  const char* p = buf.data();
  const char* end = buf.data() + got + 1;
  auto next_line = [&](const char*& ls, const char*& le) -> bool {
    if (p >= end - 1 && p >= end) return false;
    if (p >= buf.data() + got) return false;
    ls = p;
    const char* nl = static_cast<const char*>(std::memchr(p, '\n', end - p));
    le = nl ? nl : end;
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
  out.src.clear();
  out.dst.clear();
  out.w.clear();
  long lineno = n + 1;
  while (next_line(ls, le)) {
    ++lineno;
    const char* q1 = static_cast<const char*>(std::memchr(ls, '"', le - ls));
    if (!q1) {
      bool blank = true;
      for (const char* c = ls; c < le; ++c)
        if (*c != ' ' && *c != '\t' && *c != '\r') blank = false;
      if (blank) continue;
      err = "malformed edge line " + std::to_string(lineno);
      return CPG_ERR_IO;
    }
    const char* q2 = static_cast<const char*>(std::memchr(q1 + 1, '"', le - q1 - 1));
    const char* q3 = q2 ? static_cast<const char*>(std::memchr(q2 + 1, '"', le - q2 - 1)) : nullptr;
    const char* q4 = q3 ? static_cast<const char*>(std::memchr(q3 + 1, '"', le - q3 - 1)) : nullptr;
    long u = 0, v = 0;
    const char* a = q1 + 1;
    const char* b = q3 ? q3 + 1 : nullptr;
    if (!q4 || !parse_long(a, q2, u) || !parse_long(b, q4, v) || u < 0 ||
        u >= n || v < 0 || v >= n) {
      err = "malformed edge line " + std::to_string(lineno);
      return CPG_ERR_IO;
    }
    float w = 1.0f;
    if (!ignore_wgts) {
      const char* comma = static_cast<const char*>(std::memchr(ls, ',', le - ls));
      if (comma) {
        const char* c = static_cast<const char*>(std::memchr(q4 + 1, ',', le - q4 - 1));
        if (c) {
          std::string tok(c + 1, le);
          w = std::strtof(tok.c_str(), nullptr);
        }
      }
    }
    out.src.push_back(static_cast<int32_t>(u));
    out.dst.push_back(static_cast<int32_t>(v));
    out.w.push_back(w);
  }
  return CPG_OK;
}

Status edges_to_csr(const EdgeList& el, HostGraph& g, std::string& err) {
  const int64_t n = el.n;
  const int64_t m = static_cast<int64_t>(el.src.size());
  if (m > INT32_MAX - 1) {
    err = "too many edges for 32-bit CSR offsets";
    return CPG_ERR_INVALID;
  }
  g.n = el.n;
  g.m = static_cast<int32_t>(m);
  g.adjp.assign(n + 1, 0);
  g.iadjp.assign(n + 1, 0);
  for (int64_t e = 0; e < m; ++e) {
    if (el.src[e] < 0 || el.src[e] >= n || el.dst[e] < 0 || el.dst[e] >= n) {
      err = "edge endpoint out of range";
      return CPG_ERR_INVALID;
    }
    g.adjp[el.src[e] + 1]++;
    g.iadjp[el.dst[e] + 1]++;
  }
  for (int64_t v = 0; v < n; ++v) {
    g.adjp[v + 1] += g.adjp[v];
    g.iadjp[v + 1] += g.iadjp[v];
  }
  g.adj.resize(m);
  g.w.resize(m);
  g.iadj.resize(m);
  std::vector<int32_t> fill(n, 0);
  for (int64_t e = 0; e < m; ++e) {
    int32_t s = el.src[e];
    int32_t p = g.adjp[s] + fill[s]++;
    g.adj[p] = el.dst[e];
    g.w[p] = el.w[e];
  }
  std::fill(fill.begin(), fill.end(), 0);
  for (int64_t e = 0; e < m; ++e) {
    int32_t d = el.dst[e];
    int32_t p = g.iadjp[d] + fill[d]++;
    g.iadj[p] = el.src[e];
  }
  return CPG_OK;
}

Status csr_to_graph(int32_t n, int32_t m, const int32_t* adjp,
                    const int32_t* adjncy, const float* w, HostGraph& g,
                    std::string& err) {
  if (n < 0 || m < 0 || !adjp || (m > 0 && (!adjncy || !w))) {
    err = "null CSR buffer";
    return CPG_ERR_INVALID;
  }
  if (adjp[0] != 0 || adjp[n] != m) {
    err = "CSR offsets must start at 0 and end at m";
    return CPG_ERR_INVALID;
  }
  EdgeList el;
  el.n = n;
  el.src.resize(m);
  el.dst.assign(adjncy, adjncy + m);
  el.w.assign(w, w + m);
  for (int32_t v = 0; v < n; ++v) {
    if (adjp[v] > adjp[v + 1]) {
      err = "CSR offsets must be non-decreasing";
      return CPG_ERR_INVALID;
    }
    for (int32_t e = adjp[v]; e < adjp[v + 1]; ++e) el.src[e] = v;
  }
  return edges_to_csr(el, g, err);
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

}  // namespace cpg
