// Host builders of the BVSS (bit-vector slice set) form, sigma = 8.
//
// pack_bvss restates build_bvss_from_fanout_csr (gpucpg/tc_sfxt_bvss.cuh:
// 106-156) and, applied to the transposed deviation relation, the A_dev
// builder (gpucpg/tc_pfxt_bvss.cuh:117-175): rows are visited in id order,
// each row's columns are merged into one 8-bit mask per interval, and the
// slices of an interval keep row order.  Instead of one hash map per row the
// builder sorts each row's interval ids and then counting-sorts all slices by
// interval, which keeps the same order.
#include "cpg_internal.hpp"

#include <algorithm>
#include <numeric>

namespace cpg {

namespace {

Status check_csr(int32_t n, const int32_t* row_ptr, const int32_t* cols, std::string& err) {
  if (n < 0 || !row_ptr) {
    err = "BVSS: null CSR";
    return CPG_ERR_INVALID;
  }
  if (row_ptr[0] != 0) {
    err = "BVSS: row_ptr must start at 0";
    return CPG_ERR_INVALID;
  }
  for (int32_t r = 0; r < n; ++r)
    if (row_ptr[r] > row_ptr[r + 1]) {
      err = "BVSS: row_ptr must be nondecreasing";
      return CPG_ERR_INVALID;
    }
  if (row_ptr[n] > 0 && !cols) {
    err = "BVSS: null column array";
    return CPG_ERR_INVALID;
  }
  for (int32_t e = 0; e < row_ptr[n]; ++e)
    if (cols[e] < 0 || cols[e] >= n) {
      err = "BVSS: column outside [0, n)";
      return CPG_ERR_INVALID;
    }
  return CPG_OK;
}

// Packs slices already grouped by interval (sl_row/sl_mask, interval i's
// slices at [off[i], off[i+1])) into VSS of 128.
void pack_slices(HostBvss& out, const std::vector<int64_t>& off,
                 const std::vector<int32_t>& sl_row, const std::vector<uint32_t>& sl_mask) {
  out.ptr.assign(static_cast<size_t>(out.n_intervals) + 1, 0);
  out.v2r.clear();
  out.cnt.clear();
  out.rows.clear();
  out.masks.clear();
  int32_t nv = 0;
  for (int32_t iv = 0; iv < out.n_intervals; ++iv) {
    out.ptr[iv] = nv;
    for (int64_t b = off[iv]; b < off[iv + 1]; b += 128) {
      const int64_t e = std::min<int64_t>(b + 128, off[iv + 1]);
      out.v2r.push_back(iv);
      out.cnt.push_back(static_cast<uint8_t>(e - b));
      out.rows.resize(static_cast<size_t>(nv + 1) * 128, -1);
      out.masks.resize(static_cast<size_t>(nv + 1) * 32, 0u);
      for (int64_t t = b; t < e; ++t) {
        const int32_t slot = static_cast<int32_t>(t - b);
        const int32_t lane = slot % 32, chunk = slot / 32;
        out.rows[static_cast<size_t>(nv) * 128 + lane * 4 + chunk] = sl_row[t];
        out.masks[static_cast<size_t>(nv) * 32 + lane] |= sl_mask[t] << (8 * chunk);
      }
      ++nv;
    }
  }
  out.ptr[out.n_intervals] = nv;
  out.n_vss = nv;
}

}  // namespace

Status pack_bvss(int32_t n, const int32_t* row_ptr, const int32_t* cols, HostBvss& out,
                 std::string& err) {
  Status st = check_csr(n, row_ptr, cols, err);
  if (st != CPG_OK) return st;
  out = HostBvss{};
  out.n_rows = n;
  out.n_intervals = (n + 7) / 8;
  out.row_bits.assign(static_cast<size_t>(n), 0);
  // pass 1: each row's slices in interval order
  std::vector<int32_t> s_int, s_row;
  std::vector<uint32_t> s_mask;
  s_int.reserve(static_cast<size_t>(row_ptr[n]));
  s_row.reserve(static_cast<size_t>(row_ptr[n]));
  s_mask.reserve(static_cast<size_t>(row_ptr[n]));
  std::vector<int32_t> tmp;
  for (int32_t r = 0; r < n; ++r) {
    tmp.assign(cols + row_ptr[r], cols + row_ptr[r + 1]);
    std::sort(tmp.begin(), tmp.end());
    int32_t bits = 0;
    for (size_t i = 0; i < tmp.size();) {
      const int32_t iv = tmp[i] >> 3;
      uint32_t m = 0;
      while (i < tmp.size() && (tmp[i] >> 3) == iv) m |= 1u << (tmp[i++] & 7);
      s_int.push_back(iv);
      s_row.push_back(r);
      s_mask.push_back(m);
      bits += __builtin_popcount(m);
    }
    out.row_bits[r] = bits;
    out.total_set_bits += static_cast<uint64_t>(bits);
  }
  const size_t ns = s_int.size();
  out.unpadded_slices = ns;
  // pass 2: stable counting sort of the slices by interval
  std::vector<int64_t> off(static_cast<size_t>(out.n_intervals) + 1, 0);
  for (size_t i = 0; i < ns; ++i) off[s_int[i] + 1]++;
  for (int32_t i = 0; i < out.n_intervals; ++i) off[i + 1] += off[i];
  std::vector<int32_t> g_row(ns);
  std::vector<uint32_t> g_mask(ns);
  {
    std::vector<int64_t> fill(off.begin(), off.end() - 1);
    for (size_t i = 0; i < ns; ++i) {
      const int64_t at = fill[s_int[i]]++;
      g_row[at] = s_row[i];
      g_mask[at] = s_mask[i];
    }
  }
  pack_slices(out, off, g_row, g_mask);
  return CPG_OK;
}

Status pack_bvss_compact(int32_t n, const int32_t* dev_off, HostBvss& out, std::string& err) {
  if (n < 0 || !dev_off || dev_off[0] != 0) {
    err = "BVSS: invalid compact deviation offsets";
    return CPG_ERR_INVALID;
  }
  for (int32_t v = 0; v < n; ++v)
    if (dev_off[v] > dev_off[v + 1]) {
      err = "BVSS: compact deviation offsets must be nondecreasing";
      return CPG_ERR_INVALID;
    }
  out = HostBvss{};
  out.n_rows = dev_off[n];
  out.n_intervals = (n + 7) / 8;
  // every deviation is one slice of its source's interval with the source's
  // bit; sources in id order, so the interval's slices are already grouped
  std::vector<int64_t> off(static_cast<size_t>(out.n_intervals) + 1, 0);
  const size_t ns = static_cast<size_t>(dev_off[n]);
  std::vector<int32_t> row(ns);
  std::vector<uint32_t> mask(ns);
  for (int32_t v = 0; v < n; ++v) {
    off[(v >> 3) + 1] += dev_off[v + 1] - dev_off[v];
    for (int32_t d = dev_off[v]; d < dev_off[v + 1]; ++d) {
      row[d] = d;
      mask[d] = 1u << (v & 7);
    }
  }
  for (int32_t i = 0; i < out.n_intervals; ++i) off[i + 1] += off[i];
  out.unpadded_slices = ns;
  out.total_set_bits = ns;
  pack_slices(out, off, row, mask);
  return CPG_OK;
}

std::vector<int32_t> bvss_decode_row(const HostBvss& b, int32_t row) {
  std::vector<int32_t> cols;
  for (int32_t vss = 0; vss < b.n_vss; ++vss) {
    const int32_t iv = b.v2r[vss];
    for (int32_t slot = 0; slot < 128; ++slot) {
      if (b.rows[static_cast<size_t>(vss) * 128 + slot] != row) continue;
      const int32_t lane = slot / 4, chunk = slot % 4;
      const uint32_t m = (b.masks[static_cast<size_t>(vss) * 32 + lane] >> (8 * chunk)) & 0xffu;
      for (int32_t bit = 0; bit < 8; ++bit)
        if (m & (1u << bit)) cols.push_back(iv * 8 + bit);
    }
  }
  std::sort(cols.begin(), cols.end());
  return cols;
}

double bvss_density_sample(int32_t n, const int32_t* row_ptr, const int32_t* cols,
                           int32_t rows) {
  uint64_t slices = 0, bits = 0;
  std::vector<int32_t> tmp;
  const int32_t lim = std::min(n, rows);
  for (int32_t r = 0; r < lim; ++r) {
    tmp.assign(cols + row_ptr[r], cols + row_ptr[r + 1]);
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    for (size_t i = 0; i < tmp.size();) {
      const int32_t iv = tmp[i] >> 3;
      while (i < tmp.size() && (tmp[i] >> 3) == iv) {
        ++bits;
        ++i;
      }
      ++slices;
    }
  }
  return slices ? static_cast<double>(bits) / static_cast<double>(slices) : 0.0;
}

}  // namespace cpg
