// Header-only C++ shim: the reference's gpucpg::CpGen surface
// (gpucpg/gpucpg.cuh:119-431) rebuilt over the C ABI of libcpg_b200.so.
// Callers of the reference keep their code: read_input, levelize,
// report_paths(k, ...), get_slacks, get_pfxt_nodes, reset, num_verts,
// num_edges, and the prop_time / expand_time fields.  Errors that the
// reference turned into exit(1) or std::runtime_error become
// gpucpg::CpgError exceptions on the C++ side (the ABI itself never throws).
#pragma once

#include <chrono>
#include <cstdint>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../cpg.h"

namespace gpucpg {

// Same enumerators as the reference (gpucpg.cuh:41-72).  The B200 path always
// runs levelize-then-relax with the G-PathGen result set; other values are
// accepted so existing call sites compile.
enum class PropDistMethod { BASIC = 0, CUDA_GRAPH, BFS_TOP_DOWN_PRIVATIZED, BFS_TOP_DOWN,
  BFS_PRIVATIZED_MERGED, BFS_HYBRID, BFS_HYBRID_PRIVATIZED, TEST_COUNT_MF,
  LEVELIZE_THEN_RELAX, LEVELIZE_HYBRID_THEN_RELAX, BFS_TD_RELAX_BU_PRIVATIZED };
enum class PfxtExpMethod { BASIC = 0, PRECOMP_SPURS, ATOMIC_ENQ, SHORT_LONG, SEQUENTIAL };
enum class CsrReorderMethod { NONE = -1, V_ORIENTED = 0, V_ORIENTED_TILE_SCAN, E_ORIENTED,
  E_ORIENTED_VEC2, RABBIT, GORDER, CORDER };

// PfxtNode (gpucpg.cuh:74-107): same fields, same order.
using PfxtNode = cpg_path_node;

class CpgError : public std::runtime_error {
 public:
  CpgError(cpg_status s, const std::string& what)
      : std::runtime_error(what), status(s) {}
  cpg_status status;
};

class CpGen {
 public:
  explicit CpGen(const cpg_options* opts = nullptr) {
    check(cpg_create(&h_, opts), "cpg_create");
  }
  ~CpGen() { if (h_) cpg_destroy(h_); }
  CpGen(const CpGen&) = delete;
  CpGen& operator=(const CpGen&) = delete;

  void read_input(const std::string& filename, bool ignore_wgts = false) {
    check(cpg_load_text(h_, filename.c_str(), ignore_wgts ? 1 : 0), "read_input");
  }
  void levelize() { check(cpg_levelize(h_), "levelize"); }

  void report_paths(int k, int /*max_dev_lvls*/ = 10, bool /*enable_compress*/ = true,
                    PropDistMethod = PropDistMethod::LEVELIZE_THEN_RELAX,
                    PfxtExpMethod = PfxtExpMethod::SHORT_LONG,
                    bool = false, float = 0.005f, float = 5.0f, int = 8,
                    bool = false, bool = false, bool = false, bool = false,
                    CsrReorderMethod = CsrReorderMethod::NONE, bool = false,
                    std::optional<float> = std::nullopt,
                    std::optional<std::string> = std::nullopt) {
    const auto t0 = std::chrono::steady_clock::now();
    check(cpg_report_paths(h_, k), "report_paths");
    const auto t1 = std::chrono::steady_clock::now();
    cpg_stats s{};
    cpg_get_stats(h_, &s);
    prop_time = std::chrono::duration<double, std::micro>(s.sfxt_ms * 1000.0);
    expand_time = std::chrono::duration<double, std::micro>(t1 - t0) - prop_time;
    total_gen_paths = static_cast<int>(s.paths_accepted);
  }

  std::vector<float> get_slacks(int k) {
    std::vector<float> out(k > 0 ? k : 0);
    int64_t n = 0;
    check(cpg_get_costs(h_, k, out.data(), &n), "get_slacks");
    out.resize(static_cast<size_t>(n));
    return out;
  }

  std::vector<PfxtNode> get_pfxt_nodes(int k) {
    std::vector<PfxtNode> out(k > 0 ? k : 0);
    int64_t n = 0;
    check(cpg_get_paths(h_, k, out.data(), &n), "get_pfxt_nodes");
    out.resize(static_cast<size_t>(n));
    return out;
  }

  void reset() { check(cpg_reset(h_), "reset"); }
  size_t num_verts() const { return static_cast<size_t>(cpg_num_verts(h_)); }
  size_t num_edges() const { return static_cast<size_t>(cpg_num_edges(h_)); }
  cpg_handle* handle() { return h_; }

  std::chrono::duration<double, std::micro> prop_time{0};
  std::chrono::duration<double, std::micro> expand_time{0};
  int total_gen_paths{0};

 private:
  void check(cpg_status s, const char* what) {
    if (s != CPG_OK)
      throw CpgError(s, std::string(what) + ": " + cpg_status_string(s) + ": " +
                            (h_ ? cpg_last_error(h_) : ""));
  }
  cpg_handle* h_ = nullptr;
};

}  // namespace gpucpg
