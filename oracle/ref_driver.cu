// Test infrastructure only: a driver for the reference gpu-cpg library, used to
// produce golden vectors and the reference timing beside this project's own
// numbers.  It links the reference's gpucpg/gpucpg.cu, compiled from the
// reference tree by oracle/Makefile (target `ref`) into oracle/_ref/.
//
// It calls the reference's public CpGen API exactly as the reference's own
// golden writer does (examples/tc-pfxt-gate5.cu:15-44: reset(), then
// report_paths(k, 10, true, LEVELIZE_THEN_RELAX, SHORT_LONG, false, 0.005f,
// 5.0f, 8, false, false, false, true, CsrReorderMethod::NONE, false), then
// get_slacks(k)), and writes costs with 9 significant digits like
// write_costs (examples/tc-pfxt-gate5.cu:63-72).
//
// Modes:
//   gpg   FILE K OUT [TRIALS]  G-PathGen (SHORT_LONG) costs; prints timing
//   seq   FILE K OUT           the reference's CPU SEQUENTIAL path
//                              (gpucpg.cu:21230-21300); prints expand_time
//   sfxt  FILE OUT             per-vertex "succ dist_fixed_point" lines
//   nodes FILE K OUT           "level from to slack" per returned GPG node
#include "gpucpg.cuh"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

using namespace std::chrono_literals;

namespace {

void run_gpg(gpucpg::CpGen& g, int k) {
  g.reset();
  g.report_paths(k, 10, true, gpucpg::PropDistMethod::LEVELIZE_THEN_RELAX,
                 gpucpg::PfxtExpMethod::SHORT_LONG, false, 0.005f, 5.0f, 8,
                 false, false, false, true, gpucpg::CsrReorderMethod::NONE,
                 false);
}

void run_seq(gpucpg::CpGen& g, int k) {
  g.reset();
  g.report_paths(k, 10, true, gpucpg::PropDistMethod::LEVELIZE_THEN_RELAX,
                 gpucpg::PfxtExpMethod::SEQUENTIAL, false, 0.005f, 5.0f, 8,
                 false, false, false, false, gpucpg::CsrReorderMethod::NONE,
                 false);
}

double step_sum_ms(const gpucpg::CpGen& g) {
  double ms = 0.0;
  for (const auto& t : g.short_long_step_times) ms += t / 1ms;
  return ms;
}

void write_costs(const std::string& path, const std::vector<float>& c) {
  std::ofstream os(path);
  os.precision(9);
  for (float x : c) os << x << '\n';
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: ref_driver gpg|seq|sfxt|nodes FILE ...\n");
    return 2;
  }
  const std::string mode = argv[1];
  const std::string file = argv[2];
  gpucpg::CpGen g;
  auto t0 = std::chrono::steady_clock::now();
  g.read_input(file);
  auto t1 = std::chrono::steady_clock::now();
  std::cout << "REFDRV read_input_ms="
            << std::chrono::duration<double, std::milli>(t1 - t0).count()
            << " N=" << g.num_verts() << " M=" << g.num_edges() << std::endl;

  if (mode == "gpg" || mode == "nodes") {
    const int k = std::atoi(argv[3]);
    const std::string out = argv[4];
    const int trials = (mode == "gpg" && argc > 5) ? std::atoi(argv[5]) : 1;
    for (int t = 0; t < trials; ++t) {
      run_gpg(g, k);
      std::cout << "REFDRV trial=" << t << " pfxt_step_ms=" << step_sum_ms(g)
                << " prop_ms=" << g.prop_time / 1ms
                << " expand_ms=" << g.expand_time / 1ms
                << " total_paths=" << g.total_gen_paths << std::endl;
    }
    if (mode == "gpg") {
      write_costs(out, g.get_slacks(k));
    } else {
      std::ofstream os(out);
      os.precision(9);
      for (const auto& n : g.get_pfxt_nodes(k))
        os << n.level << ' ' << n.from << ' ' << n.to << ' ' << n.slack << '\n';
    }
  } else if (mode == "seq") {
    const int k = std::atoi(argv[3]);
    const std::string out = argv[4];
    run_seq(g, k);
    std::cout << "REFDRV seq expand_ms=" << g.expand_time / 1ms
              << " prop_ms=" << g.prop_time / 1ms << std::endl;
    write_costs(out, g.get_slacks(k));
  } else if (mode == "sfxt") {
    const std::string out = argv[3];
    run_gpg(g, 1);
    std::stringstream succ_dist;
    g.dump_succ_dists(succ_dist);
    std::stringstream fixed;
    g.dump_sfxt_by_vertex(fixed);
    std::ofstream os(out);
    std::string l1, l2;
    while (std::getline(succ_dist, l1) && std::getline(fixed, l2)) {
      int succ = 0;
      float unused = 0.f;
      std::istringstream(l1) >> succ >> unused;
      long long idx = 0;
      double d = 0.0;
      std::istringstream(l2) >> idx >> d;
      os << succ << ' ' << std::llround(d * 10000.0) << '\n';
    }
  } else {
    std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
  }
  return 0;
}
