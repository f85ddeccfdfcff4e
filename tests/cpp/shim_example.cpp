// A reference-style caller (the shape of examples/tc-pfxt-gate5.cu:15-44)
// compiled against the C++ shim.  Built by tests: syntax-checked on CPU,
// linked and run against libcpg_b200.so on a GPU.
#include <cstdio>
#include <cstdlib>

#include "gpucpg/cpgen.hpp"

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: shim_example GRAPH K\n");
    return 2;
  }
  try {
    gpucpg::CpGen cpgen;
    cpgen.read_input(argv[1]);
    const int k = std::atoi(argv[2]);
    cpgen.reset();
    cpgen.report_paths(k, 10, true, gpucpg::PropDistMethod::LEVELIZE_THEN_RELAX,
                       gpucpg::PfxtExpMethod::SHORT_LONG, false, 0.005f, 5.0f, 8,
                       false, false, false, true, gpucpg::CsrReorderMethod::NONE,
                       false);
    for (float c : cpgen.get_slacks(k)) std::printf("%.9g\n", c);
    const auto nodes = cpgen.get_pfxt_nodes(k);
    std::fprintf(stderr, "nodes=%zu verts=%zu edges=%zu\n", nodes.size(),
                 cpgen.num_verts(), cpgen.num_edges());
  } catch (const gpucpg::CpgError& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
