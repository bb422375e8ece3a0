// Drives the C++ facade in the reference's call order on an OFF mesh and prints the
// octree depth, solve report and iso levels as one JSON line (used by tests/test_cpp_facade.py).
#include <cstdio>

#include "its/ThinShells.hpp"

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s mesh.off res out_prefix\n", argv[0]);
    return 2;
  }
  std::vector<double> V;
  std::vector<int32_t> F;
  its::ThinShells::readOff(argv[1], V, F);
  const int res = std::atoi(argv[2]);
  its::ThinShells shell(V, F, res, res, res, true, 1.0);
  shell.creatShell(1e-10, ITS_STOP_NORMAL);
  const auto iso = shell.getShellIsoVal();
  const std::string pre = argv[3];
  shell.mcVisualization(pre + "_inner.obj", {2 * res, 2 * res, 2 * res}, pre + "_outer.obj", {2 * res, 2 * res, 2 * res},
                        "", {0, 0, 0});
  const its_solve_report& r = shell.solveReport();
  std::printf("{\"depth\": %d, \"iterations\": %lld, \"converged\": %d, \"inner\": %.17g, \"outer\": %.17g}\n",
              shell.treeDepth, (long long)r.iterations, r.converged, iso[0], iso[1]);
  return 0;
}
