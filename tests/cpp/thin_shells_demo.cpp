// Drives the C++ facade in the reference's call order on an OFF mesh and prints the
// octree depth, solve report and iso levels as one JSON line (used by tests/test_cpp_facade.py).
#include <cstdio>

#include "its/ThinShells.hpp"

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s mesh.off|mesh.obj res out_prefix [share_net.f32]\n", argv[0]);
    return 2;
  }
  std::vector<double> V;
  std::vector<int32_t> F;
  const std::string path = argv[1];
  if (path.size() > 4 && path.substr(path.size() - 4) == ".obj") its::ThinShells::readObj(path, V, F);
  else its::ThinShells::readOff(path, V, F);
  const int res = std::atoi(argv[2]);
  its::ThinShells shell(V, F, res, res, res, true, 1.0);
  if (argc > 4) shell.creatShell(1e-6, ITS_STOP_RESIDUAL, argv[4]);  // learned start
  else shell.creatShell(1e-10, ITS_STOP_NORMAL);
  const auto iso = shell.getShellIsoVal();
  const std::string pre = argv[3];
  shell.mcVisualization(pre + "_inner.obj", {2 * res, 2 * res, 2 * res}, pre + "_outer.obj", {2 * res, 2 * res, 2 * res},
                        "", {0, 0, 0});
  shell.mcVisualization("", {0, 0, 0}, pre + "_outer_welded.obj", {2 * res, 2 * res, 2 * res}, "", {0, 0, 0}, true);
  const its_solve_report& r = shell.solveReport();
  std::printf("{\"depth\": %d, \"iterations\": %lld, \"converged\": %d, \"rel_residual\": %.17g, \"inner\": %.17g, "
              "\"outer\": %.17g}\n",
              shell.treeDepth, (long long)r.iterations, r.converged, r.rel_residual, iso[0], iso[1]);
  return 0;
}
