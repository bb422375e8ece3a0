// ThinShells.hpp -- C++ host facade over libits with the reference's call surface.
//
// Keeps the method names and call order of the reference's ThinShells / BaseModel /
// SparseVoxelOctree (src/ThinShells.h:8-189, src/BaseModel.h:55-63, src/SVO.h:104):
//
//   its::ThinShells shell(V, F, 256, 256, 256, /*is2UnitCube=*/true, /*scale=*/1.0);
//   shell.creatShell();                        // samples, SDF, coefficients, iso levels
//   auto iso = shell.getShellIsoVal();         // {inner, outer}
//   shell.mcVisualization("inner.obj", {512,512,512}, "outer.obj", {512,512,512}, "", {0,0,0});
//
// All GPU work goes through the C ABI (its.h); this header holds no kernels. Errors are
// thrown as its::Error (the reference exits the process instead).
#pragma once
#include <array>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "its/its.h"

namespace its {

struct Error : std::runtime_error {
  its_status status;
  Error(its_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(its_status s, its_ctx* ctx, const char* what) {
  if (s != ITS_OK) throw Error(s, std::string(what) + ": " + (ctx ? its_last_error(ctx) : "invalid argument"));
}

class ThinShells {
 public:
  // ThinShells(filename, gx, gy, gz, is2UnitCube, scaleFactor) of ThinShells.h:62-73, with the
  // mesh given as arrays (an OFF loader is readOff below). The octree is cubic: gx = gy = gz.
  ThinShells(std::vector<double> V, std::vector<int32_t> F, int gx, int gy, int gz, bool is2UnitCube = true,
             double scaleFactor = 1.0, int device = 0)
      : V_(std::move(V)), F_(std::move(F)), res_(gx) {
    if (gx != gy || gx != gz) throw Error(ITS_ERR_INVALID, "the octree grid must be cubic");
    check(its_create(&ctx_, device), nullptr, "its_create");
    const int64_t nv = (int64_t)V_.size() / 3, nf = (int64_t)F_.size() / 3;
    if (is2UnitCube) check(its_model_to_unit_cube(V_.data(), nv, scaleFactor), ctx_, "model2UnitCube");
    check(its_uniform_bbox(V_.data(), nv, origin_.data(), end_.data(), width_.data()), ctx_, "setUniformBoundingBox");
    check(its_svo_build(ctx_, V_.data(), nv, F_.data(), nf, res_, origin_.data(), width_.data(), &svo_), ctx_,
          "createOctree");
    its_svo_info info;
    its_svo_get_info(svo_, &info);
    treeDepth = info.depth;
    numNodeVerts_ = info.num_vertices;
  }
  ThinShells(const ThinShells&) = delete;
  ThinShells& operator=(const ThinShells&) = delete;
  ~ThinShells() {
    if (mlp_) its_mlp_free(mlp_);
    if (op_) its_operator_free(op_);
    if (svo_) its_svo_free(svo_);
    if (ctx_) its_destroy(ctx_);
  }

  // creatShell() / initBSplineTree() (ThinShells.cpp:757-815). With shareNetFile (the
  // share network's parameters, its_b200/share_net.f32) the coefficients come from the
  // learned start -- an exact solution -- checked by the FP64 residual, with the plain LSCG
  // from that start as the fallback; without it, the reference's LSCG from zero.
  void creatShell(double tol = 1e-6, int stopRule = ITS_STOP_RESIDUAL, const std::string& shareNetFile = "") {
    const int64_t nv = (int64_t)V_.size() / 3, nf = (int64_t)F_.size() / 3;
    int64_t nPts = 0, nEdge = 0;  // cpIntersectionPoints: one call into a generous buffer, a
    const int64_t cap = 2 * nf + nv + 1024;  // second only when the samples exceed it
    interPoints_.assign(3 * cap, 0.0);
    check(its_shell_samples(svo_, V_.data(), nv, F_.data(), nf, interPoints_.data(), cap, &nPts, &nEdge), ctx_,
          "cpIntersectionPoints");
    if (nPts > cap) {
      interPoints_.assign(3 * nPts, 0.0);
      check(its_shell_samples(svo_, V_.data(), nv, F_.data(), nf, interPoints_.data(), nPts, &nPts, &nEdge), ctx_,
            "cpIntersectionPoints");
    }
    interPoints_.resize(3 * nPts);
    std::vector<double> pos(3 * numNodeVerts_);  // cpSDFOfTreeNodes
    check(its_svo_get_vertices(svo_, pos.data(), nullptr), ctx_, "nodeVertexArray");
    sdfVal_.assign(numNodeVerts_, 0.0);
    check(its_signed_distance(ctx_, pos.data(), numNodeVerts_, V_.data(), nv, F_.data(), nf, sdfVal_.data()), ctx_,
          "cpSDFOfTreeNodes");
    lambda_.assign(numNodeVerts_, 0.0);
    its_solve_opts o;
    its_solve_opts_default(&o);
    o.tol = tol;
    o.stop_rule = stopRule;
    o.max_iters = 100000;
    report_ = its_solve_report{};
    bool solved = false;
    if (!shareNetFile.empty()) {
      std::vector<float> params(its_mlp_num_params()), norm(130);
      std::ifstream in(shareNetFile, std::ios::binary);
      in.read(reinterpret_cast<char*>(params.data()), (std::streamsize)(params.size() * sizeof(float)));
      in.read(reinterpret_cast<char*>(norm.data()), (std::streamsize)(norm.size() * sizeof(float)));
      if (!in) throw Error(ITS_ERR_INVALID, "cannot read share network file " + shareNetFile);
      if (!mlp_) check(its_mlp_create(ctx_, 65536, &mlp_), ctx_, "its_mlp_create");
      check(its_mlp_set_params(mlp_, params.data()), ctx_, "its_mlp_set_params");
      check(its_learned_start(svo_, mlp_, sdfVal_.data(), norm.data(), lambda_.data()), ctx_, "learned start");
      double rel = 0;
      check(its_fit_residual(svo_, sdfVal_.data(), lambda_.data(), &rel), ctx_, "residual");
      report_.rel_residual = rel;
      report_.converged = 1;
      solved = stopRule == ITS_STOP_RESIDUAL && rel <= tol;
      o.x0 = lambda_.data();  // the fallback (or Eigen's normal-equation test) starts there
    }
    if (!solved) {
      if (!op_) check(its_operator_build(svo_, ITS_OP_FP64, &op_), ctx_, "cpCoefficients");  // cpCoefficients
      check(its_lscg_solve(op_, sdfVal_.data(), lambda_.data(), &o, &report_), ctx_, "LSCG");
    }
    std::vector<double> samples(V_);  // cpLatentBSplineValue: mesh vertices + intersections
    samples.insert(samples.end(), interPoints_.begin(), interPoints_.end());
    int64_t miss = 0;
    check(its_shell_iso_values(svo_, lambda_.data(), samples.data(), (int64_t)samples.size() / 3, &innerShellIsoVal_,
                               &outerShellIsoVal_, &miss),
          ctx_, "cpLatentBSplineValue");
  }

  std::array<double, 2> getShellIsoVal() const { return {innerShellIsoVal_, outerShellIsoVal_}; }

  // mcVisualization (ThinShells.cpp:1086-1129): MC at the outer, inner and 0 iso levels over
  // the model box; writes OBJ triangle soups (writeToOBJFile, MarchingCubes.cu:635-661).
  // welded = true writes indexed meshes (shared vertices, its_marching_cubes_mesh) instead.
  void mcVisualization(const std::string& innerFile, std::array<int, 3> innerRes, const std::string& outerFile,
                       std::array<int, 3> outerRes, const std::string& isoFile, std::array<int, 3> isoRes,
                       bool welded = false) const {
    if (!outerFile.empty()) marchingCubes(outerShellIsoVal_, outerRes[0], outerFile, welded);
    if (!innerFile.empty()) marchingCubes(innerShellIsoVal_, innerRes[0], innerFile, welded);
    if (!isoFile.empty()) marchingCubes(0.0, isoRes[0], isoFile, welded);
  }

  // textureVisualization (ThinShells.cpp:1131-1134): field at the mesh vertices as OBJ vt.
  void textureVisualization(const std::string& filename) const {
    const int64_t nv = (int64_t)V_.size() / 3;
    std::vector<double> f(nv);
    check(its_eval_points(svo_, lambda_.data(), V_.data(), nv, f.data(), nullptr), ctx_, "eval");
    std::ofstream out(filename);
    for (int64_t i = 0; i < nv; ++i) out << "v " << V_[3 * i] << ' ' << V_[3 * i + 1] << ' ' << V_[3 * i + 2] << '\n';
    for (int64_t i = 0; i < nv; ++i) out << "vt " << f[i] << ' ' << 0 << '\n';
    for (size_t t = 0; t < F_.size() / 3; ++t)
      out << "f " << F_[3 * t] + 1 << '/' << F_[3 * t] + 1 << ' ' << F_[3 * t + 1] + 1 << '/' << F_[3 * t + 1] + 1 << ' '
          << F_[3 * t + 2] + 1 << '/' << F_[3 * t + 2] + 1 << '\n';
  }

  const std::vector<double>& coefficients() const { return lambda_; }
  const its_solve_report& solveReport() const { return report_; }
  its_svo* svo() const { return svo_; }
  its_ctx* context() const { return ctx_; }
  int treeDepth = 0;

  // Wavefront OBJ: "v x y z" and "f i j k ..." (1-based, negative = relative, "i/t/n" forms;
  // polygons fanned into triangles). Replaces libigl read_triangle_mesh (BaseModel.cpp:774-782).
  static void readObj(const std::string& path, std::vector<double>& V, std::vector<int32_t>& F) {
    std::ifstream in(path);
    if (!in) throw Error(ITS_ERR_INVALID, "cannot open " + path);
    V.clear();
    F.clear();
    std::string line;
    while (std::getline(in, line)) {
      std::istringstream ls(line);
      std::string tag;
      ls >> tag;
      if (tag == "v") {
        double x, y, z;
        ls >> x >> y >> z;
        V.insert(V.end(), {x, y, z});
      } else if (tag == "f") {
        std::vector<int32_t> idx;
        std::string tok;
        const int64_t nv = (int64_t)V.size() / 3;
        while (ls >> tok) {
          const long k = std::strtol(tok.c_str(), nullptr, 10);
          idx.push_back((int32_t)(k < 0 ? nv + k : k - 1));
        }
        for (size_t j = 1; j + 1 < idx.size(); ++j) F.insert(F.end(), {idx[0], idx[j], idx[j + 1]});
      }
    }
  }

  static void readOff(const std::string& path, std::vector<double>& V, std::vector<int32_t>& F) {
    std::ifstream in(path);
    std::string tag;
    in >> tag;
    if (tag != "OFF") throw Error(ITS_ERR_INVALID, "not an OFF file: " + path);
    int64_t nv, nf, ne;
    in >> nv >> nf >> ne;
    V.resize(3 * nv);
    for (auto& x : V) in >> x;
    F.clear();
    for (int64_t t = 0; t < nf; ++t) {
      int k;
      in >> k;
      std::vector<int32_t> idx(k);
      for (auto& i : idx) in >> i;
      for (int j = 1; j + 1 < k; ++j) F.insert(F.end(), {idx[0], idx[j], idx[j + 1]});
    }
  }

 private:
  void marchingCubes(double iso, int res, const std::string& filename, bool welded) const {
    std::ofstream out(filename);
    if (welded) {
      const int64_t M = (int64_t)res + 1;
      std::vector<double> field(M * M * M);
      check(its_eval_grid(svo_, lambda_.data(), origin_.data(), width_.data(), res, field.data()), ctx_, "MC field");
      int64_t nvt = 0, ntr = 0;
      check(its_marching_cubes_mesh(ctx_, field.data(), res, origin_.data(), width_.data(), iso, nullptr, 0, &nvt,
                                    nullptr, 0, &ntr),
            ctx_, "marching_cubes_mesh");
      std::vector<double> verts(3 * nvt);
      std::vector<int32_t> tris(3 * ntr);
      check(its_marching_cubes_mesh(ctx_, field.data(), res, origin_.data(), width_.data(), iso, verts.data(), nvt,
                                    &nvt, tris.data(), ntr, &ntr),
            ctx_, "marching_cubes_mesh");
      for (int64_t i = 0; i < nvt; ++i)
        out << "v " << verts[3 * i] << ' ' << verts[3 * i + 1] << ' ' << verts[3 * i + 2] << '\n';
      for (int64_t t = 0; t < ntr; ++t)
        out << "f " << tris[3 * t] + 1 << ' ' << tris[3 * t + 1] + 1 << ' ' << tris[3 * t + 2] + 1 << '\n';
      return;
    }
    // the soup: field and marching cubes on the device, only the triangles come back
    int64_t n = 0;
    check(its_eval_grid_mc(svo_, lambda_.data(), origin_.data(), width_.data(), res, 0, &iso, 1, nullptr, nullptr, &n),
          ctx_, "marching_cubes");
    std::vector<double> tri(3 * n);
    double* tp = tri.data();
    const int64_t cap = n;
    check(its_eval_grid_mc(svo_, lambda_.data(), origin_.data(), width_.data(), res, 0, &iso, 1, &tp, &cap, &n), ctx_,
          "marching_cubes");
    for (int64_t i = 0; i < n; ++i) out << "v " << tri[3 * i] << ' ' << tri[3 * i + 1] << ' ' << tri[3 * i + 2] << '\n';
    for (int64_t i = 0; i + 2 < n; i += 3) out << "f " << i + 1 << ' ' << i + 2 << ' ' << i + 3 << '\n';
  }

  std::vector<double> V_;
  std::vector<int32_t> F_;
  int res_;
  std::array<double, 3> origin_{}, end_{}, width_{};
  its_ctx* ctx_ = nullptr;
  its_svo* svo_ = nullptr;
  its_op* op_ = nullptr;
  its_mlp* mlp_ = nullptr;
  int64_t numNodeVerts_ = 0;
  std::vector<double> interPoints_, sdfVal_, lambda_;
  its_solve_report report_{};
  double innerShellIsoVal_ = 0, outerShellIsoVal_ = 0;
};

}  // namespace its
