// CPU oracle (test infrastructure): flat extern "C" surface loaded by tests/ and
// bench.py's CPU-baseline leg through ctypes (oracle/__init__.py).
#include <cstring>
#include <new>

#include "orc_fit.hpp"

using namespace orc;

namespace {
struct Points { std::vector<V3> pts; size_t nEdge = 0; };
}

extern "C" {

void orc_model_to_unit_cube(double* V, int64_t nv, double scale) { modelToUnitCube(V, nv, scale); }
void orc_uniform_bbox(const double* V, int64_t nv, double* o, double* e, double* w) { uniformBBox(V, nv, o, e, w); }
void orc_tri_attributes(const double* V, const int32_t* F, int64_t nf, double* n, double* a, double* d) {
  triAttributes(V, F, nf, n, a, d);
}
void orc_morton_encode(const uint32_t* xyz, int64_t n, uint32_t* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = mortonEncode(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
}
void orc_morton_decode(const uint32_t* m, int64_t n, uint32_t* xyz) {
  for (int64_t i = 0; i < n; ++i) mortonDecode(m[i], xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
}
// The hat basis at single points: value (baseFunction4Point) and gradient as
// de_BaseFunction4Point forms it (BSpline.hpp:37-57), for the known-answer pin against the
// reference's own BSpline.hpp.
void orc_hat(const double* p, const double* w, const double* q, int64_t n, double* val, double* grad) {
  for (int64_t i = 0; i < n; ++i) {
    const V3 c{p[3 * i], p[3 * i + 1], p[3 * i + 2]}, x{q[3 * i], q[3 * i + 1], q[3 * i + 2]};
    const double wd = w[i];
    val[i] = baseFunction4Point(c, wd, x);
    const double bx = baseFunction(x.x, c.x, wd), by = baseFunction(x.y, c.y, wd), bz = baseFunction(x.z, c.z, wd);
    grad[3 * i] = deBaseFunction(x.x, c.x, wd) * by * bz;
    grad[3 * i + 1] = bx * deBaseFunction(x.y, c.y, wd) * bz;
    grad[3 * i + 2] = bx * by * deBaseFunction(x.z, c.z, wd);
  }
}

void orc_luts(int16_t* parent, int16_t* child, int16_t* vert, int16_t* edge) {
  short p[8][27], c[8][27], v[64], e[48];
  neighborLUTs(p, c);
  vertSharedLUT(v);
  edgeSharedLUT(e);
  std::memcpy(parent, p, sizeof(p));
  std::memcpy(child, c, sizeof(c));
  std::memcpy(vert, v, sizeof(v));
  std::memcpy(edge, e, sizeof(e));
}

void* orc_svo_build(const double* V, int64_t nv, const int32_t* F, int64_t nf, int res, const double* origin,
                    const double* width) {
  return new Svo(buildSvo(V, nv, F, nf, res, origin, width));
}
void orc_svo_free(void* h) { delete static_cast<Svo*>(h); }
// out: depth, voxels, fine nodes, tree nodes, vertices, edges
void orc_svo_counts(void* h, int64_t* out) {
  const Svo& s = *static_cast<Svo*>(h);
  out[0] = s.treeDepth; out[1] = (int64_t)s.numVoxels; out[2] = (int64_t)s.numFineNodes;
  out[3] = (int64_t)s.numTreeNodes; out[4] = (int64_t)s.numVerts; out[5] = (int64_t)s.edges.size();
}
void orc_svo_depth_counts(void* h, int64_t* nodes, int64_t* verts) {
  const Svo& s = *static_cast<Svo*>(h);
  for (int d = 0; d < s.treeDepth; ++d) {
    nodes[d] = (int64_t)s.depthNumNodes[d];
    verts[d] = (int64_t)s.depthVerts[d].size();
  }
}
void orc_svo_voxels(void* h, uint32_t* out) {
  const Svo& s = *static_cast<Svo*>(h);
  std::memcpy(out, s.voxels.data(), s.voxels.size() * sizeof(uint32_t));
}
void orc_svo_nodes(void* h, uint32_t* morton, uint32_t* parent, uint32_t* childs, uint8_t* isLeaf, double* origin,
                   double* width, uint32_t* nb) {
  const Svo& s = *static_cast<Svo*>(h);
  for (size_t i = 0; i < s.nodes.size(); ++i) {
    const Node& n = s.nodes[i];
    if (morton) morton[i] = n.morton;
    if (parent) parent[i] = n.parent;
    if (childs) for (int k = 0; k < 8; ++k) childs[8 * i + k] = n.childs[k];
    if (isLeaf) isLeaf[i] = n.isLeaf ? 1 : 0;
    if (origin) { origin[3 * i] = n.origin.x; origin[3 * i + 1] = n.origin.y; origin[3 * i + 2] = n.origin.z; }
    if (width) width[i] = n.width;
    if (nb) for (int k = 0; k < 27; ++k) nb[27 * i + k] = n.nb[k];
  }
}
void orc_svo_vertices(void* h, double* pos, uint32_t* owner) {
  const Svo& s = *static_cast<Svo*>(h);
  size_t i = 0;
  for (int d = 0; d < s.treeDepth; ++d)
    for (const VertexRec& v : s.depthVerts[d]) {
      if (pos) { pos[3 * i] = v.pos.x; pos[3 * i + 1] = v.pos.y; pos[3 * i + 2] = v.pos.z; }
      if (owner) owner[i] = v.owner;
      ++i;
    }
}
void orc_svo_edges(void* h, double* p0, double* p1, uint32_t* owner) {
  const Svo& s = *static_cast<Svo*>(h);
  for (size_t i = 0; i < s.edges.size(); ++i) {
    const EdgeRec& e = s.edges[i];
    if (p0) { p0[3 * i] = e.p0.x; p0[3 * i + 1] = e.p0.y; p0[3 * i + 2] = e.p0.z; }
    if (p1) { p1[3 * i] = e.p1.x; p1[3 * i + 1] = e.p1.y; p1[3 * i + 2] = e.p1.z; }
    if (owner) owner[i] = e.owner;
  }
}

void* orc_assemble(void* h) { return new Csr(assemble(*static_cast<Svo*>(h))); }
int64_t orc_csr_rows(void* a) { return static_cast<Csr*>(a)->n; }
int64_t orc_csr_nnz(void* a) { return (int64_t)static_cast<Csr*>(a)->col.size(); }
void orc_csr_get(void* a, int64_t* rowptr, int32_t* col, double* val) {
  const Csr& A = *static_cast<Csr*>(a);
  if (rowptr) std::memcpy(rowptr, A.rowptr.data(), A.rowptr.size() * sizeof(int64_t));
  if (col) std::memcpy(col, A.col.data(), A.col.size() * sizeof(int32_t));
  if (val) std::memcpy(val, A.val.data(), A.val.size() * sizeof(double));
}
void* orc_csr_from(int64_t n, const int64_t* rowptr, const int32_t* col, const double* val) {
  Csr* A = new Csr;
  A->n = n;
  A->rowptr.assign(rowptr, rowptr + n + 1);
  A->col.assign(col, col + rowptr[n]);
  A->val.assign(val, val + rowptr[n]);
  return A;
}
void orc_csr_free(void* a) { delete static_cast<Csr*>(a); }
// report: iterations, converged, breakdown, rel_residual, normal_rel_residual
int orc_cgls(void* a, const double* b, double* x, double tol, int64_t maxIters, int stop, double* report) {
  const Csr& A = *static_cast<Csr*>(a);
  const Csr T = transpose(A);
  CglsReport r = cgls(A, T, b, x, tol, maxIters, stop);
  if (report) {
    report[0] = (double)r.iterations; report[1] = r.converged; report[2] = r.breakdown;
    report[3] = r.rel_residual; report[4] = r.normal_rel_residual;
  }
  return r.converged ? 0 : 1;
}

void orc_exact_start(void* h, void* a, const double* b, const double* shares, double* lambda) {
  exactStart(*static_cast<Svo*>(h), *static_cast<Csr*>(a), b, shares, lambda);
}

void orc_exact_start_surplus(void* h, void* a, const double* b, const double* shares, double* lambda) {
  exactStartSurplus(*static_cast<Svo*>(h), *static_cast<Csr*>(a), b, shares, lambda);
}

void orc_point_gradient(void* h, const double* lambda, const double* P, const double* before, int64_t m,
                        const double* boxOrigin, const double* boxEnd, double* val, double* grad, uint8_t* missing) {
  pointValGradient(*static_cast<Svo*>(h), lambda, P, before, m, boxOrigin, boxEnd, val, grad, missing);
}

void* orc_intersections(void* h, const double* V, int64_t nv, const int32_t* F, int64_t nf) {
  Points* p = new Points;
  p->pts = intersections(*static_cast<Svo*>(h), V, nv, F, nf, &p->nEdge);
  return p;
}
int64_t orc_points_count(void* p, int64_t* nEdge) {
  if (nEdge) *nEdge = (int64_t)static_cast<Points*>(p)->nEdge;
  return (int64_t)static_cast<Points*>(p)->pts.size();
}
void orc_points_get(void* p, double* out) {
  const auto& v = static_cast<Points*>(p)->pts;
  for (size_t i = 0; i < v.size(); ++i) { out[3 * i] = v[i].x; out[3 * i + 1] = v[i].y; out[3 * i + 2] = v[i].z; }
}
void orc_points_free(void* p) { delete static_cast<Points*>(p); }

void orc_signed_distance(const double* P, int64_t m, const double* V, const int32_t* F, int64_t nf, double* out) {
  signedDistance(P, m, V, F, nf, out);
}
void* orc_cubic_assemble(void* h, const double* samples, int64_t m) {
  return new Csr(cubicAssemble(*static_cast<Svo*>(h), samples, m));
}
void orc_cubic_eval(void* h, const double* lambda, const double* P, int64_t m, double* out) {
  cubicEval(*static_cast<Svo*>(h), lambda, P, m, out);
}
void orc_cubic_eval_grid(void* h, const double* lambda, const double* origin, const double* width, int R,
                         double* out) {
  cubicEvalGrid(*static_cast<Svo*>(h), lambda, origin, width, R, out);
}
void orc_offset_samples(const double* V, int64_t nv, const int32_t* F, int64_t nf, double eps, double* pts,
                        double* tgt) {
  offsetSamples(V, nv, F, nf, eps, pts, tgt);
}
void orc_bspline3(const double* t, int64_t n, double* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = bspline3(t[i]);
}
void orc_signed_distance_bvh(const double* P, int64_t m, const double* V, const int32_t* F, int64_t nf,
                             double* out) {
  signedDistanceBvh(P, m, V, F, nf, out);
}
void orc_eval_points(void* h, const double* lambda, const double* P, int64_t m, double* out, uint8_t* missing) {
  evalPoints(*static_cast<Svo*>(h), lambda, P, m, out, missing);
}
void orc_eval_brute(void* h, const double* lambda, const double* P, int64_t m, double* out) {
  evalBrute(*static_cast<Svo*>(h), lambda, P, m, out);
}
void orc_eval_grid(void* h, const double* lambda, const double* origin, const double* width, int R, double* out) {
  evalGrid(*static_cast<Svo*>(h), lambda, origin, width, R, out);
}
// Two calls: with verts/tris NULL the counts; then the arrays.
void orc_marching_cubes_mesh(const double* field, int R, const double* origin, const double* width, double iso,
                             double* verts, int32_t* tris, int64_t* counts) {
  std::vector<double> v;
  std::vector<int32_t> t;
  marchingCubesMesh(field, R, origin, width, iso, v, t);
  counts[0] = (int64_t)(v.size() / 3);
  counts[1] = (int64_t)(t.size() / 3);
  if (verts) std::memcpy(verts, v.data(), v.size() * sizeof(double));
  if (tris) std::memcpy(tris, t.data(), t.size() * sizeof(int32_t));
}
void orc_point_query(void* h, const double* lambda, const double* P, int64_t m, const double* boxOrigin,
                     const double* boxEnd, double inner, double outer, double* values, int8_t* labels) {
  pointQuery(*static_cast<Svo*>(h), lambda, P, m, boxOrigin, boxEnd, inner, outer, values, labels);
}
int64_t orc_marching_cubes(const double* field, int R, const double* origin, const double* width, double iso,
                           uint8_t* cube, double* tri, int64_t maxVerts) {
  return marchingCubes(field, R, origin, width, iso, cube, tri, maxVerts);
}

}  // extern "C"
