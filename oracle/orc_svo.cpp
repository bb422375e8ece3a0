// CPU oracle (test infrastructure): model pre-processing and the sparse voxel octree.
// Restates BaseModel.cpp:24-92, CUDACompute.cu:79-96 and SVO.cu:366-1110 of the
// reference on the CPU. See orc_common.hpp for the arithmetic conventions.
#include "orc_svo.hpp"

#include <algorithm>
#include <cstring>
#include <stdexcept>

namespace orc {

// BaseModel::calcUnitCubeTransformMatrix + model2UnitCube (BaseModel.cpp:54-92).
void modelToUnitCube(double* V, int64_t nv, double scaleFactor) {
  if (nv <= 0) return;
  V3 bmin{V[0], V[1], V[2]}, bmax = bmin;
  for (int64_t i = 1; i < nv; ++i)
    for (int a = 0; a < 3; ++a) {
      bmin[a] = std::min(bmin[a], V[3 * i + a]);
      bmax[a] = std::max(bmax[a], V[3 * i + a]);
    }
  double scale = bmax[0] - bmin[0];
  for (int d = 1; d < 3; ++d) scale = std::max<double>(scale, bmax[d] - bmin[d]);
  scale *= scaleFactor;
  V3 center;
  for (int a = 0; a < 3; ++a) center[a] = 0.5 * bmax[a] + 0.5 * bmin[a];
  for (int a = 0; a < 3; ++a) center[a] -= scale / 2;
  const double inv = 1. / scale;
  for (int64_t i = 0; i < nv; ++i)
    for (int a = 0; a < 3; ++a) V[3 * i + a] = (V[3 * i + a] + (-center[a])) * inv;
}

// BaseModel::setUniformBoundingBox (BaseModel.cpp:24-51): cubic box, the short axes
// padded by a FLOAT delta, then every side padded by width/11.
void uniformBBox(const double* V, int64_t nv, double origin[3], double end[3], double width[3]) {
  V3 mn{V[0], V[1], V[2]}, mx = mn;
  for (int64_t i = 1; i < nv; ++i)
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], V[3 * i + a]);
      mx[a] = std::max(mx[a], V[3 * i + a]);
    }
  V3 o = mn, e = mx, len = mx - mn;
  float maxLen = (float)dmax(len.x, dmax(len.y, len.z));
  for (int a = 0; a < 3; ++a) {
    if ((double)maxLen == len[a]) continue;
    float delta = (float)((double)maxLen - len[a]);
    o[a] = mn[a] - (double)(delta / 2.0f);
    e[a] = mx[a] + (double)(delta / 2.0f);
  }
  V3 eps;
  for (int a = 0; a < 3; ++a) eps[a] = (e[a] - o[a]) / 11;
  o = o - eps;
  e = e + eps;
  for (int a = 0; a < 3; ++a) {
    origin[a] = o[a];
    end[a] = e[a];
    width[a] = e[a] - o[a];
  }
}

// modelTriAttributeKernel (CUDACompute.cu:79-96).
void triAttributes(const double* V, const int32_t* F, int64_t nf, double* normal, double* area,
                   double* dir) {
  for (int64_t t = 0; t < nf; ++t) {
    V3 p1{V[3 * F[3 * t]], V[3 * F[3 * t] + 1], V[3 * F[3 * t] + 2]};
    V3 p2{V[3 * F[3 * t + 1]], V[3 * F[3 * t + 1] + 1], V[3 * F[3 * t + 1] + 2]};
    V3 p3{V[3 * F[3 * t + 2]], V[3 * F[3 * t + 2] + 1], V[3 * F[3 * t + 2] + 2]};
    V3 n = cross3(p2 - p1, p3 - p1);
    if (normal) { normal[3 * t] = n.x; normal[3 * t + 1] = n.y; normal[3 * t + 2] = n.z; }
    if (area) area[t] = 0.5 * std::sqrt(dot3(n, n));
    if (dir) dir[t] = dot3(-n, p1);
  }
}

// surfaceVoxelize (SVO.cu:366-493): Schwarz-Seidel conservative triangle/box test.
// Writes morton|flag into the dense Morton-indexed array, as the reference does.
static void voxelizeTriangle(const V3& p0, const V3& p1, const V3& p2, const int gs[3],
                             const V3& origin, const V3& unit, std::vector<uint32_t>& dense) {
  V3 v0 = p0 - origin, v1 = p1 - origin, v2 = p2 - origin;
  V3 e0 = v1 - v0, e1 = v2 - v1, e2 = v0 - v2;
  V3 n = cross3(e0, e1);
  {
    double z = dot3(n, n);
    if (z > 0.0) {
      double s = std::sqrt(z);
      n = {n.x / s, n.y / s, n.z / s};
    }
  }
  V3 bmin = vmin(v0, vmin(v1, v2)), bmax = vmax(v0, vmax(v1, v2));
  int gmin[3], gmax[3];
  for (int a = 0; a < 3; ++a) {
    gmin[a] = clampi((int)(bmin[a] / unit[a]), 0, gs[a] - 1);
    gmax[a] = clampi((int)(bmax[a] / unit[a]), 0, gs[a] - 1);
  }
  V3 c{0.0, 0.0, 0.0};
  if (n.x > 0.0) c.x = unit.x;
  if (n.y > 0.0) c.y = unit.y;
  if (n.z > 0.0) c.z = unit.z;
  const double d1 = dot3(n, c - v0);
  const double d2 = dot3(n, (unit - c) - v0);

  // 2-D edge normals and offsets for the three projections.
  struct E2 { double a, b, d; };
  auto mk = [](double a, double b, bool flip, double pa, double pb, double ua, double ub) {
    if (flip) { a = -a; b = -b; }
    double d = (-1.0 * (a * pa + b * pb)) + dmax(0.0, ua * a);
    d = d + dmax(0.0, ub * b);
    return E2{a, b, d};
  };
  const V3 ev[3] = {e0, e1, e2};
  const V3 vv[3] = {v0, v1, v2};
  E2 xy[3], yz[3], zx[3];
  for (int i = 0; i < 3; ++i) {
    xy[i] = mk(-1.0 * ev[i].y, ev[i].x, n.z < 0.0, vv[i].x, vv[i].y, unit.x, unit.y);
    yz[i] = mk(-1.0 * ev[i].z, ev[i].y, n.x < 0.0, vv[i].y, vv[i].z, unit.y, unit.z);
    zx[i] = mk(-1.0 * ev[i].x, ev[i].z, n.y < 0.0, vv[i].z, vv[i].x, unit.z, unit.x);
  }
  for (int z = gmin[2]; z <= gmax[2]; ++z)
    for (int y = gmin[1]; y <= gmax[1]; ++y)
      for (int x = gmin[0]; x <= gmax[0]; ++x) {
        V3 p{(double)x * unit.x, (double)y * unit.y, (double)z * unit.z};
        double nDOTp = dot3(n, p);
        if ((nDOTp + d1) * (nDOTp + d2) > 0.0) continue;
        bool out = false;
        for (int i = 0; i < 3 && !out; ++i) if ((xy[i].a * p.x + xy[i].b * p.y) + xy[i].d < 0.0) out = true;
        for (int i = 0; i < 3 && !out; ++i) if ((yz[i].a * p.y + yz[i].b * p.z) + yz[i].d < 0.0) out = true;
        for (int i = 0; i < 3 && !out; ++i) if ((zx[i].a * p.z + zx[i].b * p.x) + zx[i].d < 0.0) out = true;
        if (out) continue;
        uint32_t m = mortonEncode((uint32_t)x, (uint32_t)y, (uint32_t)z);
        dense[m] = m | kMortonFlag;
      }
}

static V3 nodeOrigin(const V3& g, double w, uint32_t morton) {
  uint32_t x, y, z;
  mortonDecode(morton, x, y, z);
  return {g.x + w * (double)x, g.y + w * (double)y, g.z + w * (double)z};
}

// SparseVoxelOctree::createOctree (SVO.cu:674-856) with constructNodeNeighbors
// (SVO.cu:861-911) and constructNodeVertexAndEdge (SVO.cu:913-1110).
Svo buildSvo(const double* V, int64_t nv, const int32_t* F, int64_t nf, int res,
             const double origin[3], const double width[3]) {
  (void)nv;
  Svo s;
  s.res = res;
  s.gridOrigin = {origin[0], origin[1], origin[2]};
  for (int a = 0; a < 3; ++a) s.unit[a] = width[a] / res;
  const int gs[3] = {res, res, res};
  size_t gridCNodeSize = (size_t)mortonEncode(res - 1, res - 1, res - 1) + 1;
  size_t gridTreeNodeSize = gridCNodeSize % 8 ? gridCNodeSize + 8 - (gridCNodeSize % 8) : gridCNodeSize;
  double unitNodeWidth = s.unit.x;

  std::vector<uint32_t> dense(gridCNodeSize, 0);
  for (int64_t t = 0; t < nf; ++t) {
    V3 p[3];
    for (int k = 0; k < 3; ++k) {
      int vi = F[3 * t + k];
      p[k] = {V[3 * vi], V[3 * vi + 1], V[3 * vi + 2]};
    }
    voxelizeTriangle(p[0], p[1], p[2], gs, s.gridOrigin, s.unit, dense);
  }

  std::vector<size_t> esum;  // d_esumTreeNodesArray
  int treeDepth = 0;
  while (true) {
    std::vector<uint32_t> pact;
    for (size_t i = 0; i < dense.size(); ++i)
      if (dense[i] >> 31) pact.push_back(dense[i]);
    const size_t numC = pact.size();
    if (!numC) break;
    ++treeDepth;
    if (treeDepth == 1) {
      s.numVoxels = numC;
      s.voxels.resize(numC);
      for (size_t i = 0; i < numC; ++i) s.voxels[i] = pact[i] & kMortonMask;
    }
    size_t numNodes = 1;
    std::vector<size_t> sumTree(1, 0);  // inclusive scan of cpNumNodes counts
    std::vector<uint32_t> parentDense;
    if (numC > 1) {
      parentDense.assign(gridTreeNodeSize, 0);
      const uint32_t first = (pact[0] >> 3) & 0xfffffff;
      parentDense[first] = first | kMortonFlag;
      sumTree.assign(numC, 0);
      for (size_t i = 1; i < numC; ++i) {
        size_t add = 0;
        if (((pact[i] >> 3) & 0xfffffff) != ((pact[i - 1] >> 3) & 0xfffffff)) {
          const uint32_t pm = (pact[i] >> 3) & 0xfffffff;
          parentDense[pm] = pm | kMortonFlag;
          add = 8;
        }
        sumTree[i] = sumTree[i - 1] + add;
      }
      numNodes = sumTree.back() + 8;
    }
    s.depthNumNodes.push_back(numNodes);

    std::vector<Node> level(numNodes);
    std::vector<uint32_t> beg(numC);
    const size_t levelStart = s.nodes.size();
    const size_t childStart = esum.size() >= 2 ? esum[esum.size() - 2] : 0;
    for (size_t i = 0; i < numC; ++i) {
      const uint32_t key = pact[i] & 7u;
      const uint32_t morton = pact[i] & kMortonMask;
      // A lone root at a non-zero key would land out of bounds in the reference;
      // it is placed at slot 0 here (documented deviation for that degenerate case).
      const size_t address = (numC == 1) ? 0 : sumTree[i] + key;
      Node& nd = level[address];
      nd.morton = morton;
      nd.origin = nodeOrigin(s.gridOrigin, unitNodeWidth, morton);
      nd.width = unitNodeWidth;
      beg[i] = (morton / 8) * 8;
      if (treeDepth > 1) {  // createNode_2 (SVO.cu:596-638)
        nd.isLeaf = false;
        for (int k = 0; k < 8; ++k) {
          nd.childs[k] = (uint32_t)(childStart + i * 8 + k);
          s.nodes[childStart + i * 8 + k].parent = (uint32_t)(levelStart + address);
        }
      }
    }
    beg.erase(std::unique(beg.begin(), beg.end()), beg.end());
    for (size_t t = 0; t < numNodes; ++t) {  // createRemainNode (SVO.cu:640-672)
      if (level[t].morton == 0) {
        const uint32_t morton = beg[t / 8] + (uint32_t)(t & 7);
        level[t].morton = morton;
        level[t].origin = nodeOrigin(s.gridOrigin, unitNodeWidth, morton);
        level[t].width = unitNodeWidth;
      }
    }
    if (treeDepth == 1) {
      esum.push_back(0);
      s.numFineNodes = numNodes;
    }
    s.nodes.insert(s.nodes.end(), level.begin(), level.end());
    esum.push_back(numNodes + esum.back());

    if (numC <= 1) break;  // the single-root level (numNodes/8 == 0)
    uint32_t mx = 0;
    for (uint32_t v : parentDense) mx = std::max(mx, v);
    const uint32_t numParent = (mx & kMortonMask) + ((mx >> 31) & 1);
    if (numParent == 0) break;
    parentDense.resize(numParent);
    dense.swap(parentDense);
    unitNodeWidth *= 2.0;
    gridCNodeSize = numParent;
    gridTreeNodeSize = gridCNodeSize % 8 ? gridCNodeSize + 8 - (gridCNodeSize % 8) : gridCNodeSize;
    if (numNodes / 8 == 0) break;
  }
  s.treeDepth = treeDepth;
  s.numTreeNodes = s.nodes.size();
  s.esumNodes = esum;

  // ---- neighbours (SVO.cu:861-911): top-down through the parent/child LUTs.
  short pLUT[8][27], cLUT[8][27];
  neighborLUTs(pLUT, cLUT);
  if (treeDepth >= 1) {
    const size_t root = s.nodes.size() - 1;
    s.nodes[root].nb[13] = (uint32_t)root;
    for (int d = treeDepth - 2; d >= 0; --d) {
      for (size_t t = esum[d]; t < esum[d] + s.depthNumNodes[d]; ++t) {
        Node& nd = s.nodes[t];
        const Node& p = s.nodes[nd.parent];
        const int key = nd.morton & 7;
        for (int k = 0; k < 27; ++k) {
          const uint32_t pn = p.nb[pLUT[key][k]];
          nd.nb[k] = (pn != kNone) ? s.nodes[pn].childs[cLUT[key][k]] : kNone;
        }
      }
    }
  }

  // ---- per-depth unique corner vertices (SVO.cu:913-963, 1064-1096).
  short vLUT[64];
  vertSharedLUT(vLUT);
  s.depthVerts.resize(treeDepth);
  s.esumVerts.assign(treeDepth + 1, 0);
  for (int d = 0; d < treeDepth; ++d) {
    std::vector<VertexRec> vs;
    vs.reserve(s.depthNumNodes[d] * 8);
    for (size_t t = esum[d]; t < esum[d] + s.depthNumNodes[d]; ++t) {
      const Node& nd = s.nodes[t];
      for (int k = 0; k < 8; ++k) {
        const double ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
        V3 corner{nd.origin.x + nd.width * ox, nd.origin.y + nd.width * oy, nd.origin.z + nd.width * oz};
        size_t idx = t;
        for (int j = 0; j < 8; ++j) {
          const uint32_t nb = nd.nb[vLUT[k * 8 + j]];
          if (nb < idx) idx = nb;
        }
        vs.push_back({corner, (uint32_t)idx});
      }
    }
    std::stable_sort(vs.begin(), vs.end(), [](const VertexRec& a, const VertexRec& b) {
      int t = lessPoint(a.pos, b.pos);
      if (t == 0) return a.owner < b.owner;
      return t == 1;
    });
    auto end = std::unique(vs.begin(), vs.end(), [](const VertexRec& a, const VertexRec& b) {
      return isApprox(a.pos, b.pos, 1e-9);
    });
    vs.erase(end, vs.end());
    s.esumVerts[d + 1] = s.esumVerts[d] + vs.size();
    s.depthVerts[d] = std::move(vs);
  }
  s.numVerts = s.esumVerts[treeDepth];

  // ---- unique fine-node edges (SVO.cu:965-1008, 1098-1110).
  short eLUT[48];
  edgeSharedLUT(eLUT);
  std::vector<EdgeRec> es;
  es.reserve(s.numFineNodes * 12);
  for (size_t t = 0; t < s.numFineNodes; ++t) {
    const Node& nd = s.nodes[t];
    for (int e = 0; e < 12; ++e) {
      const int a = kEdgeCorners[e][0], b = kEdgeCorners[e][1];
      V3 pa{nd.origin.x + ((a & 1) ? nd.width : 0.0), nd.origin.y + (((a >> 1) & 1) ? nd.width : 0.0),
            nd.origin.z + (((a >> 2) & 1) ? nd.width : 0.0)};
      V3 pb{nd.origin.x + ((b & 1) ? nd.width : 0.0), nd.origin.y + (((b >> 1) & 1) ? nd.width : 0.0),
            nd.origin.z + (((b >> 2) & 1) ? nd.width : 0.0)};
      size_t idx = t;
      for (int j = 0; j < 4; ++j) {
        const uint32_t nb = nd.nb[eLUT[e * 4 + j]];
        if (nb < idx) idx = nb;
      }
      es.push_back({pa, pb, (uint32_t)idx});
    }
  }
  std::stable_sort(es.begin(), es.end(), [](const EdgeRec& a, const EdgeRec& b) {
    int t0 = lessPoint(a.p0, b.p0);
    if (t0 == 0) {
      int t1 = lessPoint(a.p1, b.p1);
      if (t1 == 0) return a.owner < b.owner;
      return t1 == 1;
    }
    return t0 == 1;
  });
  auto eend = std::unique(es.begin(), es.end(), [](const EdgeRec& a, const EdgeRec& b) {
    return (isApprox(a.p0, b.p0, 1e-12) && isApprox(a.p1, b.p1, 1e-12)) ||
           (isApprox(a.p0, b.p1, 1e-12) && isApprox(a.p1, b.p0, 1e-12));
  });
  es.erase(eend, es.end());
  s.edges = std::move(es);
  return s;
}

}  // namespace orc
