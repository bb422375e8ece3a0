// CPU oracle (test infrastructure): octree data structures. See orc_common.hpp.
#pragma once
#include <cstddef>
#include <vector>

#include "orc_common.hpp"

namespace orc {

struct Node {  // SVONode (SVO.h:15-32)
  uint32_t morton = 0;
  bool isLeaf = true;
  V3 origin{0, 0, 0};
  double width = 0;
  uint32_t parent = kNone;
  uint32_t childs[8] = {kNone, kNone, kNone, kNone, kNone, kNone, kNone, kNone};
  uint32_t nb[27];
  Node() { for (auto& v : nb) v = kNone; }
};
struct VertexRec { V3 pos; uint32_t owner; };        // node_vertex_type (SVO.h:36)
struct EdgeRec { V3 p0, p1; uint32_t owner; };       // node_edge_type (SVO.h:35)

struct Svo {
  int res = 0;
  V3 gridOrigin{0, 0, 0};
  V3 unit{0, 0, 0};  // unitVoxelSize per axis (SVO.cu:683-686)
  int treeDepth = 0;
  size_t numVoxels = 0, numFineNodes = 0, numTreeNodes = 0, numVerts = 0;
  std::vector<uint32_t> voxels;           // surface voxels, ascending Morton
  std::vector<size_t> depthNumNodes, esumNodes;
  std::vector<Node> nodes;                // finest depth first, root last
  std::vector<std::vector<VertexRec>> depthVerts;
  std::vector<size_t> esumVerts;
  std::vector<EdgeRec> edges;             // fine-node edges, sorted
};

void modelToUnitCube(double* V, int64_t nv, double scaleFactor);
void uniformBBox(const double* V, int64_t nv, double origin[3], double end[3], double width[3]);
void triAttributes(const double* V, const int32_t* F, int64_t nf, double* normal, double* area, double* dir);
Svo buildSvo(const double* V, int64_t nv, const int32_t* F, int64_t nf, int res,
             const double origin[3], const double width[3]);

}  // namespace orc
