// Octree object shared by the translation units of libits.
#pragma once
#include "its_ctx.cuh"

namespace its {
struct LearnedPlan;  // the captured learned fit of an octree (its_learned.cu)
void destroyPlan(LearnedPlan* p);
}  // namespace its

struct its_svo {
  its_ctx* ctx = nullptr;
  its::SvoDevice d;
  its::LearnedPlan* plan = nullptr;
};

namespace its {
// Checks face indices and vertex finiteness on the device.
its_status validateMesh(its_ctx* ctx, const double* dV, int64_t nv, const int32_t* dF, int64_t nf);
its_status svoBuild(its_ctx* ctx, const double* dV, int64_t nv, const int32_t* dF, int64_t nf, int res,
                    const double origin[3], const double width[3], its_svo* s);
// Face samples (centroid, unit normal) summed per fine node in face order, then per coarser
// node over its 8 children in order, into d.nodeSample* (its_features.cu).
its_status nodeSampleStats(its_ctx* ctx, SvoDevice& d, const double* dV, const int32_t* dF, int64_t nf);
// The vertices coincident with a coarser corner (lattice coordinates all even below the
// root depth), ascending, into ids (capacity numVerts); *count their number.
its_status coincidentIds(its_ctx* ctx, const SvoDevice& d, int64_t* ids, int64_t* count);
// Features 38-45 of the share network for every coincident vertex into d.coincGeom: they
// depend on the octree and the mesh's face samples only (its_features.cu).
its_status coincidentGeometry(its_ctx* ctx, SvoDevice& d);
}  // namespace its
