/*
 * its.h -- C ABI of libits, a B200 (sm_100a) implementation of the ITS thin-shell path:
 * sparse voxel octree by triangle voxelisation, hierarchical hat-basis assembly over the
 * octree's corner vertices, LSCG fit of the coefficients, shell iso levels, dense field
 * evaluation and marching cubes.
 *
 * Conventions
 *  - Every call returns an its_status; the message of the last failure is its_last_error().
 *    Nothing in the library calls exit() or throws across this boundary.
 *  - Array arguments may be host or device pointers (CUDA unified addressing tells them
 *    apart); results are written to the memory the caller passes. Vectors of 3-D points
 *    are row-major (x,y,z) doubles; faces are int32 triples.
 *  - Objects (its_svo, its_op) live on the GPU of the context that made them and are used
 *    on the context's stream. A context must not be used by two host threads at once.
 *  - Integer outputs (Morton codes, topology, case indices) are bit-exact with the CPU
 *    restatement of the reference in oracle/; floating-point outputs carry tolerances
 *    stated in the tests.
 * Each declaration names the reference interface it replaces (file:line, paths inside
 * the Alan-Leo-Wong/ITS tree).
 */
#ifndef ITS_ITS_H_
#define ITS_ITS_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif
#ifdef __cplusplus
extern "C" {
#endif

typedef enum its_status {
  ITS_OK = 0,
  ITS_ERR_INVALID = 1,  /* bad argument, non-finite input, size out of range */
  ITS_ERR_CUDA = 2,     /* a CUDA runtime call failed */
  ITS_ERR_OOM = 3,      /* device allocation failed */
  ITS_ERR_TIMEOUT = 4,  /* a bounded device wait ran out */
  ITS_ERR_NOT_CONVERGED = 5,
  ITS_ERR_STATE = 6     /* object used in the wrong state */
} its_status;

typedef struct its_ctx its_ctx;
typedef struct its_svo its_svo;
typedef struct its_op its_op;

/* ---- context: owns the device, stream and allocator pool --------------------------- */
/* Replaces the per-call device selection of DeviceQuery.cuh:41 (getMaxComputeDevice). */
its_status its_create(its_ctx** ctx, int device);
its_status its_destroy(its_ctx* ctx);
const char* its_last_error(const its_ctx* ctx);
/* Work is issued on this stream (a cudaStream_t; NULL = the context's own stream). */
its_status its_set_stream(its_ctx* ctx, void* cuda_stream);
its_status its_synchronize(its_ctx* ctx);
const char* its_version(void);
/* Number of kernels this context has launched so far (a diagnostic counter). */
int64_t its_kernel_launches(const its_ctx* ctx);
/* Copies bytes of host memory (pageable or page-locked) to device memory of the context's GPU
   and waits for the copy. A pageable source of 32 MB or more goes through two page-locked
   chunks that several host threads fill while the previous chunk is in flight (the same path
   every entry point takes for large pageable inputs). No counterpart in the reference, which
   copies its arrays with cudaMemcpy. */
its_status its_copy_to_device(its_ctx* ctx, void* dst, const void* src, int64_t bytes);
/* The autotuner. With enable = 1 the first call of a tunable launch (the dense field's brick
   shape, the marching-cubes tile, the exact start's block size) for a given shape key times
   every candidate on the context's stream and keeps the fastest; later calls reuse the choice. Every candidate computes the
   same bits, so tuning changes speed only. cache_path (NULL: none) persists the choices as
   "key value" lines and is read here. No counterpart in the reference. */
its_status its_set_autotune(its_ctx* ctx, int enable, const char* cache_path);
/* The choices made so far as "key value" lines (length without the terminating zero). */
its_status its_autotune_choices(const its_ctx* ctx, char* buf, int64_t size, int64_t* length);
/* Self-check of the division the field kernels use (a multiply and two FMAs from the
   correctly rounded reciprocal, Markstein's theorem): counts the pairs whose quotient differs
   from the GPU's correctly rounded a[i] / b[i]. No counterpart in the reference. */
its_status its_check_division(its_ctx* ctx, const double* a, const double* b, int64_t n, int64_t* mismatches);

/* ---- a1-a2: model pre-processing (host) ----------------------------------------------- */
/* BaseModel::model2UnitCube / calcUnitCubeTransformMatrix (src/BaseModel.cpp:54-92). */
its_status its_model_to_unit_cube(double* verts, int64_t nverts, double scale_factor);
/* BaseModel::setUniformBoundingBox (src/BaseModel.cpp:24-51). */
its_status its_uniform_bbox(const double* verts, int64_t nverts, double origin[3], double end[3],
                            double width[3]);

/* ---- a3: triangle attributes ----------------------------------------------------------- */
/* cuAcc::launch_modelTriAttributeKernel (src/cuAcc/CUDACompute.h:14, .cu:79-109):
   normal = (p2-p1)x(p3-p1) (not normalised), area = |normal|/2, dir = -normal.p1.
   Any output may be NULL. */
its_status its_tri_attributes(its_ctx* ctx, const double* verts, int64_t nverts, const int32_t* faces,
                              int64_t nfaces, double* normal, double* area, double* dir);

/* ---- a4-a8: sparse voxel octree ----------------------------------------------------------- */
typedef struct its_svo_info {
  int res, depth;
  int64_t num_voxels, num_fine_nodes, num_nodes, num_vertices, num_edges;
  int64_t nodes_per_depth[16];
  int64_t vertices_per_depth[16];
  double origin[3], unit[3];
  double build_ms;           /* device time of its_svo_build (from the voxelisation on) */
  double learned_tables_ms;  /* of which the learned fit's octree-only tables: per-node face-sample
                                sums, coincident vertices and their geometric features */
} its_svo_info;
/* SparseVoxelOctree::createOctree (src/SVO.h:104, src/cuAcc/SVO.cu:674-856) together with
   constructNodeAtrributes (SVO.cu:1112-1118): voxelises the triangles at res^3 (res a power
   of two, 1..1024) inside the box (origin, width), builds every level, the 27-neighbour
   tables, the per-depth corner vertices and the fine-node edges. */
its_status its_svo_build(its_ctx* ctx, const double* verts, int64_t nverts, const int32_t* faces,
                         int64_t nfaces, int res, const double origin[3], const double width[3],
                         its_svo** out);
its_status its_svo_free(its_svo* svo);
its_status its_svo_get_info(const its_svo* svo, its_svo_info* info);
/* Surface voxels (the compacted level-0 occupancy, SVO.cu:722-749), ascending Morton. */
its_status its_svo_get_voxels(its_svo* svo, uint32_t* morton);
/* svoNodeArray (SVO.h:50-51): finest depth first, root last. childs is 8 per node,
   neighbors 27 per node (slot (dx+1)+3(dy+1)+9(dz+1)); UINT32_MAX marks "none".
   origin is 3 per node. Any output may be NULL. */
its_status its_svo_get_nodes(its_svo* svo, uint32_t* morton, uint32_t* parent, uint32_t* childs,
                             uint8_t* is_leaf, double* origin, double* width, uint32_t* neighbors);
/* nodeVertexArray (SVO.h:55-62): unique corners per depth in (x,y,z) order, depths
   concatenated; owner = lowest index of a node having the corner. */
its_status its_svo_get_vertices(its_svo* svo, double* pos, uint32_t* owner);
/* fineNodeEdgeArray (SVO.h:57, SVO.cu:1098-1110). */
its_status its_svo_get_edges(its_svo* svo, double* p0, double* p1, uint32_t* owner);

/* ---- a9: shell samples --------------------------------------------------------------- */
/* ThinShells::cpIntersectionPoints (src/ThinShells.cpp:38-479): mesh-edge x fine-node-face
   points (sorted, unique) followed by fine-node-edge x triangle points. With out_points NULL
   only the counts are returned; otherwise the first min(capacity, *num_points) points are
   written (a caller can pass a generous buffer once and call again only when *num_points
   exceeds it). */
its_status its_shell_samples(its_svo* svo, const double* verts, int64_t nverts, const int32_t* faces,
                             int64_t nfaces, double* out_points, int64_t capacity, int64_t* num_points,
                             int64_t* num_edge_points);

/* ---- a10: right-hand side -------------------------------------------------------------- */
/* ThinShells::cpSDFOfTreeNodes (src/ThinShells.cpp:481-509; libigl signed_distance with the
   fast winding number): exact distance to the mesh, negative where the winding number
   exceeds 1/2. */
its_status its_signed_distance(its_ctx* ctx, const double* points, int64_t npoints, const double* verts,
                               int64_t nverts, const int32_t* faces, int64_t nfaces, double* out);

/* ---- a11: operator assembly --------------------------------------------------------------- */
typedef enum its_op_mode { ITS_OP_FP64 = 0, ITS_OP_FP32_VALUES = 1 } its_op_mode;
/* The sparse system of ThinShells::cpCoefficients (src/ThinShells.cpp:511-606): one row per
   corner vertex with the diagonal 1, coincident finer vertices (1) and the non-zero hat values
   of the corners of every ancestor of the vertex's owner node. Stored as CSR with ascending
   columns plus its transpose; ITS_OP_FP32_VALUES also keeps float copies of the values for
   the mixed-precision solver. */
its_status its_operator_build(its_svo* svo, int mode, its_op** out);
/* Basis options of its_operator_build_ex. No counterpart in the reference: its basis is the
   degree-1 hat (src/BSpline.hpp:4-22) and its fit samples are the corner vertices
   (src/ThinShells.cpp:481-606); extra sample rows follow the uncompiled
   src/ThinShellsOctree.deprecated.cpp:139-187, which appends one row per sample point. */
typedef struct its_basis_opts {
  int degree;              /* 1: the reference's hats (its_operator_build); 3: cubic B-splines */
  const double* samples;   /* extra fit points, 3 per point, rows after the corner vertices' */
  int64_t num_samples;     /* (cubic basis only; 0 for none) */
} its_basis_opts;
/* The fit system in the chosen basis. Cubic: vertex v at depth d, lattice point (X,Y,Z), carries
   the tensor product of uniform cubic B-splines of width w_d = unit * 2^d centred at
   origin + (X,Y,Z) w_d; row r < num_vertices is the basis at corner vertex r (its exact lattice
   point), row num_vertices + i at samples[i]. With extra samples the system is stored square
   (rows x rows, the columns past the vertices empty): its_lscg_solve then takes b and lambda
   with rows entries, lambda's entries past the vertices staying 0. */
its_status its_operator_build_ex(its_svo* svo, int mode, const its_basis_opts* opts, its_op** out);
its_status its_operator_free(its_op* op);
its_status its_operator_info(const its_op* op, int64_t* rows, int64_t* nnz);
its_status its_operator_get_csr(its_op* op, int64_t* rowptr, int32_t* col, double* val);
/* y = A x (transpose = 0) or y = A^T x (transpose = 1). With x and y in device memory the
   call returns without waiting for the GPU (work is ordered on the context's stream). */
its_status its_operator_apply(its_op* op, const double* x, double* y, int transpose);

/* ---- a12: least-squares conjugate gradient ----------------------------------------------- */
typedef enum its_stop_rule {
  ITS_STOP_NORMAL = 0,   /* Eigen LSCG: ||A^T r|| <= tol ||A^T b|| */
  ITS_STOP_RESIDUAL = 1  /* ||b - A x|| <= tol ||b|| */
} its_stop_rule;
typedef enum its_precision {
  ITS_PREC_FP64 = 0,     /* every operation in FP64 */
  ITS_PREC_MIXED = 1     /* FP32 SpMV, FP64 dots/residual, FP64 iterative refinement */
} its_precision;
typedef struct its_solve_opts {
  double tol;           /* default: DBL_EPSILON (Eigen's default) */
  int64_t max_iters;    /* default (<= 0): 2 * columns (Eigen's default) */
  int stop_rule;        /* its_stop_rule */
  int precision;        /* its_precision */
  int ir_steps;         /* mixed: outer refinement steps (default 3) */
  double inner_tol;     /* mixed: inner relative tolerance (default 1e-3) */
  const double* x0;     /* warm start (NULL: zero start, Eigen's solve()) */
  int check_every;      /* iterations per convergence check / graph launch (default 8) */
} its_solve_opts;
typedef struct its_solve_report {
  int64_t iterations;   /* Eigen's count: direction updates before the stop */
  int converged, breakdown;
  double rel_residual;         /* ||b - A x|| / ||b|| */
  double normal_rel_residual;  /* ||A^T(b - A x)|| / ||A^T b|| */
  double ms;                   /* device time of the solve */
  int64_t inner_iterations;    /* mixed: CGLS iterations summed over refinement steps */
} its_solve_report;
its_status its_solve_opts_default(its_solve_opts* opts);
/* Eigen::LeastSquaresConjugateGradient::compute + solve (src/ThinShells.cpp:615-617). */
its_status its_lscg_solve(its_op* op, const double* b, double* lambda, const its_solve_opts* opts,
                          its_solve_report* report);

/* Batched form of its_lscg_solve for many independent fits (one operator per mesh, all on one
   context): every mesh runs Eigen's CGLS with its own scalars, stopping test and iteration
   count, but each SpMV and reduction covers the whole batch in one launch and converged
   meshes drop out. b[i] and lambda[i] are mesh i's vectors (host or device); opts->x0, when
   set, points to an array of count warm-start vectors. FP64 only. reports has count entries
   (ms is the batch's device time). No single-call counterpart in the reference, which fits
   one mesh per ThinShells object (src/ThinShells.cpp:615-617). */
its_status its_lscg_solve_batch(its_op* const* ops, int64_t count, const double* const* b, double* const* lambda,
                                const its_solve_opts* opts, its_solve_report* reports);

/* Exact start (hierarchical surplus). Coincident corner vertices of different depths have
   identical rows, so A lambda = b is consistent and its exact solutions differ only in how
   each point's value is split among its coincident vertices. This pass fixes the split
   (vertices whose lattice coordinates are all even below the root depth take shares[v],
   or 0 when shares is NULL) and gives every other row its surplus in explicit form,
   lambda_v = G_v - sum_c A(v,c) G_c over the corners c of the owner's parent cell, with
   G = b less the shares of the finer coincident vertices at each point: one matrix-free
   pass over the rows (generated from the octree), one or two launches. The result is an exact solution;
   its_lscg_solve with it as x0 stops at its residual test. No counterpart in the reference
   (which starts Eigen's CGLS from zero, src/ThinShells.cpp:615-617). Vectors may be host or
   device memory. */
its_status its_exact_start(its_svo* svo, const double* b, const double* shares, double* lambda);
/* The same for count octrees of one context (one or two launches for all of them); shares
   may be NULL or hold NULL entries. */
its_status its_exact_start_batch(its_svo* const* svos, int64_t count, const double* const* b,
                                 const double* const* shares, double* const* lambda);
/* ||b - A lambda|| / ||b|| without an assembled operator: rows above the finest depth summed
   as A has them (generated from the octree), finest rows through their parent cell's
   trilinear interpolant of the coarser field -- the same A lambda, to rounding -- every sum in
   a fixed order. */
its_status its_fit_residual(its_svo* svo, const double* b, const double* lambda, double* rel_residual);
its_status its_fit_residual_batch(its_svo* const* svos, int64_t count, const double* const* b,
                                  const double* const* lambda, double* rel_residual);

/* ---- a13: field at points and the shell iso levels ------------------------------------- */
/* ThinShells::cpLatentBSplineValue (src/ThinShells.cpp:655-755): each point's fine node by
   Morton code, then lambda times the hats of the 8 corners of that node and of every
   ancestor. Points outside every fine node get 0 and missing[i] = 1 (missing may be NULL). */
its_status its_eval_points(its_svo* svo, const double* lambda, const double* points, int64_t npoints,
                           double* out, uint8_t* missing);
/* innerShellIsoVal / outerShellIsoVal (ThinShells.cpp:743-744): min and max of the field
   over the points, skipping points outside every fine node. */
its_status its_shell_iso_values(its_svo* svo, const double* lambda, const double* points, int64_t npoints,
                                double* inner, double* outer, int64_t* num_missing);

/* ThinShells::multiPointQuery (src/ThinShells.cpp:1183-1420; CUDA branch cuAcc::cpPointQuery,
   src/cuAcc/CUDACompute.cu:1070-1156): field at arbitrary points (the sum over all corner
   vertices, evaluated through the lattice), points outside the model box grown by one box
   width taking the outer iso value; label 1 (value >= outer), -1 (value <= inner) or 0
   (between: inside the thin shell). values or labels may be NULL. */
its_status its_point_query(its_svo* svo, const double* lambda, const double* points, int64_t npoints,
                           const double box_origin[3], const double box_end[3], double inner, double outer,
                           double* values, int8_t* labels);

/* ThinShells::getPointValGradient (src/ThinShells.cpp:1800-1866), the gradients behind the
   point normals of ThinShells.cpp:1658-1735: a point outside the box [box_origin, box_end]
   moves halfway towards its previous position (before, may be NULL) until inside, then the
   field and its gradient (de_BaseFunction, BSpline.hpp:30-57) over its fine node's chain.
   gradients: 3 per point; points in no fine node get 0 and missing[i] = 1 (may be NULL). */
its_status its_point_value_gradient(its_svo* svo, const double* lambda, const double* points, const double* before,
                                   int64_t npoints, const double box_origin[3], const double box_end[3], double* values,
                                   double* gradients, uint8_t* missing);

/* ---- cubic basis: field, and the offset shell samples ----------------------------------
   No counterpart in the reference (see its_basis_opts). Field of cubic coefficients (one per
   corner vertex) at points / on the (res+1)^3 lattice origin + i*width/res (x fastest): the sum
   over every depth and every vertex whose support holds the point, in the order the rows of
   its_operator_build_ex use, so A lambda equals the field at the rows' points bit for bit. */
its_status its_eval_points_cubic(its_svo* svo, const double* lambda, const double* points, int64_t npoints,
                                 double* out);
its_status its_eval_grid_cubic(its_svo* svo, const double* lambda, const double origin[3], const double width[3],
                               int res, double* field);
/* Offset shell samples: at every mesh vertex the unit area-weighted normal n (the sum of the
   unnormalised normals (p1-p0)x(p2-p0) of its faces, in face order, made unit) and the points
   v + eps n (target +eps) for all vertices, then v - eps n (target -eps): points 6*nverts
   doubles, targets 2*nverts (either may be NULL). A vertex with no face gets both points at v. */
its_status its_offset_samples(its_ctx* ctx, const double* verts, int64_t nverts, const int32_t* faces, int64_t nfaces,
                              double eps, double* points, double* targets);

/* ---- a14-a15: dense field and marching cubes -------------------------------------------- */
/* The field of MC::launch_computSDFKernel (src/cuAcc/MarchingCubes/MarchingCubes.cu:464-536,
   CUDACompute.cu:435-510) on the (res+1)^3 lattice origin + i*width/res, x fastest. */
its_status its_eval_grid(its_svo* svo, const double* lambda, const double origin[3], const double width[3],
                         int res, double* field);
/* MC::marching_cubes (src/cuAcc/MarchingCubes/MarchingCubes.h:136-139) on a lattice field:
   cube_index (res^3 bytes, NULL allowed) with bit i = field[corner i] < iso in the corner
   order of MarchingCubes.cu:233-241; triangle vertices (3 doubles each) in voxel order: the
   first min(capacity, num_verts) are written, the rest of tri_verts is left as it was.
   With tri_verts NULL only num_verts is returned. */
its_status its_marching_cubes(its_ctx* ctx, const double* field, int res, const double origin[3],
                              const double width[3], double iso, uint8_t* cube_index, double* tri_verts,
                              int64_t capacity, int64_t* num_verts);
/* The marching-cubes driver of ThinShells::mcVisualization (src/ThinShells.cpp:1086-1129 ->
   MC::marching_cubes, src/cuAcc/MarchingCubes/MarchingCubes.cu:672-714) in one call: the field
   of lambda on the (res+1)^3 lattice is evaluated once into device scratch (field_mode 0:
   its_eval_grid, bit-exact; 1: its_eval_grid_fast) and stays on the device while marching
   cubes runs at each of the n_iso levels. Level k writes up to capacity[k] vertices to
   tri_verts[k] (host or device; tri_verts NULL or a NULL entry: count only) and its total
   vertex count to num_verts[k]. */
its_status its_eval_grid_mc(its_svo* svo, const double* lambda, const double origin[3], const double width[3], int res,
                            int field_mode, const double* iso, int n_iso, double* const* tri_verts,
                            const int64_t* capacity, int64_t* num_verts);
/* Welded, indexed form of MC::marching_cubes' triangle soup (writeToOBJFile,
   src/cuAcc/MarchingCubes/MarchingCubes.cu:635-661, emits 3 fresh vertices per triangle): one
   vertex per active lattice edge (numbered in edge-id order, id = 3*((z*(res+1)+y)*(res+1)+x)+axis)
   placed by the reference's lerp from the lower to the upper lattice point, and triangles as
   int32 index triples in voxel order with the soup's winding. NULL outputs: counts only. */
its_status its_marching_cubes_mesh(its_ctx* ctx, const double* field, int res, const double origin[3],
                                   const double width[3], double iso, double* verts, int64_t vert_capacity,
                                   int64_t* num_verts, int32_t* tris, int64_t tri_capacity, int64_t* num_tris);
/* FP32 forms of the dense field and marching cubes (the precision mode): the field is summed in
   FP32 from FP32 copies of the coefficients and corner positions (quotients by one reciprocal
   multiply), 4 bytes per lattice point; marching cubes classifies and interpolates the FP32
   values (vertex positions in FP64). No counterpart in the reference (FP64 only). */
its_status its_eval_grid_f32(its_svo* svo, const double* lambda, const double origin[3], const double width[3],
                             int res, float* field);
/* The dense field of its_eval_grid (FP64) / its_eval_grid_f32 (FP32) on a lattice aligned with
   the octree -- origin and width the octree's box (to 1e-6 of a cell), res = the octree's res
   * 1, 2, 4 or 8 (the marching-cubes grids of ThinShells::mcVisualization,
   src/ThinShells.cpp:1086-1129) -- built coarse to fine by trilinear prolongation over dense
   per-depth lattices: the cost of writing the field once instead of evaluating every point at
   every depth. Not bit for bit its_eval_grid: the hats sit on the octree's exact lattice
   points, where the reference's corner positions and a single-precision-padded box differ by
   ~1e-9 (field within ~1e-7 of max |field|, tested); any other lattice falls back to
   its_eval_grid / its_eval_grid_f32. Scratch: 8 (FP32: 4) bytes per point of every depth's
   lattice, ((res_octree + 1)^3 * 8 / 7 points). */
its_status its_eval_grid_fast(its_svo* svo, const double* lambda, const double origin[3], const double width[3],
                              int res, double* field);
its_status its_eval_grid_fast_f32(its_svo* svo, const double* lambda, const double origin[3], const double width[3],
                                  int res, float* field);
its_status its_marching_cubes_f32(its_ctx* ctx, const float* field, int res, const double origin[3],
                                  const double width[3], double iso, uint8_t* cube_index, double* tri_verts,
                                  int64_t capacity, int64_t* num_verts);
/* No counterpart in the reference. The same results as its_marching_cubes for callers that
   cannot let the library allocate device memory (an application that holds the GPU's memory in
   its own fixed budget, a frame loop that cudaMalloc's implicit synchronisation would stall):
   no cudaMalloc/cudaFree, the scan scratch is a fixed 64 KiB file-scope device array.
   field, cube_index and tri_verts must be device memory of the context's GPU; res <= 256
   (ITS_ERR_INVALID beyond). Calls on one device share the array (overlapping calls race); the
   call waits on its stream for num_verts. The first call on a device looks up the array's
   address and keeps it: make that first call before any stream capture, and do not reset the
   device (cudaDeviceReset) afterwards. */
its_status its_marching_cubes_noalloc(its_ctx* ctx, const double* field, int res, const double origin[3],
                                      const double width[3], double iso, uint8_t* cube_index, double* tri_verts,
                                      int64_t capacity, int64_t* num_verts);

/* ---- learned shares: the share network --------------------------------------------------
   No counterpart in the reference. A 64 -> 128 -> 128 -> 128 -> 1 GELU network (BF16
   weights and activations, FP32 accumulation, tcgen05 tensor-core GEMMs) that predicts the
   coefficient of each corner vertex coincident with a coarser corner in the minimum-norm
   solution, i.e. the shares of its_exact_start. Parameters: its_mlp_num_params() FP32
   values, W1[128x64] b1 W2[128x128] b2 W3[128x128] b3 w4[128] b4 (W[out][in]). Feature rows
   are 64 FP32 values, already normalised. Pointers may be host or device memory. */
typedef struct its_mlp its_mlp;
/* batch: rows per training step and per inference chunk, a multiple of 128. */
its_status its_mlp_create(its_ctx* ctx, int64_t batch, its_mlp** out);
its_status its_mlp_free(its_mlp* mlp);
int64_t its_mlp_num_params(void);
/* Loads parameters and resets the Adam state. */
its_status its_mlp_set_params(its_mlp* mlp, const float* params);
its_status its_mlp_get_params(its_mlp* mlp, float* params);
/* Predictions: one persistent kernel for all layers (weights and activations in shared memory). */
its_status its_mlp_forward(its_mlp* mlp, const float* features, int64_t n, float* out);
/* The same predictions for device features and output, queued on the context's stream
   without waiting (for callers that pipeline inference with their own work); a tensor-core
   wait that ran out sets a sticky flag that its_mlp_check reports. */
its_status its_mlp_forward_async(its_mlp* mlp, const float* features, int64_t n, float* out);
/* The same from features already in the kernel's input form, as the learned fit's features
   kernel writes them: ceil(n / 128) tiles of 128 rows x 64 BF16 features (16 KB each, device
   memory, 16-byte aligned), rows of 128 bytes, the 16-byte chunk c of row r stored at chunk
   position c ^ (r % 8) of its row (128-byte swizzle, 8-row atoms of 1 KB). after_kernel != 0
   declares that the previous operation on the context's stream is a kernel launch: the
   network's blocks may then be scheduled while that kernel drains (programmatic dependent
   launch; the network reads its input only after that kernel has completed). */
its_status its_mlp_forward_tiles_async(its_mlp* mlp, const void* tiles, int64_t n, float* out, int after_kernel);
/* Waits for the context's stream; ITS_ERR_TIMEOUT if a network kernel's bounded wait ran out. */
its_status its_mlp_check(its_mlp* mlp);
/* The same predictions layer by layer through the training kernels (bit-identical). */
its_status its_mlp_forward_layers(its_mlp* mlp, const float* features, int64_t n, float* out);
/* Gradient of mean((out - y)^2) over n rows (n <= batch, a multiple of 64), no update. */
its_status its_mlp_gradient(its_mlp* mlp, const float* features, const float* y, int64_t n, float* grad,
                            float* loss);
/* steps Adam steps (lr, beta 0.9 / 0.999, eps 1e-8) on random batches of n resident rows;
   loss_curve (NULL or steps entries) receives each step's mean squared error. */
its_status its_mlp_train(its_mlp* mlp, const float* features, const float* y, int64_t n, int64_t steps, float lr,
                         uint64_t seed, float* loss_curve);
/* Features of the vertices coincident with a coarser corner (the shares of the exact start),
   64 per vertex: the signed distance, zero-share surplus values of the vertex's copies and
   lattice neighbours, neighbour presence, depth, cell width, and the face samples of the
   octree's mesh (summed per node at its_svo_build) in the owner node's 27-neighbourhood:
   count, mean offset, mean normal, 1 - |mean normal|. norm (NULL or 128 values: mean[64],
   scale[64]) normalises (f - mean) * scale. features == NULL: *count only; else capacity >=
   *count rows, and ids (NULL or capacity entries) receives the vertex of each row
   (ascending). */
its_status its_share_features(its_svo* svo, const double* b, const float* norm, float* features, int64_t capacity,
                              int64_t* ids, int64_t* count);
/* Learned start: features, the share network, then its_exact_start with the predicted
   shares (prediction * norm[129] + norm[128]). norm: 130 values (input mean[64], input
   scale[64], output mean, output scale). lambda: an exact solution whose null-space part is
   the network's. */
its_status its_learned_start(its_svo* svo, its_mlp* mlp, const double* b, const float* norm, double* lambda);
/* The same for count octrees of one context (one network pass over all of them). */
its_status its_learned_start_batch(its_svo* const* svos, int64_t count, its_mlp* mlp, const double* const* b,
                                   const float* norm, double* const* lambda);
/* The learned fit of one octree, in place of ThinShells::creatShell's LSCG from zero
   (src/ThinShells.cpp:608-653): its_learned_start, then ||b - A lambda|| / ||b|| (as
   its_fit_residual), then, when that exceeds tol, its_lscg_solve (FP64, ITS_STOP_RESIDUAL)
   from the learned start. The start and the check run as a CUDA graph captured on the first
   call and replayed while the network (the same its_mlp, not another made since), norm, the
   context's stream and the device addresses of b and lambda stay the same (host vectors go
   through buffers of the octree's own; page-locked ones are copied by the graph itself, lambda
   while the residual runs, so their addresses are part of what must stay the same); the graph
   reads b and the network's parameters afresh every time.
   Complete on return. report (may be NULL): iterations = LSCG iterations after the start (0
   when the start passed), converged, rel_residual, ms = device time from the start's first
   kernel to the end of the residual check (the device clock, read by those kernels), plus the
   fallback LSCG's when it runs; copies of host vectors are not included. */
its_status its_learned_fit(its_svo* svo, its_mlp* mlp, const double* b, const float* norm, double tol,
                           double* lambda, its_solve_report* report);

#ifdef __cplusplus
}
#endif
#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* ITS_ITS_H_ */
