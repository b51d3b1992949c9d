/*
 * uaamg.h -- C ABI of the B200 UAAMG-PCG library (libuaamg_b200.so).
 *
 * Drop-in boundary for the reference's SIMD_UAAMG pressure solver.  Every
 * entry point names the reference interface it replaces (paths inside the
 * reference project).  The reference passes OpenVDB grids by shared_ptr; this
 * ABI passes the same content as a flattened leaf list (uaamg_leaf_grid,
 * identical to an OpenVDB LeafNode<T,3> payload: origin, 512-bit value mask,
 * 512 values with offset 64x+8y+z).
 *
 * Conventions
 *  - Status codes, never exceptions: UAAMG_SUCCESS (0) and UAAMG_FAILED (1)
 *    are the reference's PoissonSolver::SUCCESS / FAILED
 *    (SIMD_UAAMG/simd_vdb_poisson.h:149-152); negative values are errors,
 *    described by uaamg_last_error() (thread-local).
 *  - Vectors (pressure, right-hand side) are "leaf-dense": float[leaf][512]
 *    over the handle's DOF leaves (uaamg_poisson_dof_topology), zero at
 *    voxels that are not degrees of freedom.  This is the buffer layout of
 *    the grid LaplacianWithLevel::getZeroVectorGrid() returns.
 *  - Functions without a suffix take HOST pointers and copy to and from the
 *    device inside the call.  *_device functions take device pointers and
 *    return after enqueueing on the handle's stream.
 *  - One handle per host thread (the reference object is not re-entrant either).
 */
#ifndef UAAMG_H
#define UAAMG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UAAMG_SUCCESS 0
#define UAAMG_FAILED 1
#define UAAMG_ERR_INVALID_ARGUMENT (-1)
#define UAAMG_ERR_CUDA (-2)
#define UAAMG_ERR_OUT_OF_MEMORY (-3)
#define UAAMG_ERR_DOMAIN_TOO_LARGE (-4)
#define UAAMG_ERR_NO_DEVICE (-5)
#define UAAMG_ERR_TIMEOUT (-6)

/* PoissonSolver::SmootherOption (SIMD_UAAMG/simd_vdb_poisson.h:143-148) */
#define UAAMG_SMOOTHER_SCHEDULED_RELAXED_JACOBI 0
#define UAAMG_SMOOTHER_WEIGHTED_JACOBI 1
#define UAAMG_SMOOTHER_RED_BLACK_GAUSS_SEIDEL 2
#define UAAMG_SMOOTHER_SPAI0 3

/* LaplacianApplySIMD::WorkingMode (SIMD_UAAMG/simd_vdb_poisson.cpp:685-692) */
#define UAAMG_MODE_WEIGHTED_JACOBI 0
#define UAAMG_MODE_RESIDUAL 1
#define UAAMG_MODE_LAPLACIAN 2
#define UAAMG_MODE_RED_GS 3
#define UAAMG_MODE_BLACK_GS 4
#define UAAMG_MODE_SPAI0 5

/* A flattened openvdb::FloatGrid (components = 1) or Vec3fGrid (components = 3).
 * origins and masks are host memory; values are host memory unless
 * values_on_device != 0.  masks may be NULL (all voxels active). */
typedef struct uaamg_leaf_grid {
    int64_t leaf_count;
    const int32_t* origins;   /* [leaf_count][3], multiples of 8 */
    const uint64_t* masks;    /* [leaf_count][8] or NULL */
    const float* values;      /* [leaf_count][512][components] */
    int32_t components;       /* 1 or 3 */
    int32_t values_on_device; /* 0: host pointer, 1: device pointer */
    float background[3];      /* tree background per component */
} uaamg_leaf_grid;

typedef struct uaamg_poisson uaamg_poisson;

/* Build the level-0 matrix and the multigrid hierarchy.
 * Replaces LaplacianWithLevel::createPressurePoissonLaplacian(liquid_phi,
 * face_weights, dt) (SIMD_UAAMG/simd_vdb_poisson.h:54-57, .cpp:95-99) followed
 * by PoissonSolver::PoissonSolver(level0) (simd_vdb_poisson.h:153-160, which
 * runs constructMultigridHierarchy, .cpp:1813-1842).  dx is the voxel size of
 * liquid_phi (the reference reads liquid_phi->voxelSize()[0]). */
int uaamg_poisson_create(const uaamg_leaf_grid* liquid_phi, const uaamg_leaf_grid* face_weights,
                         float dt, float dx, uaamg_poisson** out);
/* uaamg_poisson_create with the construction enqueued on `stream` (a
 * cudaStream_t; NULL = the handle's own stream): it is ordered after the
 * caller's work on that stream (inputs that stream produced need no host
 * synchronisation), and the stream stays the handle's (uaamg_poisson_set_stream). */
int uaamg_poisson_create_on_stream(const uaamg_leaf_grid* liquid_phi, const uaamg_leaf_grid* face_weights, float dt,
                                   float dx, void* stream, uaamg_poisson** out);
/* The pressure step of FLIP_vdb's solve_pressure_simd (FLIP_vdb.cpp:3132-3148)
 * up to the solve, in one call: createPressurePoissonLaplacian(liquid_phi,
 * face_weights, dt) + PoissonSolver(level0) (as uaamg_poisson_create) and
 * createPressurePoissonRightHandSide(face_weights, vx, vy, vz, solid_velocity,
 * dt) (simd_vdb_poisson.cpp:101-127), with the rhs kept on the device for
 * uaamg_poisson_solve_*_resident.  Each host input crosses the bus once (the
 * face weights feed both the matrix and the rhs), and the velocity uploads run
 * on a second stream while the hierarchy is built.  Pinned host inputs make
 * the uploads asynchronous, and a face grid (face weights, velocities, solid
 * velocity) in pinned memory is read by a kernel through its device mapping,
 * only at the leaves the construction reads (those holding liquid and the
 * next leaf above them along x, y or z); pinned inputs stay unchanged until
 * the handle's stream has passed the construction (a solve has returned).
 * Device inputs (values_on_device) are read in place.  uaamg_poisson_create
 * reads its face weights the same way. */
int uaamg_poisson_create_with_rhs(const uaamg_leaf_grid* liquid_phi, const uaamg_leaf_grid* face_weights,
                                  const uaamg_leaf_grid* vx, const uaamg_leaf_grid* vy, const uaamg_leaf_grid* vz,
                                  const uaamg_leaf_grid* solid_velocity, float dt, float dx, void* stream,
                                  uaamg_poisson** out);
/* Kernel shapes of the solves by level size (process-wide).  Every setting
 * gives the same results (a pass that carries a level-0 dot product switches
 * kernels at a fixed size, whatever pipe_min_leaves is).  The defaults are the
 * measured ones; uaamg_b200/tuning holds tables an autotuner wrote.  A change
 * applies to the next solve of every handle (cached graphs are rebuilt).  No
 * counterpart in the reference (its kernels have one shape). */
typedef struct {
    int32_t staged_min_leaves;  /* levels of at least this many leaves sweep with the bulk-copy staged kernels (64) */
    int32_t split_min_leaves;   /* ... store a computed source (first sweep, prolongation) before sweeping (1024) */
    int32_t pipe_min_leaves;    /* ... sweep and restrict with the persistent pipelined kernels (8192) */
    int32_t elem_ctas_per_sm;   /* CTAs per SM of the grid-stride passes, 1..32 (16) */
    int32_t bottom_cycle;       /* 1: both visits of the level above the coarsest, with the coarsest solves, as one
                                 * thread-block-cluster launch where the level fits (1) */
} uaamg_tuning;
int uaamg_get_tuning(uaamg_tuning* out);
int uaamg_set_tuning(const uaamg_tuning* tuning);

/* ~PoissonSolver / ~LaplacianWithLevel */
int uaamg_poisson_destroy(uaamg_poisson* h);

/* Public fields of PoissonSolver (simd_vdb_poisson.h:165-169):
 * mSmoother, mMaxIteration (100), mRelativeTolerance (1e-7). */
int uaamg_poisson_set_smoother(uaamg_poisson* h, int smoother);
int uaamg_poisson_set_max_iterations(uaamg_poisson* h, int max_iterations);
int uaamg_poisson_set_relative_tolerance(uaamg_poisson* h, float relative_tolerance);
/* mIterationTaken (simd_vdb_poisson.h:165) of the last solve */
int uaamg_poisson_iterations(const uaamg_poisson* h);
/* |r|_inf at the end of the last solve (the reference prints it per iteration,
 * simd_vdb_poisson.cpp:2194) */
float uaamg_poisson_final_residual(const uaamg_poisson* h);

/* mMultigridHierarchy.size() and per level mNumDof / leaf count */
int uaamg_poisson_num_levels(const uaamg_poisson* h);
int64_t uaamg_poisson_num_dof(const uaamg_poisson* h, int level);
int64_t uaamg_poisson_leaf_count(const uaamg_poisson* h, int level);
/* Topology of a level's DOF grid (mDofIndex tree without empty leaves, in
 * OpenVDB tree order): origins [n][3], masks [n][8] (host memory). */
int uaamg_poisson_dof_topology(const uaamg_poisson* h, int level, int32_t* origins, uint64_t* masks);
/* Every voxel's DOF index (mDofIndex values, setDofIndex .cpp:637-671), -1 off DOF. */
int uaamg_poisson_dof_index(const uaamg_poisson* h, int level, int32_t* out);

/* LaplacianWithLevel::createPressurePoissonRightHandSide(face_weights, vx, vy,
 * vz, solid_velocity, dt) (simd_vdb_poisson.h:59-65, .cpp:101-127).
 * rhs_out: host float[leaf][512] over the level-0 DOF leaves. */
int uaamg_poisson_build_rhs(uaamg_poisson* h, const uaamg_leaf_grid* face_weights,
                            const uaamg_leaf_grid* vx, const uaamg_leaf_grid* vy,
                            const uaamg_leaf_grid* vz, const uaamg_leaf_grid* solid_velocity,
                            float dt, float* rhs_out);
int uaamg_poisson_build_rhs_device(uaamg_poisson* h, const uaamg_leaf_grid* face_weights,
                                   const uaamg_leaf_grid* vx, const uaamg_leaf_grid* vy,
                                   const uaamg_leaf_grid* vz, const uaamg_leaf_grid* solid_velocity,
                                   float dt, float* d_rhs_out);

/* PoissonSolver::solveMultigridPCG(in_out_pressure, rhs) (simd_vdb_poisson.h:162,
 * .cpp:2155-2226).  pressure holds the initial guess on entry. Returns
 * UAAMG_SUCCESS / UAAMG_FAILED (or an error); *iterations = mIterationTaken. */
int uaamg_poisson_solve_pcg(uaamg_poisson* h, float* pressure, const float* rhs, int* iterations);
int uaamg_poisson_solve_pcg_device(uaamg_poisson* h, float* d_pressure, const float* d_rhs,
                                   int* iterations);
/* The rest of solve_pressure_simd (FLIP_vdb.cpp:3143-3157) on a handle made by
 * uaamg_poisson_create_with_rhs: the pressure set to zero, solveMultigridPCG
 * (or, after FAILED, solvePureMultigrid) with the rhs built at creation, the
 * pressure (float[leaf][512] over the level-0 DOF leaves) written to host or
 * device memory.  Returns as uaamg_poisson_solve_pcg / _solve_mg;
 * UAAMG_ERR_INVALID_ARGUMENT when the handle holds no rhs. */
int uaamg_poisson_solve_pcg_resident(uaamg_poisson* h, float* pressure, int* iterations);
int uaamg_poisson_solve_pcg_resident_device(uaamg_poisson* h, float* d_pressure, int* iterations);
int uaamg_poisson_solve_mg_resident(uaamg_poisson* h, float* pressure, int* iterations);
/* The rhs built at creation, into host or device memory (cudaMemcpyDefault). */
int uaamg_poisson_copy_rhs(uaamg_poisson* h, float* rhs_out);
/* PoissonSolver::solvePureMultigrid (simd_vdb_poisson.h:163, .cpp:2228-2267) */
int uaamg_poisson_solve_mg(uaamg_poisson* h, float* pressure, const float* rhs, int* iterations);
int uaamg_poisson_solve_mg_device(uaamg_poisson* h, float* d_pressure, const float* d_rhs,
                                  int* iterations);

/* r = b - A x over level 0 and |r|_inf: LaplacianWithLevel::residualApply
 * (simd_vdb_poisson.cpp:1347-1357) followed by PoissonSolver::levelAbsMax
 * (.cpp:2270-2276, grid_abs_max_op, openvdb_grid_math_op.h:4-43).  Device
 * pointers; d_r: float[leaf][512], d_norm: one float.  Uses the handle's
 * reduction scratch (one partial per leaf), so calls on one handle must not
 * overlap; returns after enqueueing on the handle's stream. */
int uaamg_poisson_residual_norm_device(uaamg_poisson* h, const float* d_x, const float* d_b, float* d_r,
                                       float* d_norm);

/* Allocation-free variant of uaamg_poisson_residual_norm_device, same inputs,
 * outputs and results.  No counterpart in the reference.  For callers that
 * must not allocate GPU memory while they run, e.g. a simulation loop that
 * reserves its whole device budget up front (an allocation can synchronise the
 * device, take milliseconds, or fail once the budget is spent) or a host
 * application that owns the device heap through its own allocator.  The
 * reduction scratch is a fixed array inside the library (2 MiB per device,
 * kept until the process exits) instead of memory allocated per handle;
 * nothing is allocated by the call.  Limit: level 0 may hold at most 262144
 * leaves (134 M voxels); larger levels are rejected with
 * UAAMG_ERR_INVALID_ARGUMENT.  The array's device address is looked up
 * (cudaGetSymbolAddress) when the handle is created, with the handle's device
 * current; the call must be made with that device current too, otherwise it is
 * rejected with UAAMG_ERR_INVALID_ARGUMENT and nothing is launched.  All calls
 * on a device share the one array, so calls whose kernels overlap on the GPU
 * (different streams or handles) race and must be serialised by the caller. */
int uaamg_poisson_residual_norm_noalloc(uaamg_poisson* h, const float* d_x, const float* d_b, float* d_r,
                                        float* d_norm);

/* Per-level operators, public methods of LaplacianWithLevel
 * (simd_vdb_poisson.h:90-115).  Host pointers, level-dense vectors.
 *   mode: UAAMG_MODE_*; weight: Jacobi weight; w_sor: SOR weight of GS modes.
 * residualApply / laplacianApply / weightedJacobiApply / spai0Apply and one
 * red or black Gauss-Seidel pass (.cpp:1347-1433). */
int uaamg_poisson_level_apply(uaamg_poisson* h, int level, int mode, float weight, float w_sor,
                              const float* lhs, const float* rhs, float* out);
/* setGridToResultAfterFirstJacobi / ...FirstSPAI0 / ...FirstRBGS<true> (.cpp:1435-1582).
 * kind: 0 Jacobi (uses weight), 1 SPAI0, 2 red-black Gauss-Seidel (uses w_sor). */
int uaamg_poisson_level_first_sweep(uaamg_poisson* h, int level, int kind, float weight,
                                    float w_sor, const float* rhs, float* out);
/* restriction (fine level -> level+1) and prolongation<true> (level+1 -> level),
 * .cpp:1624-1754. prolongation adds alpha*coarse into fine (in/out). */
int uaamg_poisson_level_restrict(uaamg_poisson* h, int fine_level, const float* fine, float* coarse);
int uaamg_poisson_level_prolongate(uaamg_poisson* h, int fine_level, const float* coarse,
                                   float* fine, float alpha);
/* Effective level coefficients after trimDefaultNodes (.cpp:1756-1811): diag,
 * minus-x/y/z face entries ([n][512]) and per-leaf trimmed flags
 * (bit0 diag, bit1 x, bit2 y, bit3 z). */
int uaamg_poisson_level_coefficients(const uaamg_poisson* h, int level, float* diag, float* cx,
                                     float* cy, float* cz, uint8_t* flags);
/* Coarsest-level solve (Eigen CG, 10 iterations, zero guess: .cpp:2114-2152). */
int uaamg_poisson_coarsest_solve(uaamg_poisson* h, const float* rhs, float* out);
/* One preconditioner application z = M^-1 r (muCyclePreconditioner<2,true>(z, r, 0, 3)). */
int uaamg_poisson_precondition(uaamg_poisson* h, const float* r, float* z);

/* Diagnostics: one PCG solve (device pointers) driven from the host with a
 * CUDA event pair around every kernel; returns per kernel class its total
 * device time and launch count.  names: max_classes * 64 chars.  No
 * counterpart in the reference (it keeps wall-clock timers, singletons/Timer.h). */
int uaamg_poisson_profile_pcg(uaamg_poisson* h, float* d_pressure, const float* d_rhs, int max_classes,
                              char* names, double* total_ms, int64_t* counts, int* nclasses);

/* Stream (cudaStream_t as void*) used by *_device calls; NULL = the handle's own stream.
 * The handle's own stream is non-blocking: it is not ordered with the legacy
 * default stream or any other stream, so device inputs written on another
 * stream must be complete (or that stream's work ordered before the call, by
 * an event the handle's stream waits on) before a call reads them, and work
 * on other streams that reads a call's device outputs waits for the handle's
 * stream the same way.  uaamg_poisson_get_stream returns the stream the
 * handle's calls run on. */
int uaamg_poisson_set_stream(uaamg_poisson* h, void* stream);
int uaamg_poisson_get_stream(const uaamg_poisson* h, void** stream);
/* PCG driver: 1 (default) host-driven loop for a handle's first solve and the
 * CUDA-graph solve (conditional WHILE node) from the second solve on; 2 the
 * graph always; 0 the host-driven loop always.
 * In mode 1 a handle's first solve may replay a graph from the process's
 * solve-graph cache instead: when the exact launch sequence of the solve
 * (kernels, shapes, argument bytes, i.e. the same hierarchy shape with its
 * buffers at the same addresses) equals that of a graph captured for an
 * earlier handle.  A graph is captured for the cache the second time a launch
 * sequence is seen.  Results are the same bits as the host-driven loop.
 * Environment UAAMG_SOLVE_GRAPH_CACHE=0 (read at handle creation) turns it off. */
int uaamg_poisson_set_graph_mode(uaamg_poisson* h, int use_graph);
/* Solve-graph cache counters of the process (pressure and viscosity solves):
 * first solves that replayed a cached graph, and graphs captured into the
 * cache. */
int uaamg_solve_graph_cache_stats(int64_t* hits, int64_t* captures);
/* Kernels launched through this handle since it was created: hierarchy build,
 * right-hand side and every solve (kernels inside the solve graph included). */
int64_t uaamg_poisson_kernel_launches(const uaamg_poisson* h);

/* ======================================================================== */
/* Mixed-precision pressure solve: PoissonSolver::solveMultigridPCG
 * (simd_vdb_poisson.cpp:2155-2226) with the preconditioner's hierarchy
 * (coefficients and mu-cycle vectors of every level) stored in 16-bit floats
 * and FP32 arithmetic, the outer CG in FP32 on the FP32 level-0 operator with
 * FP64 dot accumulation, the true residual recomputed every
 * `replacement interval` iterations, and the coarsest level solved directly
 * in FP64 (dense inverse).  The reference has no such form; its FP32 solve is
 * uaamg_poisson_solve_pcg.  Jacobi smoothers only (the default
 * ScheduledRelaxedJacobi, or WeightedJacobi); the coarsest system must be
 * positive definite (a domain with a free surface). */
#define UAAMG_PRECISION_FP16 1
#define UAAMG_PRECISION_BF16 2
/* Build the 16-bit hierarchy and the FP64 coarsest inverse now (otherwise the
 * first mixed solve does it); setup_ms (may be NULL) receives the time taken. */
int uaamg_poisson_prepare_mixed(uaamg_poisson* h, int precision, double* setup_ms);
/* True-residual replacement interval of the mixed form (default 25). */
int uaamg_poisson_set_residual_replacement(uaamg_poisson* h, int every);
int uaamg_poisson_solve_pcg_mixed(uaamg_poisson* h, int precision, float* pressure, const float* rhs,
                                  int* iterations);
int uaamg_poisson_solve_pcg_mixed_device(uaamg_poisson* h, int precision, float* d_pressure, const float* d_rhs,
                                         int* iterations);
/* |b - A x|_inf and |b|_inf over the DOF, computed in FP64 from the FP32
 * level-0 matrix (device vectors): out[0], out[1].  An accuracy check with no
 * counterpart in the reference. */
int uaamg_poisson_true_residual_fp64(uaamg_poisson* h, const float* d_x, const float* d_b, double* out);
/* FP64 reference solution of the level-0 system A x = b (device pointers:
 * d_rhs float[leaf][512], d_x double[leaf][512] out), the yardstick the
 * accuracy of every form is stated against.  A is the matrix of getTriplets
 * (SIMD_UAAMG/simd_vdb_poisson.cpp:129-206) assembled from the FP32
 * coefficients, exactly in FP64; flexible PCG in FP64 preconditioned by the
 * handle's FP32 W-cycle on a power-of-two-scaled residual; stops when the true
 * residual |b - A x|_2 <= rel_tol |b|_2 (the criterion of Eigen's CG).
 * Returns UAAMG_SUCCESS, or UAAMG_FAILED after max_iter iterations;
 * *rel_residual = the final |b - A x|_2 / |b|_2.  No counterpart in the
 * reference (its harness compares against Eigen solvers). */
int uaamg_poisson_solve_fp64_reference(uaamg_poisson* h, const float* d_rhs, double* d_x, double rel_tol,
                                       int max_iter, int* iterations, double* rel_residual);

/* uaamg_poisson_solve_pcg_mixed_device with every kernel launched from a
 * host-driven loop and timed with CUDA events; per kernel class (label, up to
 * max_classes, names 64 bytes each) the summed ms and the launch count, as
 * uaamg_poisson_profile_pcg. */
int uaamg_poisson_profile_pcg_mixed(uaamg_poisson* h, int precision, float* d_pressure, const float* d_rhs,
                                    int max_classes, char* names, double* total_ms, int64_t* counts, int* nclasses);

/* ======================================================================== */
/* The steps either side of the pressure solve in a FLIP projection.        */

/* The liquid SDF adjusted inside solids before the pressure solve:
 * FLIP_Solver_OpenVDB::immerse_liquid_phi_in_solids (FLIP_vdb/FLIP_vdb.cpp:
 * 2856-2942), its value passes, on the liquid SDF's own leaves.  In leaves
 * where the solid SDF has a leaf at the same origin (probeConstLeaf), with the
 * solid SDF sampled trilinearly (BoxSampler) at voxel centres:
 *   1. active voxels inside the solid: phi -= dx / 2 (:2860-2877);
 *   2. voxels active after one 26-neighbour dilation, inside the solid: the
 *      least of 3 dx and the pass-1 values of the face neighbours visited in
 *      the order +x, -x, +y, -y, +z, -z up to the first negative one, if there
 *      is one; else a negative value becomes max(background, -solid)
 *      (:2883-2938).
 * values_out: float[leaf_count][512] (may alias the liquid's device values in
 * the _device form).  The two topology dilations of the reference (:2881, 26
 * neighbours; :2941, 6 neighbours) are the caller's: leaves they add keep the
 * background value, as in the reference, whose second pass only visits the
 * leaves that existed before the first dilation.  The _device form takes the
 * liquid's values in device memory (values_on_device) or host memory, writes
 * device memory on `stream` and returns without waiting. */
int uaamg_immerse_liquid_phi(const uaamg_leaf_grid* solid_sdf, const uaamg_leaf_grid* liquid_phi, float dx,
                             float* values_out);
int uaamg_immerse_liquid_phi_device(const uaamg_leaf_grid* solid_sdf, const uaamg_leaf_grid* liquid_phi, float dx,
                                    float* d_values_out, void* stream);

/* Solid face weights on a given topology: for every active voxel (masks may
 * be NULL: all voxels), 1 - fraction_inside of the solid over each of its
 * three minus faces, from the solid SDF at the 8 voxel corners, clamped to
 * [0, 1] and set to 0 below 1e-2; inactive voxels get (1, 1, 1).  weights:
 * float[leaf_count][512][3].  Replaces FLIP_Solver_OpenVDB::
 * calculate_face_weights (FLIP_vdb/FLIP_vdb.cpp:2669-2752) on the topology
 * the caller provides there (the liquid SDF's dilated by 2 voxels,
 * :2672-2675); fraction_inside(bl, br, tl, tr) is levelset_util.cpp:23-100.
 * The _device form writes device memory on the given stream (NULL: the
 * default stream) and returns without waiting. */
int uaamg_face_weights(const uaamg_leaf_grid* solid_sdf, int64_t leaf_count, const int32_t* origins,
                       const uint64_t* masks, float* weights);
int uaamg_face_weights_device(const uaamg_leaf_grid* solid_sdf, int64_t leaf_count, const int32_t* origins,
                              const uint64_t* masks, float* d_weights, void* stream);

/* Pressure-gradient update of one velocity channel (0 x, 1 y, 2 z) with the
 * pressure solution of handle h (leaf-dense on its level 0): at every active
 * voxel of `velocity` whose face weight is positive and which has a DOF on
 * either side, u += -dt (p - p_below) / dx / theta (theta = fraction_inside
 * of the liquid SDF between the two cells, at least 0.02, when either is
 * air); the reflected velocity is the updated one plus the update again; a
 * face with weight w < 1 then becomes (1 - s) u + s u_solid with
 * s = (1 - w) friction.  Voxels without an update become inactive.  Outputs
 * (float[leaf][512], uint64[leaf][8]): velocity_out, mask_out (the new active
 * set), update_out and reflected_out (may be NULL; the input value where
 * there is no update).  Replaces FLIP_Solver_OpenVDB::apply_pressure_gradient
 * (FLIP_vdb.cpp:2571-2667) for one channel; friction is
 * boundary_friction_coefficient. */
int uaamg_poisson_apply_pressure_gradient(uaamg_poisson* h, const uaamg_leaf_grid* liquid_phi,
                                          const uaamg_leaf_grid* face_weights, const uaamg_leaf_grid* solid_velocity,
                                          const float* pressure, float dt, float friction, int channel,
                                          const uaamg_leaf_grid* velocity, float* velocity_out, uint64_t* mask_out,
                                          float* update_out, float* reflected_out);
/* Device form: pressure, velocity (updated in place), the mask and the
 * optional outputs are device pointers; velocity->masks and ->origins stay
 * host pointers.  Runs on the handle's stream without waiting. */
int uaamg_poisson_apply_pressure_gradient_device(uaamg_poisson* h, const uaamg_leaf_grid* liquid_phi,
                                                 const uaamg_leaf_grid* face_weights,
                                                 const uaamg_leaf_grid* solid_velocity, const float* d_pressure,
                                                 float dt, float friction, int channel,
                                                 const uaamg_leaf_grid* velocity, float* d_velocity,
                                                 uint64_t* d_mask_out, float* d_update_out, float* d_reflected_out);

/* Velocity extrapolation of one channel into new voxels, n_layer layers
 * (vdb_velocity_extrapolator::union_extrapolate, FLIP_vdb/
 * vdb_velocity_extrapolator.cpp:585-662, the part after its topology steps).
 * The output grid has n_out leaves (out_origins [n_out][3]); values
 * [n_out][512] and masks [n_out][8] hold the channel (new leaves: the
 * background, inactive) and are updated in place.  The fill set lists, for
 * n_fill distinct output leaves fill_leaf[e], the voxels still to fill
 * (fill_masks [n_fill][8]: the union topology minus the channel's active
 * voxels).  Each layer gives every fill voxel with an active face neighbour
 * (active before the layer) the mean of those neighbours, summed in the order
 * -x, +x, -y, +y, -z, +z, and makes it active.  Host pointers. */
int uaamg_extrapolate_channel(int n_layer, int64_t n_out, const int32_t* out_origins, float* values,
                              uint64_t* masks, int64_t n_fill, const int32_t* fill_leaf,
                              const uint64_t* fill_masks);
/* The same with values [n_out][512] and masks [n_out][8] in device memory,
 * updated in place on `stream` (NULL: the legacy default stream); out_origins,
 * fill_leaf and fill_masks are host arrays (the topology, uploaded on the
 * stream).  Enqueued only: the call returns before the layers finish. */
int uaamg_extrapolate_channel_device(int n_layer, int64_t n_out, const int32_t* out_origins, float* values,
                                     uint64_t* masks, int64_t n_fill, const int32_t* fill_leaf,
                                     const uint64_t* fill_masks, void* stream);

/* ======================================================================== */
/* Batched pressure solves: PoissonSolver::solveMultigridPCG
 * (simd_vdb_poisson.cpp:2155-2226) of many independent instances in one CUDA
 * graph launch.  The reference has no batched form; each instance's result,
 * iteration count and status are identical to its own solveMultigridPCG.
 *
 * A batch references solver handles made by uaamg_poisson_create (hierarchies
 * of any size and depth); it does not own them, and they must outlive it.
 * While a batch solve runs, its instances must not be used on their own. */
typedef struct uaamg_batch uaamg_batch;

int uaamg_batch_create(int count, uaamg_poisson* const* instances, uaamg_batch** out);
int uaamg_batch_destroy(uaamg_batch* b);
int uaamg_batch_size(const uaamg_batch* b);
/* mSmoother, mMaxIteration, mRelativeTolerance for every instance of the
 * batch (defaults: those of the first instance at creation) */
int uaamg_batch_set_smoother(uaamg_batch* b, int smoother);
int uaamg_batch_set_max_iterations(uaamg_batch* b, int max_iterations);
int uaamg_batch_set_relative_tolerance(uaamg_batch* b, float tolerance);
/* Solve every instance i: pressure[i] (in: initial guess, out: solution) and
 * rhs[i] are leaf-dense vectors of instance i (host pointers here, device
 * pointers in the _device form).  iterations[i] and status[i]
 * (UAAMG_SUCCESS / UAAMG_FAILED) may be NULL.  Returns UAAMG_SUCCESS when
 * every instance succeeded, UAAMG_FAILED otherwise, or a negative error. */
int uaamg_batch_solve_pcg(uaamg_batch* b, float* const* pressure, const float* const* rhs, int* iterations,
                          int* status);
int uaamg_batch_solve_pcg_device(uaamg_batch* b, float* const* d_pressure, const float* const* d_rhs,
                                 int* iterations, int* status);
/* Per-instance results of the last solve (any pointer may be NULL). */
int uaamg_batch_results(const uaamg_batch* b, int* iterations, int* status, float* final_residual);
/* Stream of the batch's calls (NULL = its own non-blocking stream; the
 * ordering rules of uaamg_poisson_set_stream apply). */
int uaamg_batch_set_stream(uaamg_batch* b, void* stream);
int uaamg_batch_get_stream(const uaamg_batch* b, void** stream);
/* 1 (default): host-driven loop for the batch's first solve, the CUDA graph
 * with a WHILE node from the second solve on; 2: the graph always; 0: the
 * host-driven loop always. */
int uaamg_batch_set_graph_mode(uaamg_batch* b, int use_graph);
/* Kernels launched by the last batched solve. */
int64_t uaamg_batch_kernel_launches(const uaamg_batch* b);

/* ======================================================================== */
/* Variational viscosity: simd_viscosity3d / L_with_level
 * (SIMD_UAAMG/simd_viscosity3d.h:12-320, simd_viscosity3d.cpp).
 *
 * Vectors are leaf-dense over the handle's level-0 leaf set, three channels:
 * float[3][leaf][512] (channel c = face velocity component c), zero at every
 * voxel that is not a DOF of that channel (uaamg_viscosity_topology gives the
 * leaves and the per-channel DOF masks).  All input grids share one index
 * space: voxel centre i at world i*dx, face channel c of voxel g at g - e_c/2
 * (the transforms of L_with_level::initialize_transforms, .cpp:80-148). */
typedef struct uaamg_viscosity uaamg_viscosity;

/* L_with_level apply modes (working_mode, simd_viscosity3d.h:14) */
#define UAAMG_VMODE_NORMAL 0
#define UAAMG_VMODE_RESIDUAL 1
#define UAAMG_VMODE_JACOBI 2
#define UAAMG_VMODE_RED_GS 3
#define UAAMG_VMODE_BLACK_GS 4

/* Level 0 and the multigrid hierarchy: replaces
 * L_with_level::create_viscosity_matrix(viscosity, liquid_sdf, solid_sdf, dt,
 * rho) (.cpp:14-50) and the hierarchy part of the simd_viscosity3d
 * constructor (.cpp:3621-3658: coarse levels while ndof > 4000, level-0
 * trimming, coarsest explicit solver).  dx is the voxel size of liquid_sdf.
 * viscosity may have no leaves (constant: its background), as at the call
 * site FLIP_vdb.cpp:3173-3182. */
int uaamg_viscosity_create(const uaamg_leaf_grid* viscosity, const uaamg_leaf_grid* liquid_sdf,
                           const uaamg_leaf_grid* solid_sdf, float dt, float rho, float dx,
                           uaamg_viscosity** out);
/* uaamg_viscosity_create with the construction enqueued on `stream` (see
 * uaamg_poisson_create_on_stream). */
int uaamg_viscosity_create_on_stream(const uaamg_leaf_grid* viscosity, const uaamg_leaf_grid* liquid_sdf,
                                     const uaamg_leaf_grid* solid_sdf, float dt, float rho, float dx, void* stream,
                                     uaamg_viscosity** out);
int uaamg_viscosity_destroy(uaamg_viscosity* h);
/* simd_viscosity3d::m_max_iter (100) */
int uaamg_viscosity_set_max_iterations(uaamg_viscosity* h, int max_iterations);
/* simd_viscosity3d::m_iteration of the last solve: the 0-based index of the
 * iteration in which pcg_solve returned */
int uaamg_viscosity_iterations(const uaamg_viscosity* h);
float uaamg_viscosity_final_residual(const uaamg_viscosity* h);
/* m_matrix_levels.size() and per level m_ndof / leaf count */
int uaamg_viscosity_num_levels(const uaamg_viscosity* h);
int64_t uaamg_viscosity_num_dof(const uaamg_viscosity* h, int level);
int64_t uaamg_viscosity_leaf_count(const uaamg_viscosity* h, int level);
/* Leaf set of a level (the coefficient pattern leaves, OpenVDB tree order):
 * origins [n][3] and the DOF masks of m_velocity_DOF, [3][n][8] (host memory). */
int uaamg_viscosity_topology(const uaamg_viscosity* h, int level, int32_t* origins, uint64_t* dof_masks);
/* DOF indices of m_velocity_DOF (set_dof, .cpp:500-538), [3][n][512], -1 off DOF. */
int uaamg_viscosity_dof_index(const uaamg_viscosity* h, int level, int32_t* out);

/* L_with_level::build_rhs(velocity, solid_velocity) (.cpp:2005-2087), the
 * m_rhs of the simd_viscosity3d constructor.  u, v, w: the three channels of
 * the packed3grids velocity; solid_velocity: a vec3 grid (may be NULL or have
 * no leaves). */
int uaamg_viscosity_build_rhs(uaamg_viscosity* h, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                              const uaamg_leaf_grid* w, const uaamg_leaf_grid* solid_velocity, float* rhs_out);
int uaamg_viscosity_build_rhs_device(uaamg_viscosity* h, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                                     const uaamg_leaf_grid* w, const uaamg_leaf_grid* solid_velocity,
                                     float* d_rhs_out);
/* The velocity at every DOF: the warm start the call site writes into the
 * result before pcg_solve (FLIP_vdb.cpp:3188-3198). */
int uaamg_viscosity_gather_velocity(uaamg_viscosity* h, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                                    const uaamg_leaf_grid* w, float* out);
int uaamg_viscosity_gather_velocity_device(uaamg_viscosity* h, const uaamg_leaf_grid* u,
                                           const uaamg_leaf_grid* v, const uaamg_leaf_grid* w, float* d_out);

/* simd_viscosity3d::pcg_solve(in_lhs, tolerance) (.cpp:3691-3754) with m_rhs =
 * rhs.  velocity holds the initial guess on entry.  Returns UAAMG_SUCCESS when
 * |r|_inf <= tolerance * |r0|_inf held, UAAMG_FAILED when the loop returned at
 * iteration max_iterations - 1 (the reference returns void in both cases and
 * never reports divergence); *iterations = m_iteration. */
int uaamg_viscosity_solve_pcg(uaamg_viscosity* h, float* velocity, const float* rhs, float tolerance,
                              int* iterations);
int uaamg_viscosity_solve_pcg_device(uaamg_viscosity* h, float* d_velocity, const float* d_rhs,
                                     float tolerance, int* iterations);
/* The viscosity step of the reference's call site in one call
 * (FLIP_vdb.cpp:3178-3219: simd_viscosity3d(L, liquid_velocity, solid_velocity),
 * the warm start from the velocity, pcg_solve): u, v, w (and the solid
 * velocity, which may be NULL) are uploaded once, the rhs and the initial
 * guess are built on the device, and only the solved velocity [3][nl][512]
 * is returned (host pointer).  Identical results to uaamg_viscosity_build_rhs +
 * uaamg_viscosity_gather_velocity + uaamg_viscosity_solve_pcg. */
int uaamg_viscosity_solve_velocity(uaamg_viscosity* h, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                                   const uaamg_leaf_grid* w, const uaamg_leaf_grid* solid_velocity, float tolerance,
                                   float* velocity_out, int* iterations);

/* Level operations (host pointers), for parity checks against the reference's
 * L_with_level members: one light_weight_applier pass (L_apply,
 * residual_apply, Jacobi_apply, and the RED_GS/BLACK_GS passes of one channel
 * in place, .cpp:2187-2302); XYZ_RBGS_apply (order 0) / ZYX_RBGS_apply
 * (order 1); restriction (.cpp:2353-2413); prolongation<true> (fine += P
 * coarse, .cpp:2659-2729); the coefficients [3][9][n][512] (diag, invdiag,
 * neg_x, neg_y, neg_z, cross T00, T01, T10, T11 of m_cross_channel[c]) and the
 * level-0 trimmed-leaf bits (bit 9*c+a, trim_default_nodes .cpp:1692-1721);
 * solve_exact on the coarsest level (.cpp:2652-2657); one mucycle as the
 * preconditioner (z = mucycle(0, r, 2, true, 0, 2), .cpp:3837-3884). */
int uaamg_viscosity_level_apply(uaamg_viscosity* h, int level, int mode, int channel, const float* lhs,
                                const float* rhs, float* out);
int uaamg_viscosity_level_rbgs(uaamg_viscosity* h, int level, int order, float* lhs, const float* rhs);
int uaamg_viscosity_level_restrict(uaamg_viscosity* h, int fine_level, const float* fine, float* coarse);
int uaamg_viscosity_level_prolongate(uaamg_viscosity* h, int fine_level, const float* coarse, float* fine);
int uaamg_viscosity_level_coefficients(const uaamg_viscosity* h, int level, float* coef, uint32_t* trim);
int uaamg_viscosity_coarsest_solve(uaamg_viscosity* h, const float* rhs, float* out);
int uaamg_viscosity_precondition(uaamg_viscosity* h, const float* r, float* z);

/* Diagnostics: one host-driven solve with a CUDA event pair around every
 * kernel, per kernel class total device time and launch count (no
 * counterpart in the reference). */
int uaamg_viscosity_profile_pcg(uaamg_viscosity* h, float* d_velocity, const float* d_rhs, float tolerance,
                                int max_classes, char* names, double* total_ms, int64_t* counts,
                                int* nclasses);
/* Stream of the handle's calls (NULL = its own non-blocking stream; the
 * ordering rules of uaamg_poisson_set_stream apply). */
int uaamg_viscosity_set_stream(uaamg_viscosity* h, void* stream);
int uaamg_viscosity_get_stream(const uaamg_viscosity* h, void** stream);
/* 1 (default): host-driven first solve, CUDA graph afterwards; 2 graph always; 0 never.
 * In mode 1 the first solve may replay a graph of the solve-graph cache, as
 * for uaamg_poisson_set_graph_mode. */
int uaamg_viscosity_set_graph_mode(uaamg_viscosity* h, int use_graph);
int64_t uaamg_viscosity_kernel_launches(const uaamg_viscosity* h);

/* packed_FloatGrid3 (SIMD_UAAMG/packed3grids.h, .cpp:11-83): the velocity of
 * the reference's call sites as three staggered channel FloatGrids.
 * from_vec3 (:11-43): channel c of a Vec3fGrid (components 3) with the vec3
 * grid's leaf topology (its origins and masks): component c at active voxels,
 * background[c] elsewhere.  out_c* are [leaf_count][512] floats, host memory
 * (host values) or device memory (the _device form, device values, enqueued on
 * `stream`).  The reference also shifts channel c's world transform by -dx/2
 * along c; leaf grids are in index space and carry no transform. */
int uaamg_packed3_from_vec3(const uaamg_leaf_grid* vec3, float* out_c0, float* out_c1, float* out_c2);
int uaamg_packed3_from_vec3_device(const uaamg_leaf_grid* vec3, float* d_c0, float* d_c1, float* d_c2, void* stream);
/* to_vec3 (:46-83): the Vec3fGrid over the union of the channels' leaves
 * (OpenVDB tree order) and active masks; component c is channel c's value at
 * its active voxels and 0 elsewhere (background (0,0,0)).  The topology call
 * returns the union's leaf count (out_origins NULL) or fills out_origins
 * [n][3] and out_masks [n][8] (leaf_count in: their capacity).  The value call
 * fills [n][512][3] floats in that order. */
int uaamg_packed3_to_vec3_topology(const uaamg_leaf_grid* c0, const uaamg_leaf_grid* c1, const uaamg_leaf_grid* c2,
                                   int64_t* leaf_count, int32_t* out_origins, uint64_t* out_masks);
int uaamg_packed3_to_vec3(const uaamg_leaf_grid* c0, const uaamg_leaf_grid* c1, const uaamg_leaf_grid* c2,
                          float* out_values);
int uaamg_packed3_to_vec3_device(const uaamg_leaf_grid* c0, const uaamg_leaf_grid* c1, const uaamg_leaf_grid* c2,
                                 float* d_out_values, void* stream);

/* ---------------------------------------------------------------------------
 * Served form: many simulations' solves on one GPU (no counterpart in the
 * reference, which solves one domain per call).  A request is one simulation
 * domain asking for `substeps` solves of one kind -- FLIP_vdb's pressure
 * projection (FLIP_vdb.cpp:3118-3168) or its viscosity step (:3170-3216) --
 * each substep with new face velocities (uaamg_server_push_velocity).  The
 * server admits queued requests in submission order while their estimated
 * device footprint fits budget_bytes (and the resident caps), keeps each
 * request's hierarchy, face weights and warm start (the previous pressure)
 * on the device until its last substep, solves the pending substeps of all
 * resident pressure requests in one batched CUDA graph per round (batching 1)
 * or one after another (batching 0), and runs every viscosity request on a
 * lane of its own (a thread and a stream) in both modes.  Each pressure result
 * is checked in FP64 (|b - A x|_inf / |b|_inf).  A result is the same alone
 * and in the mix.  The loop runs on a thread of its own; every call below is
 * thread-safe.  Inputs are copied at the call (host grids into host memory,
 * device grids into device memory), so the caller may free them at once;
 * device grids must be complete when the call is made (the copy is not
 * ordered after work on the caller's streams). */
typedef struct uaamg_server uaamg_server;
#define UAAMG_SERVER_POISSON 0
#define UAAMG_SERVER_VISCOSITY 1
typedef struct {
    int64_t budget_bytes;       /* device memory the resident requests may use (64 GiB) */
    int32_t max_poisson;        /* resident pressure requests at most (256) */
    int32_t max_viscosity;      /* resident viscosity requests, i.e. lanes, at most (16) */
    int32_t admit_per_round;    /* admissions per loop round at most (8) */
    int32_t batching;           /* 1: one batched graph per pressure round; 0: every solve alone (1) */
    int32_t keep_results;       /* 1: keep every substep's solution for uaamg_server_result (0) */
    float pressure_tolerance;   /* relative residual of the pressure PCG (1e-7) */
    float viscosity_tolerance;  /* relative residual of the viscosity PCG (1e-6) */
} uaamg_server_options;
typedef struct {
    int64_t submitted, queued, resident, done, failed;
    int64_t solves, rounds, batch_builds;
    int64_t used_bytes, peak_bytes;
    int64_t pressure_solves;   /* solves done in pressure rounds */
    int64_t pressure_busy_us;  /* wall time inside pressure rounds (rhs, solves, FP64 checks), microseconds */
} uaamg_server_stats_t;
int uaamg_server_default_options(uaamg_server_options* options);
int uaamg_server_create(const uaamg_server_options* options, uaamg_server** out);
/* Stops the loop after the work in flight, frees every request. */
int uaamg_server_destroy(uaamg_server* s);
/* A pressure request: createPressurePoissonLaplacian's inputs (liquid SDF, face
 * weights), the solid velocity of its rhs, dt, dx.  UAAMG_ERR_OUT_OF_MEMORY
 * when its estimated footprint exceeds the whole budget. */
int uaamg_server_submit_poisson(uaamg_server* s, const uaamg_leaf_grid* liquid_phi,
                                const uaamg_leaf_grid* face_weights, const uaamg_leaf_grid* solid_velocity, float dt,
                                float dx, int substeps, int64_t* request);
/* A viscosity request: simd_viscosity3d's inputs (simd_viscosity3d.h:285-290). */
int uaamg_server_submit_viscosity(uaamg_server* s, const uaamg_leaf_grid* viscosity,
                                  const uaamg_leaf_grid* liquid_sdf, const uaamg_leaf_grid* solid_sdf,
                                  const uaamg_leaf_grid* solid_velocity, float dt, float rho, float dx, int substeps,
                                  int64_t* request);
/* The face velocities (packed3grids channels) of the request's next substep. */
int uaamg_server_push_velocity(uaamg_server* s, int64_t request, const uaamg_leaf_grid* u, const uaamg_leaf_grid* v,
                               const uaamg_leaf_grid* w);
/* Waits up to timeout_s for substep `substep` of a request; its PCG status
 * (UAAMG_SUCCESS / UAAMG_FAILED), iterations, FP64 relative residual
 * (pressure; -1 for viscosity) and latency (seconds from submission).
 * UAAMG_ERR_TIMEOUT when it is not solved in time. */
int uaamg_server_wait(uaamg_server* s, int64_t request, int substep, double timeout_s, int* status, int* iterations,
                      double* fp64_residual, double* latency_s);
/* A solved substep's solution (keep_results 1): *leaf_count leaves of level 0
 * (float[leaf][512] pressure, float[3][leaf][512] velocity); x may be NULL to
 * ask for the size. */
int uaamg_server_result(uaamg_server* s, int64_t request, int substep, int64_t* leaf_count, float* x);
int uaamg_server_stats(uaamg_server* s, uaamg_server_stats_t* out);

const char* uaamg_last_error(void);
int uaamg_device_count(void);

#ifdef __cplusplus
}
#endif
#endif
