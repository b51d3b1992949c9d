/*
 * uaamg_oracle.h -- CPU oracle for the UAAMG-PCG hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * SIMD_UAAMG Poisson solver (SIMD_UAAMG/simd_vdb_poisson.cpp) on flattened
 * 8^3 leaf arrays.  It is the checker for the CUDA library and the timed CPU
 * baseline in bench.py.  Nothing in the product library links or calls it.
 *
 * Parity status: UNPINNED.  The reference needs OpenVDB, TBB and Eigen, none of
 * which exist on this machine, and it ships no golden vectors or known-answer
 * tests, so the restatement is checked against hand-derivable identities and an
 * independent explicit-matrix formulation (CG_benchmarks/main.cpp:1070-1074)
 * rather than against outputs of the reference itself.
 *
 * Conventions (same as OpenVDB's LeafNode<float,3>):
 *   voxel offset inside a leaf = 64*x + 8*y + z (local coords 0..7)
 *   value mask = 8 x uint64, bit (off & 63) of word (off >> 6)
 *   leaf origins are multiples of 8
 * Vectors are leaf-dense: [leaf][512] floats over a level's DOF leaves
 * (non-empty leaves in OpenVDB tree order), 0 at non-DOF voxels.
 */
#ifndef UAAMG_ORACLE_H
#define UAAMG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_poisson orc_poisson;

/* Smoothers, same numbering as PoissonSolver::SmootherOption
 * (SIMD_UAAMG/simd_vdb_poisson.h:143-148). */
enum { ORC_SMOOTH_SCHEDULED_JACOBI = 0, ORC_SMOOTH_WEIGHTED_JACOBI = 1,
       ORC_SMOOTH_RBGS = 2, ORC_SMOOTH_SPAI0 = 3 };

/* Apply modes of LaplacianApplySIMD::WorkingMode (simd_vdb_poisson.cpp:685-692). */
enum { ORC_MODE_JACOBI = 0, ORC_MODE_RESIDUAL = 1, ORC_MODE_LAPLACIAN = 2,
       ORC_MODE_RED_GS = 3, ORC_MODE_BLACK_GS = 4, ORC_MODE_SPAI0 = 5 };

/* Build level 0 (createPressurePoissonLaplacian) and, if build_hierarchy,
 * the coarse levels (PoissonSolver ctor).  Grids are flattened leaf grids:
 * n leaves, origins [n][3], masks [n][8] (NULL = all active), values
 * [n][512][comps], background [comps]. */
orc_poisson* orc_poisson_create(
    int64_t phi_n, const int32_t* phi_origins, const uint64_t* phi_masks,
    const float* phi_values, float phi_background,
    int64_t fw_n, const int32_t* fw_origins, const float* fw_values,
    const float* fw_background3,
    float dt, float dx, int build_hierarchy);
void orc_poisson_free(orc_poisson* h);

int  orc_num_levels(const orc_poisson* h);
int  orc_level_leaf_count(const orc_poisson* h, int level);
int  orc_level_ndof(const orc_poisson* h, int level);
void orc_level_topology(const orc_poisson* h, int level, int32_t* origins, uint64_t* masks);
/* Effective coefficients (trimmed leaves hold the defaults) and per-leaf
 * trimmed flags (bit0 diag, bit1 x, bit2 y, bit3 z). */
void orc_level_coefficients(const orc_poisson* h, int level, float* diag, float* cx,
                            float* cy, float* cz, uint8_t* flags);
void orc_level_defaults(const orc_poisson* h, int level, float* out4);

/* BuildPoissonRhs (simd_vdb_poisson.cpp:19-127). Velocity grids are scalar
 * leaf grids; solid velocity is a vec3 leaf grid (n may be 0). */
void orc_build_rhs(const orc_poisson* h,
    int64_t fw_n, const int32_t* fw_origins, const float* fw_values, const float* fw_bg3,
    int64_t vx_n, const int32_t* vx_origins, const float* vx_values, float vx_bg,
    int64_t vy_n, const int32_t* vy_origins, const float* vy_values, float vy_bg,
    int64_t vz_n, const int32_t* vz_origins, const float* vz_values, float vz_bg,
    int64_t sv_n, const int32_t* sv_origins, const float* sv_values, const float* sv_bg3,
    float* rhs_out);

/* One apply pass at a level (LightWeightApplier::operator()). weight is the
 * Jacobi weight; w_sor the SOR weight used by the GS modes. */
void orc_apply(orc_poisson* h, int level, int mode, float weight, float w_sor,
               const float* lhs, const float* rhs, float* out);
/* First sweeps from a zero guess (simd_vdb_poisson.cpp:1435-1582). */
void orc_first_jacobi(orc_poisson* h, int level, float weight, const float* rhs, float* out);
void orc_first_spai0(orc_poisson* h, int level, const float* rhs, float* out);
void orc_first_rbgs(orc_poisson* h, int level, int red_first, float w_sor,
                    const float* rhs, float* out);
/* restriction (fine level -> level+1) and prolongation (level+1 -> level). */
void orc_restrict(const orc_poisson* h, int fine_level, const float* fine, float* coarse);
void orc_prolongate(const orc_poisson* h, int fine_level, const float* coarse, float* fine,
                    float alpha);
/* Coarsest-level CG restated from Eigen::ConjugateGradient (maxIterations 10). */
void orc_coarsest_solve(orc_poisson* h, const float* rhs, float* out);
/* One preconditioner application z = M^{-1} r at level 0 (mu=2, n=3). */
void orc_precondition(orc_poisson* h, int smoother, const float* r, float* z);

/* PoissonSolver::solveMultigridPCG / solvePureMultigrid.  Returns 0 SUCCESS, 1 FAILED. */
int orc_solve_pcg(orc_poisson* h, float* x, const float* b, float rel_tol, int max_iter,
                  int smoother, int* iterations, float* final_abs_res);
int orc_solve_mg(orc_poisson* h, float* x, const float* b, float rel_tol, int max_iter,
                 int smoother, int* iterations, float* final_abs_res);

/* Level-0 BLAS-1 (simd_vdb_poisson.cpp:2270-2320). */
float orc_abs_max(const orc_poisson* h, int level, const float* v);
float orc_dot(const orc_poisson* h, int level, const float* a, const float* b);

/* Explicit matrix triplets (getTriplets, simd_vdb_poisson.cpp:129-206). Returns count;
 * pass NULL arrays to query the count. */
int64_t orc_triplets(const orc_poisson* h, int level, int32_t* rows, int32_t* cols, float* vals);
/* DOF index of every voxel of a level, -1 at non-DOF voxels ([leaf][512]). */
void orc_dof_index(const orc_poisson* h, int level, int32_t* out);

void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
