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

/* ======================================================================== */
/* Variational viscosity (SIMD_UAAMG/simd_viscosity3d.cpp).
 *
 * A level is stored over one leaf set: the leaves of the union of the three
 * channels' DOF masks dilated by 2 (level 0) or 3 (coarse levels) voxels, in
 * OpenVDB tree order (the reference's coefficient pattern,
 * simd_viscosity3d.cpp:881-899 and :1353-1362).  Vectors are
 * [3 channels][leaf][512] floats over that set, 0 at non-DOF voxels.
 * Coefficients are [3 channels][9 arrays][leaf][512]: diag, invdiag, neg_x,
 * neg_y, neg_z, T00, T01, T10, T11 (T = m_cross_channel[channel][j][k]). */
typedef struct orc_visc orc_visc;

enum { ORC_VA_DIAG = 0, ORC_VA_INVDIAG = 1, ORC_VA_NEGX = 2, ORC_VA_NEGY = 3, ORC_VA_NEGZ = 4,
       ORC_VA_T00 = 5, ORC_VA_T01 = 6, ORC_VA_T10 = 7, ORC_VA_T11 = 8, ORC_VA_COUNT = 9 };
/* L_with_level::working_mode (simd_viscosity3d.h:14) */
enum { ORC_VMODE_NORMAL = 0, ORC_VMODE_RESIDUAL = 1, ORC_VMODE_JACOBI = 2,
       ORC_VMODE_RED_GS = 3, ORC_VMODE_BLACK_GS = 4 };

/* simd_viscosity3d ctor (simd_viscosity3d.cpp:3621-3658) minus the rhs:
 * level 0 from the viscosity, liquid SDF and solid SDF grids, coarse levels
 * while ndof > 4000 (if build_hierarchy), level-0 trimming, coarsest matrix.
 * All grids share one index space (voxel centre i at world i*dx). */
orc_visc* orc_visc_create(
    int64_t liq_n, const int32_t* liq_origins, const uint64_t* liq_masks,
    const float* liq_values, float liq_background,
    int64_t sol_n, const int32_t* sol_origins, const float* sol_values, float sol_background,
    int64_t mu_n, const int32_t* mu_origins, const float* mu_values, float mu_background,
    float dt, float rho, float dx, int build_hierarchy);
void orc_visc_free(orc_visc* h);

int  orc_visc_num_levels(const orc_visc* h);
int  orc_visc_leaf_count(const orc_visc* h, int level);
int  orc_visc_ndof(const orc_visc* h, int level);
/* origins [nl][3], DOF masks [3][nl][8] */
void orc_visc_topology(const orc_visc* h, int level, int32_t* origins, uint64_t* dof_masks);
/* effective coefficients [3][9][nl][512] and per-leaf trimmed bits
 * (bit 9*channel+array) */
void orc_visc_coefficients(const orc_visc* h, int level, float* coef, uint32_t* trim);
void orc_visc_defaults(const orc_visc* h, int level, float* out27);
/* DOF index [3][nl][512], -1 at non-DOF voxels */
void orc_visc_dof_index(const orc_visc* h, int level, int32_t* out);
/* explicit matrix triplets (explicit_matrix_reducer :2415-2642); NULL to count */
int64_t orc_visc_triplets(const orc_visc* h, int level, int32_t* rows, int32_t* cols, float* vals);

/* L_with_level::build_rhs (:2005-2087): velocity channels are scalar grids,
 * solid velocity a vec3 grid (n may be 0).  rhs_out [3][nl][512]. */
void orc_visc_build_rhs(const orc_visc* h,
    int64_t u_n, const int32_t* u_origins, const float* u_values, float u_bg,
    int64_t v_n, const int32_t* v_origins, const float* v_values, float v_bg,
    int64_t w_n, const int32_t* w_origins, const float* w_values, float w_bg,
    int64_t sv_n, const int32_t* sv_origins, const float* sv_values, const float* sv_bg3,
    float* rhs_out);

/* One light_weight_applier pass (:2849-3603).  NORMAL/RESIDUAL/JACOBI write
 * all three channels of out; RED_GS/BLACK_GS update channel `channel` of
 * `out` in place (out holds the current iterate). */
void orc_visc_apply(orc_visc* h, int level, int mode, int channel,
                    const float* lhs, const float* rhs, float* out);
/* XYZ_RBGS_apply (order 0) / ZYX_RBGS_apply (order 1), in place. */
void orc_visc_rbgs(orc_visc* h, int level, int order, float* lhs, const float* rhs);
void orc_visc_restrict(const orc_visc* h, int fine_level, const float* fine, float* coarse);
/* prolongation<true>: fine += P coarse */
void orc_visc_prolongate(const orc_visc* h, int fine_level, const float* coarse, float* fine);
void orc_visc_coarsest_solve(orc_visc* h, const float* rhs, float* out);
/* Summation order of the viscosity coarsest CG (the reference leaves it to
 * Eigen): the CUDA kernel's 256-thread tree order with fused vector updates
 * (the default), or plain sequential sums with separate multiply and add. */
/* 1 (default): the Poisson applier runs 8-wide AVX2 z-lanes; 0: the scalar
 * per-voxel path.  Both give the same bits. */
void orc_set_simd(int on);
#define ORC_CG_ORDER_KERNEL 0
#define ORC_CG_ORDER_SEQUENTIAL 1
void orc_visc_set_coarsest_order(orc_visc* h, int order);
/* out = mucycle(0, r, mu=2, for_precon=true, level 0, n=2) */
void orc_visc_precondition(orc_visc* h, const float* r, float* out);
/* simd_viscosity3d::pcg_solve (:3691-3754) on x in place.  Returns 0 when
 * the stopping test held, 1 when it stopped at max_iter-1; *iterations is
 * m_iteration (the 0-based index of the last iteration run). */
int orc_visc_pcg(orc_visc* h, float* x, const float* b, float tol, int max_iter,
                 int* iterations, float* final_abs_res);
float orc_visc_abs_max(const orc_visc* h, int level, const float* v);
float orc_visc_dot(const orc_visc* h, int level, const float* a, const float* b);

/* ------------------------------------------------------------------------ */
/* The steps either side of the pressure solve (projection_oracle.c). */
float orc_fraction_inside4(float phi_bl, float phi_br, float phi_tl, float phi_tr);
/* the restated scalar helpers, for the tests that pin them against the
 * reference's own build (oracle/_ref) */
float orc_fraction_inside2(float l, float r);
float orc_tet_fraction(float p0, float p1, float p2, float p3);
float orc_cube_fraction(float p000, float p100, float p010, float p110, float p001, float p101, float p011,
                        float p111);
void orc_face_weights(int64_t solid_n, const int32_t* solid_origins, const float* solid_values, float solid_bg,
                      int64_t n, const int32_t* origins, const uint64_t* masks, float* out);
void orc_pressure_gradient(int64_t phi_n, const int32_t* phi_origins, const float* phi_values, float phi_bg,
                           int64_t fw_n, const int32_t* fw_origins, const float* fw_values, const float* fw_bg3,
                           int64_t sv_n, const int32_t* sv_origins, const float* sv_values, const float* sv_bg3,
                           int64_t p_n, const int32_t* p_origins, const uint64_t* p_masks, const float* p_values,
                           float in_dt, float dx, float friction, int channel,
                           int64_t v_n, const int32_t* v_origins, const uint64_t* v_masks, const float* v_values,
                           float* v_out, uint64_t* mask_out, float* update_out, float* reflected_out);
void orc_immerse_liquid_phi(int64_t solid_n, const int32_t* solid_origins, const float* solid_values, float solid_bg,
                            int64_t n, const int32_t* origins, const uint64_t* masks, const float* values,
                            float liquid_bg, float dx, float* values_out);
void orc_extrapolate_channel(int n_layer, int64_t n_out, const int32_t* out_origins, float* values,
                             uint64_t* masks, int64_t n_fill, const int32_t* fill_leaf, const uint64_t* fill_masks);

#ifdef __cplusplus
}
#endif
#endif
