// uaamg_simd.hpp -- header-only C++ facade with the reference's class names
// over the C ABI in uaamg.h, so FLIP_vdb-style call sites read the same:
// pressure (FLIP_vdb.cpp:3118-3168: createPressurePoissonLaplacian,
// PoissonSolver, mRelativeTolerance, mSmoother,
// createPressurePoissonRightHandSide, solveMultigridPCG, FAILED ->
// solvePureMultigrid) and viscosity (FLIP_vdb.cpp:3170-3216:
// simd_viscosity3d, m_matrix_levels[0]->get_zero_vec(), warm start,
// pcg_solve, m_iteration, m_ndof).
//
// Grids are flattened OpenVDB leaf lists (uaamg::LeafGrid); the result
// vectors are leaf-dense float[leaf][512] over the DOF leaves returned by
// LaplacianWithLevel::dofTopology().
//
// Errors are status codes, never exceptions, as in the reference (its solvers
// report through return values and printf, SIMD_UAAMG/simd_vdb_poisson.cpp:
// 2169-2206): a factory returns an empty pointer, a call returns the library's
// negative UAAMG_ERR_* code (solves keep SUCCESS / FAILED), a function that
// returns a vector returns an empty one and stores the code in *status when
// given.  Each error is also written to stderr; lastError() gives its text.
#pragma once
#include <cstdint>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "uaamg.h"

namespace simd_uaamg_b200 {

// A flattened openvdb::FloatGrid / Vec3fGrid (host memory).
struct LeafGrid {
    std::vector<int32_t> origins;  // [n][3]
    std::vector<uint64_t> masks;   // [n][8] (empty = all active)
    std::vector<float> values;     // [n][512][components]
    int components = 1;
    float background[3] = {0.f, 0.f, 0.f};

    int64_t leafCount() const { return (int64_t)(origins.size() / 3); }
    uaamg_leaf_grid view() const {
        uaamg_leaf_grid g{};
        g.leaf_count = leafCount();
        g.origins = origins.empty() ? nullptr : origins.data();
        g.masks = masks.empty() ? nullptr : masks.data();
        g.values = values.empty() ? nullptr : values.data();
        g.components = components;
        g.values_on_device = 0;
        g.background[0] = background[0];
        g.background[1] = background[1];
        g.background[2] = background[2];
        return g;
    }
};

// The message of the last failed library call on this thread.
inline std::string lastError() { return uaamg_last_error(); }

// Passes rc through; a negative code (an error) is reported on stderr.
inline int report(int rc, const char* what) {
    if (rc < 0) std::fprintf(stderr, "uaamg: %s failed (%d): %s\n", what, rc, uaamg_last_error());
    return rc;
}
inline void set_status(int* status, int rc) {
    if (status) *status = rc;
}

// LaplacianWithLevel (SIMD_UAAMG/simd_vdb_poisson.h:13-138): here the level-0
// operator together with its device hierarchy.
class LaplacianWithLevel {
public:
    using Ptr = std::shared_ptr<LaplacianWithLevel>;

    // an empty pointer on failure (*status, when given, receives the code)
    static Ptr createPressurePoissonLaplacian(const LeafGrid& liquidPhi, const LeafGrid& faceWeights, float dt,
                                              float dx, int* status = nullptr) {
        uaamg_leaf_grid a = liquidPhi.view(), b = faceWeights.view();
        uaamg_poisson* h = nullptr;
        int rc = report(uaamg_poisson_create(&a, &b, dt, dx, &h), "uaamg_poisson_create");
        set_status(status, rc);
        if (rc < 0) return Ptr();
        return Ptr(new LaplacianWithLevel(h));
    }
    ~LaplacianWithLevel() { uaamg_poisson_destroy(mHandle); }
    LaplacianWithLevel(const LaplacianWithLevel&) = delete;
    LaplacianWithLevel& operator=(const LaplacianWithLevel&) = delete;

    // an empty vector on failure
    std::vector<float> createPressurePoissonRightHandSide(const LeafGrid& faceWeights, const LeafGrid& vx,
                                                          const LeafGrid& vy, const LeafGrid& vz,
                                                          const LeafGrid& solidVelocity, float dt,
                                                          int* status = nullptr) {
        std::vector<float> rhs = getZeroVectorGrid();
        uaamg_leaf_grid w = faceWeights.view(), a = vx.view(), b = vy.view(), c = vz.view(), s = solidVelocity.view();
        int rc = report(uaamg_poisson_build_rhs(mHandle, &w, &a, &b, &c, &s, dt, rhs.data()), "build_rhs");
        set_status(status, rc);
        if (rc < 0) rhs.clear();
        return rhs;
    }
    std::vector<float> getZeroVectorGrid() const {
        return std::vector<float>((size_t)uaamg_poisson_leaf_count(mHandle, 0) * 512, 0.f);
    }
    int dofTopology(std::vector<int32_t>& origins, std::vector<uint64_t>& masks, int level = 0) const {
        int64_t n = uaamg_poisson_leaf_count(mHandle, level);
        if (n < 0) return report(UAAMG_ERR_INVALID_ARGUMENT, "dof_topology: invalid level");
        origins.resize((size_t)n * 3);
        masks.resize((size_t)n * 8);
        return report(uaamg_poisson_dof_topology(mHandle, level, origins.data(), masks.data()), "dof_topology");
    }
    int numDof(int level = 0) const { return (int)uaamg_poisson_num_dof(mHandle, level); }
    uaamg_poisson* handle() const { return mHandle; }

private:
    explicit LaplacianWithLevel(uaamg_poisson* h) : mHandle(h) {}
    uaamg_poisson* mHandle;
};

// PoissonSolver (SIMD_UAAMG/simd_vdb_poisson.h:141-207)
class PoissonSolver {
public:
    enum class SmootherOption { ScheduledRelaxedJacobi, WeightedJacobi, RedBlackGaussSeidel, SPAI0 };
    using SuccessType = int;
    static const SuccessType SUCCESS = 0;
    static const SuccessType FAILED = 1;

    explicit PoissonSolver(LaplacianWithLevel::Ptr level0) : mLevel0(std::move(level0)) {}

    // SUCCESS / FAILED, or a negative UAAMG_ERR_* code
    SuccessType solveMultigridPCG(std::vector<float>& inOutPressure, const std::vector<float>& rhs) {
        int rc = configure();
        if (rc < 0) return rc;
        if (!sizesMatch(inOutPressure, rhs)) return report(UAAMG_ERR_INVALID_ARGUMENT, "solve_pcg: vector size");
        int it = 0;
        rc = report(uaamg_poisson_solve_pcg(mLevel0->handle(), inOutPressure.data(), rhs.data(), &it), "solve_pcg");
        mIterationTaken = it;
        return rc;
    }
    SuccessType solvePureMultigrid(std::vector<float>& inOutPressure, const std::vector<float>& rhs) {
        int rc = configure();
        if (rc < 0) return rc;
        if (!sizesMatch(inOutPressure, rhs)) return report(UAAMG_ERR_INVALID_ARGUMENT, "solve_mg: vector size");
        int it = 0;
        rc = report(uaamg_poisson_solve_mg(mLevel0->handle(), inOutPressure.data(), rhs.data(), &it), "solve_mg");
        mIterationTaken = it;
        return rc;
    }

    int mIterationTaken = 0;
    int mMaxIteration = 100;
    float mRelativeTolerance = 1e-7f;
    SmootherOption mSmoother = SmootherOption::ScheduledRelaxedJacobi;

private:
    int configure() {
        if (!mLevel0) return report(UAAMG_ERR_INVALID_ARGUMENT, "PoissonSolver: no level-0 operator");
        int rc = report(uaamg_poisson_set_smoother(mLevel0->handle(), (int)mSmoother), "set_smoother");
        if (rc == 0) rc = report(uaamg_poisson_set_max_iterations(mLevel0->handle(), mMaxIteration), "set_max_iterations");
        if (rc == 0)
            rc = report(uaamg_poisson_set_relative_tolerance(mLevel0->handle(), mRelativeTolerance), "set_tolerance");
        return rc;
    }
    bool sizesMatch(const std::vector<float>& x, const std::vector<float>& b) const {
        size_t n = (size_t)uaamg_poisson_leaf_count(mLevel0->handle(), 0) * 512;
        return x.size() == n && b.size() == n;
    }
    LaplacianWithLevel::Ptr mLevel0;
};

// Three face-velocity channels (packed_FloatGrid3, SIMD_UAAMG/packed3grids.h:5-23).
struct PackedLeafGrid3 {
    LeafGrid v[3];
};

// L_with_level (SIMD_UAAMG/simd_viscosity3d.h:60-200): the level-0 viscosity
// matrix together with its device hierarchy.
class L_with_level {
public:
    using Ptr = std::shared_ptr<L_with_level>;

    // create_viscosity_matrix (simd_viscosity3d.h:86-89); dx is the voxel
    // size of liquid_sdf in the reference
    // an empty pointer on failure
    static Ptr create_viscosity_matrix(const LeafGrid& viscosity, const LeafGrid& liquidSdf,
                                       const LeafGrid& solidSdf, float dt, float rho, float dx,
                                       int* status = nullptr) {
        uaamg_leaf_grid m = viscosity.view(), l = liquidSdf.view(), s = solidSdf.view();
        uaamg_viscosity* h = nullptr;
        int rc = report(uaamg_viscosity_create(&m, &l, &s, dt, rho, dx, &h), "uaamg_viscosity_create");
        set_status(status, rc);
        if (rc < 0) return Ptr();
        return Ptr(new L_with_level(h));
    }
    ~L_with_level() { uaamg_viscosity_destroy(mHandle); }
    L_with_level(const L_with_level&) = delete;
    L_with_level& operator=(const L_with_level&) = delete;

    // get_zero_vec: three channels, float[3][leaf][512] over dofTopology()
    std::vector<float> get_zero_vec(int level = 0) const {
        return std::vector<float>((size_t)3 * uaamg_viscosity_leaf_count(mHandle, level) * 512, 0.f);
    }
    // build_rhs (simd_viscosity3d.cpp:1724-2087); an empty vector on failure
    std::vector<float> build_rhs(const PackedLeafGrid3& velocity, const LeafGrid& solidVelocity,
                                 int* status = nullptr) {
        std::vector<float> rhs = get_zero_vec();
        uaamg_leaf_grid u = velocity.v[0].view(), v = velocity.v[1].view(), w = velocity.v[2].view();
        uaamg_leaf_grid s = solidVelocity.view();
        int rc = report(uaamg_viscosity_build_rhs(mHandle, &u, &v, &w, &s, rhs.data()), "viscosity build_rhs");
        set_status(status, rc);
        if (rc < 0) rhs.clear();
        return rhs;
    }
    // the velocity at every DOF: the warm start of FLIP_vdb.cpp:3186-3198; an empty vector on failure
    std::vector<float> warm_start(const PackedLeafGrid3& velocity, int* status = nullptr) {
        std::vector<float> x = get_zero_vec();
        uaamg_leaf_grid u = velocity.v[0].view(), v = velocity.v[1].view(), w = velocity.v[2].view();
        int rc = report(uaamg_viscosity_gather_velocity(mHandle, &u, &v, &w, x.data()), "gather_velocity");
        set_status(status, rc);
        if (rc < 0) x.clear();
        return x;
    }
    int dofTopology(std::vector<int32_t>& origins, std::vector<uint64_t>& masks, int level = 0) const {
        int64_t n = uaamg_viscosity_leaf_count(mHandle, level);
        if (n < 0) return report(UAAMG_ERR_INVALID_ARGUMENT, "viscosity topology: invalid level");
        origins.resize((size_t)n * 3);
        masks.resize((size_t)n * 3 * 8);
        return report(uaamg_viscosity_topology(mHandle, level, origins.data(), masks.data()), "viscosity topology");
    }
    int64_t m_ndof() const { return uaamg_viscosity_num_dof(mHandle, 0); }
    uaamg_viscosity* handle() const { return mHandle; }

private:
    explicit L_with_level(uaamg_viscosity* h) : mHandle(h) {}
    uaamg_viscosity* mHandle;
};

// simd_viscosity3d (SIMD_UAAMG/simd_viscosity3d.h:280-330)
class simd_viscosity3d {
public:
    // simd_viscosity3d(viscosity, liquid_sdf, solid_sdf, liquid_velocity,
    // solid_velocity, dt, rho) (simd_viscosity3d.h:285-290)
    simd_viscosity3d(const LeafGrid& viscosity, const LeafGrid& liquidSdf, const LeafGrid& solidSdf,
                     const PackedLeafGrid3& liquidVelocity, const LeafGrid& solidVelocity, float dt, float rho,
                     float dx)
        : simd_viscosity3d(L_with_level::create_viscosity_matrix(viscosity, liquidSdf, solidSdf, dt, rho, dx),
                           liquidVelocity, solidVelocity) {}
    // simd_viscosity3d(level0, liquid_velocity, solid_velocity) (:292-294).
    // A constructor cannot return a code: m_status holds it (0, or the
    // negative code of the failed matrix build or rhs), and pcg_solve returns
    // it without solving.
    simd_viscosity3d(L_with_level::Ptr level0, const PackedLeafGrid3& liquidVelocity, const LeafGrid& solidVelocity)
        : m_level0(std::move(level0)) {
        if (!m_level0) {
            m_status = report(UAAMG_ERR_INVALID_ARGUMENT, "simd_viscosity3d: no level-0 matrix");
            return;
        }
        m_rhs = m_level0->build_rhs(liquidVelocity, solidVelocity, &m_status);
        m_ndof = m_level0->m_ndof();
    }

    // pcg_solve (simd_viscosity3d.cpp:3691-3754): in_lhs holds the warm start
    // and receives the solution.  Returns 0 or a negative UAAMG_ERR_* code
    // (the reference returns nothing; a call site may ignore the value).
    int pcg_solve(std::vector<float>& inLhs, float tolerance) {
        if (m_status < 0) return m_status;
        if (inLhs.size() != m_rhs.size())
            return report(UAAMG_ERR_INVALID_ARGUMENT, "viscosity solve_pcg: vector size");
        int rc = report(uaamg_viscosity_set_max_iterations(m_level0->handle(), m_max_iter), "set_max_iterations");
        if (rc < 0) return rc;
        int it = 0;
        rc = report(uaamg_viscosity_solve_pcg(m_level0->handle(), inLhs.data(), m_rhs.data(), tolerance, &it),
                    "viscosity solve_pcg");
        m_iteration = it;
        return rc < 0 ? rc : 0;
    }

    // The call site's whole viscosity step in one C-ABI call (FLIP_vdb.cpp:3178-3219): the rhs and the warm
    // start built on the device from the velocity, uploaded once, then PCG; returns the solved velocity
    // float[3][leaf][512] over dofTopology().  Bit-identical to warm_start + pcg_solve.
    // An empty vector on failure (*status, when given, receives the code).
    static std::vector<float> solve_velocity(L_with_level& level0, const PackedLeafGrid3& velocity,
                                             const LeafGrid& solidVelocity, float tolerance, int* iterations = nullptr,
                                             int maxIterations = 100, int* status = nullptr) {
        std::vector<float> x = level0.get_zero_vec();
        uaamg_leaf_grid u = velocity.v[0].view(), v = velocity.v[1].view(), w = velocity.v[2].view();
        uaamg_leaf_grid s = solidVelocity.view();
        int rc = report(uaamg_viscosity_set_max_iterations(level0.handle(), maxIterations), "set_max_iterations");
        int it = 0;
        if (rc == 0)
            rc = report(uaamg_viscosity_solve_velocity(level0.handle(), &u, &v, &w, &s, tolerance, x.data(), &it),
                        "viscosity solve_velocity");
        set_status(status, rc < 0 ? rc : 0);
        if (iterations) *iterations = it;
        if (rc < 0) x.clear();
        return x;
    }

    L_with_level::Ptr m_level0;  // m_matrix_levels[0]
    std::vector<float> m_rhs;
    int m_status = 0;  // 0, or the code of a failed construction
    int m_iteration = 0;
    int m_max_iter = 100;
    int64_t m_ndof = 0;
};

// ---------------------------------------------------------------------------
// The steps around the pressure solve of a FLIP substep.

// calculate_face_weights (FLIP_vdb.cpp:2669-2752) on the given topology
// (origins [n][3], masks [n][8] or empty = all active): float[n][512][3];
// an empty vector on failure.
inline std::vector<float> calculate_face_weights(const LeafGrid& solidSdf, const std::vector<int32_t>& origins,
                                                 const std::vector<uint64_t>& masks, int* status = nullptr) {
    const int64_t n = (int64_t)(origins.size() / 3);
    std::vector<float> w((size_t)n * 512 * 3);
    uaamg_leaf_grid s = solidSdf.view();
    int rc = report(uaamg_face_weights(&s, n, n ? origins.data() : nullptr, masks.empty() ? nullptr : masks.data(),
                                       n ? w.data() : nullptr),
                    "face_weights");
    set_status(status, rc);
    if (rc < 0) w.clear();
    return w;
}

// immerse_liquid_phi_in_solids (FLIP_vdb.cpp:2856-2942), its value passes on
// the liquid SDF's own leaves: float[n][512].  The two topology dilations of
// the reference (:2881, :2941) are the caller's.
inline std::vector<float> immerse_liquid_phi_values(const LeafGrid& solidSdf, const LeafGrid& liquidPhi, float dx,
                                                    int* status = nullptr) {
    std::vector<float> out((size_t)liquidPhi.leafCount() * 512);
    uaamg_leaf_grid s = solidSdf.view(), l = liquidPhi.view();
    int rc = report(uaamg_immerse_liquid_phi(&s, &l, dx, out.empty() ? nullptr : out.data()), "immerse_liquid_phi");
    set_status(status, rc);
    if (rc < 0) out.clear();
    return out;
}

// apply_pressure_gradient (FLIP_vdb.cpp:2571-2667) for one velocity channel
// with the pressure solved on `level0`; outputs over the channel's leaves.
struct PressureGradientResult {
    std::vector<float> velocity, update, reflected;  // [n][512]
    std::vector<uint64_t> masks;                      // [n][8]: voxels with an update
    int status = 0;                                   // 0, or the negative code of a failed call
};
inline PressureGradientResult apply_pressure_gradient(LaplacianWithLevel& level0, const LeafGrid& liquidPhi,
                                                      const LeafGrid& faceWeights, const LeafGrid& solidVelocity,
                                                      const std::vector<float>& pressure, float dt, int channel,
                                                      const LeafGrid& velocity, float friction = 0.f) {
    const size_t n = (size_t)velocity.leafCount();
    PressureGradientResult r;
    r.velocity.resize(n * 512);
    r.update.resize(n * 512);
    r.reflected.resize(n * 512);
    r.masks.resize(n * 8);
    uaamg_leaf_grid a = liquidPhi.view(), b = faceWeights.view(), c = solidVelocity.view(), v = velocity.view();
    r.status = report(uaamg_poisson_apply_pressure_gradient(level0.handle(), &a, &b, &c, pressure.data(), dt, friction,
                                                            channel, &v, r.velocity.data(), r.masks.data(),
                                                            r.update.data(), r.reflected.data()),
                      "apply_pressure_gradient");
    return r;
}

// union_extrapolate's layers (vdb_velocity_extrapolator.cpp:611-659) for one
// channel, after the caller's topology steps: values [n_out][512] and masks
// [n_out][8] of the channel's leaves extended by the touched ones, updated in
// place; fill_leaf / fill_masks: per leaf with voxels to fill, its index and
// those voxels.  Returns 0 or a negative UAAMG_ERR_* code.
inline int extrapolate_channel(int nLayer, const std::vector<int32_t>& outOrigins, std::vector<float>& values,
                               std::vector<uint64_t>& masks, const std::vector<int32_t>& fillLeaf,
                               const std::vector<uint64_t>& fillMasks) {
    const int64_t nOut = (int64_t)(outOrigins.size() / 3), nFill = (int64_t)fillLeaf.size();
    return report(uaamg_extrapolate_channel(nLayer, nOut, nOut ? outOrigins.data() : nullptr,
                                            nOut ? values.data() : nullptr, nOut ? masks.data() : nullptr, nFill,
                                            nFill ? fillLeaf.data() : nullptr, nFill ? fillMasks.data() : nullptr),
                  "extrapolate_channel");
}

}  // namespace simd_uaamg_b200
