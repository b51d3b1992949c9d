// uaamg_simd.hpp -- header-only C++ facade with the reference's class names
// over the C ABI in uaamg.h, so a FLIP_vdb-style call site
// (FLIP_vdb.cpp:3118-3168: createPressurePoissonLaplacian, PoissonSolver,
// mRelativeTolerance, mSmoother, createPressurePoissonRightHandSide,
// solveMultigridPCG, FAILED -> solvePureMultigrid) reads the same.
//
// Grids are flattened OpenVDB leaf lists (uaamg::LeafGrid); the result
// vectors are leaf-dense float[leaf][512] over the DOF leaves returned by
// LaplacianWithLevel::dofTopology().
#pragma once
#include <cstdint>
#include <memory>
#include <stdexcept>
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

inline void check(int rc, const char* what) {
    if (rc < 0) throw std::runtime_error(std::string(what) + ": " + uaamg_last_error());
}

// LaplacianWithLevel (SIMD_UAAMG/simd_vdb_poisson.h:13-138): here the level-0
// operator together with its device hierarchy.
class LaplacianWithLevel {
public:
    using Ptr = std::shared_ptr<LaplacianWithLevel>;

    static Ptr createPressurePoissonLaplacian(const LeafGrid& liquidPhi, const LeafGrid& faceWeights, float dt,
                                              float dx) {
        uaamg_leaf_grid a = liquidPhi.view(), b = faceWeights.view();
        uaamg_poisson* h = nullptr;
        check(uaamg_poisson_create(&a, &b, dt, dx, &h), "uaamg_poisson_create");
        return Ptr(new LaplacianWithLevel(h));
    }
    ~LaplacianWithLevel() { uaamg_poisson_destroy(mHandle); }
    LaplacianWithLevel(const LaplacianWithLevel&) = delete;
    LaplacianWithLevel& operator=(const LaplacianWithLevel&) = delete;

    std::vector<float> createPressurePoissonRightHandSide(const LeafGrid& faceWeights, const LeafGrid& vx,
                                                          const LeafGrid& vy, const LeafGrid& vz,
                                                          const LeafGrid& solidVelocity, float dt) {
        std::vector<float> rhs = getZeroVectorGrid();
        uaamg_leaf_grid w = faceWeights.view(), a = vx.view(), b = vy.view(), c = vz.view(), s = solidVelocity.view();
        check(uaamg_poisson_build_rhs(mHandle, &w, &a, &b, &c, &s, dt, rhs.data()), "build_rhs");
        return rhs;
    }
    std::vector<float> getZeroVectorGrid() const {
        return std::vector<float>((size_t)uaamg_poisson_leaf_count(mHandle, 0) * 512, 0.f);
    }
    void dofTopology(std::vector<int32_t>& origins, std::vector<uint64_t>& masks, int level = 0) const {
        int64_t n = uaamg_poisson_leaf_count(mHandle, level);
        origins.resize((size_t)n * 3);
        masks.resize((size_t)n * 8);
        check(uaamg_poisson_dof_topology(mHandle, level, origins.data(), masks.data()), "dof_topology");
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

    SuccessType solveMultigridPCG(std::vector<float>& inOutPressure, const std::vector<float>& rhs) {
        configure();
        int it = 0;
        int rc = uaamg_poisson_solve_pcg(mLevel0->handle(), inOutPressure.data(), rhs.data(), &it);
        check(rc, "solve_pcg");
        mIterationTaken = it;
        return rc;
    }
    SuccessType solvePureMultigrid(std::vector<float>& inOutPressure, const std::vector<float>& rhs) {
        configure();
        int it = 0;
        int rc = uaamg_poisson_solve_mg(mLevel0->handle(), inOutPressure.data(), rhs.data(), &it);
        check(rc, "solve_mg");
        mIterationTaken = it;
        return rc;
    }

    int mIterationTaken = 0;
    int mMaxIteration = 100;
    float mRelativeTolerance = 1e-7f;
    SmootherOption mSmoother = SmootherOption::ScheduledRelaxedJacobi;

private:
    void configure() {
        check(uaamg_poisson_set_smoother(mLevel0->handle(), (int)mSmoother), "set_smoother");
        check(uaamg_poisson_set_max_iterations(mLevel0->handle(), mMaxIteration), "set_max_iterations");
        check(uaamg_poisson_set_relative_tolerance(mLevel0->handle(), mRelativeTolerance), "set_tolerance");
    }
    LaplacianWithLevel::Ptr mLevel0;
};

}  // namespace simd_uaamg_b200
