"""CPU checks of the oracle (the restatement of SIMD_UAAMG/simd_vdb_poisson.cpp).

The reference itself cannot run here, so the oracle is checked against
  * an independent numpy restatement of BuildFinestMatrix (cpp:474-597),
  * the explicit-matrix formulation of the coarsening used by the reference's
    own benchmark harness, A_c = 1/2 R A P with R = P^T / 8
    (CG_benchmarks/main.cpp:1070-1074),
  * the assembled FP64 matrix for the apply modes and the converged solution,
  * published SplitMix64 test vectors for the input generator,
  * and its own golden fixture (tests/golden/make_golden.py).
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle.oracle import OraclePoisson
from uaamg_b200 import scenes
from uaamg_b200.grids import LeafGrid, dense_to_leaves, unpack_masks, vdb_leaf_order


def small_scene(n=24, seed=5):
    return scenes.sdf_box_scene(n, 0.4, [((0.5, 0.7, 0.5), 0.15)], seed=seed, dt=1.0)


def dense_from_leaves(org, vals, n):
    out = np.zeros((n + 16, n + 16, n + 16), np.float32)
    off = np.arange(512)
    x, y, z = off >> 6, (off >> 3) & 7, off & 7
    for i in range(org.shape[0]):
        out[org[i, 0] + x, org[i, 1] + y, org[i, 2] + z] = vals[i]
    return out[:n, :n, :n]


def matrix(o, level):
    r, c, v = o.triplets(level)
    n = o.ndof(level)
    return sp.csr_matrix((v.astype(np.float64), (r, c)), shape=(n, n))


def to_vec(o, level, leafdense):
    idx = o.dof_index(level)
    out = np.zeros(o.ndof(level))
    m = idx >= 0
    out[idx[m]] = leafdense[m]
    return out


# ---------------------------------------------------------------------------
def test_splitmix64_published_vectors():
    # SplitMix64 with state 0: first outputs 0xe220a8397b1dcdaf, 0x6e789e6aa1b965f4
    z = scenes.splitmix64(0, 2)
    assert int(z[0]) == 0xE220A8397B1DCDAF
    assert int(z[1]) == 0x6E789E6AA1B965F4
    u = scenes.uniform(0, 1000, -1.0, 1.0)
    assert u.min() >= -1.0 and u.max() < 1.0


def test_vdb_leaf_order_groups_internal_nodes():
    o = np.array([[128, 0, 0], [0, 0, 8], [0, 120, 0], [0, 0, 0], [-8, 0, 0], [4096, 0, 0]], np.int32)
    order = vdb_leaf_order(o)
    # root tile of -8 sorts first; inside tile 0 the 128^3 internal node of (0,*,*)
    # precedes (128,0,0); inside it the 8^3 leaves follow their 16^3 offsets
    assert o[order].tolist() == [[-8, 0, 0], [0, 0, 0], [0, 0, 8], [0, 120, 0], [128, 0, 0], [4096, 0, 0]]


def _finest_numpy(phi, w, dt, dx):
    """Independent restatement of BuildFinestMatrix on dense arrays (float32,
    same operation order).  phi: [n,n,n]; w: [n+1,n+1,n+1,3]; outside = air."""
    n = phi.shape[0]
    t = np.float32(dt) / (np.float32(dx) * np.float32(dx))
    bg = np.float32(1e3)
    P = np.full((n + 2, n + 2, n + 2), bg, np.float32)
    P[1:-1, 1:-1, 1:-1] = phi
    diag = np.zeros((n, n, n), np.float32)
    neg = [np.zeros((n, n, n), np.float32) for _ in range(3)]
    c = P[1:-1, 1:-1, 1:-1]
    for f in range(6):
        comp, pos = f // 2, f % 2 == 0
        sl = [slice(1, -1)] * 3
        sl[comp] = slice(2, None) if pos else slice(0, -2)
        other = P[tuple(sl)]
        wsl = [slice(0, n)] * 3
        if pos:
            wsl[comp] = slice(1, n + 1)
        weight = w[tuple(wsl) + (comp,)]
        term = (weight * t).astype(np.float32)
        liquid = other < 0
        with np.errstate(divide="ignore", invalid="ignore"):
            theta = np.where((c < 0) & (other >= 0), c / (c - other), np.float32(1)).astype(np.float32)
        theta = np.maximum(theta, np.float32(0.02))
        add = np.where(liquid, term, (term / theta).astype(np.float32)).astype(np.float32)
        diag = (diag + add).astype(np.float32)
        if not pos:
            neg[comp] = np.where(liquid, -term, np.float32(0)).astype(np.float32)
    dof = (c < 0) & (diag != 0)
    return diag, neg, dof


def test_finest_matrix_matches_numpy_restatement():
    n = 24
    sc = small_scene(n)
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx, hierarchy=False)
    # dense inputs
    phi = dense_from_leaves(sc.phi.origins, sc.phi.values, n)
    wd = np.ones((n + 1, n + 1, n + 1, 3), np.float32)
    wd[0, :, :, 0] = wd[n, :, :, 0] = 0
    wd[:, 0, :, 1] = wd[:, n, :, 1] = 0
    wd[:, :, 0, 2] = wd[:, :, n, 2] = 0
    diag, neg, dof = _finest_numpy(phi, wd, sc.dt, sc.dx)
    (d, cx, cy, cz), flags = o.coefficients(0)
    org, masks = o.topology(0)
    act = unpack_masks(masks)
    assert act.sum() == dof.sum() == o.ndof(0)
    dd = dense_from_leaves(org, np.where(act, d, 0), n)
    assert np.array_equal(dense_from_leaves(org, act.astype(np.float32), n) > 0, dof)
    untrimmed = np.repeat((flags & 1) == 0, 512).reshape(-1, 512)
    exact = dense_from_leaves(org, np.where(act & untrimmed, 1, 0), n) > 0
    assert np.array_equal(dd[exact], diag[exact])
    # trimmed leaves hold the default within the 1e-5 trim tolerance
    assert np.allclose(dd[dof], diag[dof], rtol=2e-5)
    for k, arr in enumerate((cx, cy, cz)):
        a = dense_from_leaves(org, np.where(act, arr, 0), n)
        assert np.allclose(a[dof], neg[k][dof], rtol=2e-5, atol=1e-3)


def test_galerkin_coarsening_is_half_rap():
    sc = small_scene(40, seed=2)
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    assert o.num_levels >= 2
    for l in range(o.num_levels - 1):
        Af = matrix(o, l)
        Ac = matrix(o, l + 1)
        fi = o.dof_index(l)
        ci = o.dof_index(l + 1)
        forg, _ = o.topology(l)
        corg, _ = o.topology(l + 1)
        # coarse DOF of every fine DOF: coarse voxel floor(g / 2)
        cmap = {}
        off = np.arange(512)
        lx, ly, lz = off >> 6, (off >> 3) & 7, off & 7
        for i in range(corg.shape[0]):
            for k in np.nonzero(ci[i] >= 0)[0]:
                cmap[(corg[i, 0] + lx[k], corg[i, 1] + ly[k], corg[i, 2] + lz[k])] = ci[i, k]
        rows, cols = [], []
        for i in range(forg.shape[0]):
            for k in np.nonzero(fi[i] >= 0)[0]:
                g = (forg[i, 0] + lx[k], forg[i, 1] + ly[k], forg[i, 2] + lz[k])
                rows.append(fi[i, k])
                cols.append(cmap[(g[0] // 2, g[1] // 2, g[2] // 2)])
        P = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(o.ndof(l), o.ndof(l + 1)))
        rap = (0.5 / 8.0) * (P.T @ Af @ P)
        diff = abs(rap - Ac).max()
        assert diff <= 3e-5 * abs(Ac).max(), (l, diff)


@pytest.mark.parametrize("mode", ["laplacian", "residual", "jacobi", "spai0"])
def test_apply_modes_match_assembled_matrix(mode):
    sc = small_scene(32, seed=1)
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    rng = np.random.default_rng(0)
    for l in range(o.num_levels):
        act = o.dof_index(l) >= 0
        x = (rng.standard_normal(act.shape) * act).astype(np.float32)
        b = (rng.standard_normal(act.shape) * act).astype(np.float32)
        A = matrix(o, l)
        xv, bv = to_vec(o, l, x), to_vec(o, l, b)
        out = to_vec(o, l, o.apply(l, mode, x, b, weight=0.75))
        Ax = A @ xv
        if mode == "laplacian":
            ref = Ax
        elif mode == "residual":
            ref = bv - Ax
        elif mode == "jacobi":
            ref = xv + 0.75 * (bv - Ax) / A.diagonal()
        else:
            rn = np.asarray(A.multiply(A).sum(axis=1)).ravel()
            ref = xv + (A.diagonal() / rn) * (bv - Ax)
        scale = np.abs(A).max() * (np.abs(xv).max() + np.abs(bv).max())
        assert np.abs(out - ref).max() <= 1e-5 * scale, (mode, l)
        # non-DOF voxels hold zero
        assert np.all(o.apply(l, mode, x, b)[~act] == 0)


def test_red_black_passes_touch_one_colour():
    sc = small_scene(24)
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    act = o.dof_index(0) >= 0
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(act.shape) * act).astype(np.float32)
    b = (rng.standard_normal(act.shape) * act).astype(np.float32)
    off = np.arange(512)
    red = (((off >> 6) + ((off >> 3) & 7) + (off & 7)) & 1) == 0
    r = o.apply(0, "red_gs", x, b)
    k = o.apply(0, "black_gs", x, b)
    assert np.array_equal(r[:, ~red], x[:, ~red])
    assert np.array_equal(k[:, red], x[:, red])
    assert not np.array_equal(r[:, red], x[:, red])


def test_restriction_prolongation_are_adjoint():
    sc = small_scene(40)
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    rng = np.random.default_rng(3)
    fa = o.dof_index(0) >= 0
    ca = o.dof_index(1) >= 0
    f = (rng.standard_normal(fa.shape) * fa).astype(np.float32)
    c = (rng.standard_normal(ca.shape) * ca).astype(np.float32)
    Rf = o.restrict(0, f)
    Pc = o.prolongate(0, c, np.zeros_like(f))
    lhs = 8.0 * np.dot(Rf.ravel().astype(np.float64), c.ravel())
    rhs = np.dot(f.ravel().astype(np.float64), Pc.ravel())
    assert abs(lhs - rhs) <= 1e-5 * (abs(lhs) + 1)


@pytest.mark.parametrize("smoother", ["scheduled_jacobi", "weighted_jacobi", "rbgs", "spai0"])
def test_pcg_solution_against_fp64(smoother):
    sc = small_scene(32, seed=4)
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    rhs = o.build_rhs(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity)
    x, st, it, nu = o.solve_pcg(o.zeros(), rhs, tol=1e-7, smoother=smoother)
    assert st == 0 and 1 <= it < 30
    A = matrix(o, 0)
    b = to_vec(o, 0, rhs)
    x64 = spla.spsolve(A.tocsc(), b)
    err = np.linalg.norm(to_vec(o, 0, x) - x64) / np.linalg.norm(x64)
    assert err < 1e-4, err
    res = np.abs(b - A @ to_vec(o, 0, x)).max() / np.abs(b).max()
    assert res < 1e-5


def test_pure_multigrid_reduces_residual():
    sc = small_scene(32, seed=4)
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    rhs = o.build_rhs(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity)
    x, st, it, nu = o.solve_mg(o.zeros(), rhs, tol=1e-5)
    assert st == 0
    assert nu <= 1e-5 * np.abs(rhs).max()


def test_coarsest_solve_is_ten_cg_iterations():
    sc = small_scene(40)
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    L = o.num_levels - 1
    act = o.dof_index(L) >= 0
    b = (np.random.default_rng(2).standard_normal(act.shape) * act).astype(np.float32)
    x = o.coarsest_solve(b)
    A = matrix(o, L)
    res = np.linalg.norm(to_vec(o, L, b) - A @ to_vec(o, L, x)) / np.linalg.norm(to_vec(o, L, b))
    assert res < 0.5  # 10 diagonal-PCG iterations reduce, but do not solve exactly


def test_golden_fixture():
    import os
    from tests.golden.make_golden import golden_scene
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "poisson_golden_40.npz"))
    sc = golden_scene()
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    assert o.num_levels == int(g["levels"])
    for l in range(o.num_levels):
        (d, cx, cy, cz), flags = o.coefficients(l)
        org, masks = o.topology(l)
        assert np.array_equal(org, g[f"l{l}_origins"]) and np.array_equal(masks, g[f"l{l}_masks"])
        for nm, a in (("diag", d), ("cx", cx), ("cy", cy), ("cz", cz)):
            assert np.array_equal(a, g[f"l{l}_{nm}"]), (l, nm)
        assert np.array_equal(flags, g[f"l{l}_flags"])
    rhs = o.build_rhs(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity)
    assert np.array_equal(rhs, g["rhs"])
    for sm in ("scheduled_jacobi", "weighted_jacobi", "rbgs", "spai0"):
        x, st, it, nu = o.solve_pcg(o.zeros(), rhs, smoother=sm)
        assert it == int(g[f"pcg_{sm}_iters"]) and st == int(g[f"pcg_{sm}_status"])
        assert np.array_equal(x, g[f"pcg_{sm}_x"])


# --------------------------------------------------------------------------- edge cases
def test_empty_domain():
    empty = LeafGrid(origins=np.zeros((0, 3), np.int32), values=np.zeros((0, 512), np.float32), background=1.0)
    fw = LeafGrid(origins=np.zeros((0, 3), np.int32), values=np.zeros((0, 512, 3), np.float32),
                  background=np.ones(3, np.float32))
    o = OraclePoisson(empty, fw, 1.0, 0.1)
    assert o.ndof(0) == 0 and o.num_levels == 1
    x, st, it, nu = o.solve_pcg(o.zeros(), o.zeros())
    assert st == 0 and it == 0


def test_isolated_voxel_without_open_faces_is_not_a_dof():
    n = 16
    phi = np.full((n, n, n), 1.0, np.float32)
    phi[3, 3, 3] = -0.5       # enclosed by solid faces: not a DOF
    phi[8:12, 8:12, 8:12] = -0.5
    w = np.ones((n + 1, n + 1, n + 1, 3), np.float32)
    for k in range(3):
        sl = [3, 3, 3]
        w[tuple(sl) + (k,)] = 0
        sl[k] = 4
        w[tuple(sl) + (k,)] = 0
    pg = dense_to_leaves(phi, background=1.0)
    fg = dense_to_leaves(w, background=np.ones(3, np.float32))
    o = OraclePoisson(pg, fg, 1.0, 1.0 / n)
    assert o.ndof(0) == 64


def test_translation_and_leaf_order_invariance():
    """Shifting the domain by a multiple of 8 * 2^(levels-1) voxels and
    permuting the input leaves changes nothing but the leaf origins."""
    sc = small_scene(40)
    o1 = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    sh = np.array([-128, 64, -64], np.int32)
    rng = np.random.default_rng(0)

    def moved(g):
        perm = rng.permutation(g.leaf_count)
        return LeafGrid(origins=g.origins[perm] + sh, values=g.values[perm], background=g.background,
                        masks=g.masks[perm])
    o2 = OraclePoisson(moved(sc.phi), moved(sc.face_weights), sc.dt, sc.dx)
    assert o1.num_levels == o2.num_levels
    for l in range(o1.num_levels):
        assert o1.ndof(l) == o2.ndof(l)
        (a1, f1), (a2, f2) = o1.coefficients(l), o2.coefficients(l)
        t1, t2 = o1.topology(l), o2.topology(l)
        k2 = {tuple(o): j for j, o in enumerate(t2[0])}
        for i, org in enumerate(t1[0]):
            j = k2[tuple(org + sh // (2 ** l))]
            assert np.array_equal(t1[1][i], t2[1][j]) and f1[i] == f2[j]
            for x1, x2 in zip(a1, a2):
                assert np.array_equal(x1[i], x2[j])
    rhs1 = o1.build_rhs(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity)
    r1, st1, it1, _ = o1.solve_pcg(o1.zeros(), rhs1)
    # map rhs into the shifted leaf order and solve there
    k2 = {tuple(o): j for j, o in enumerate(o2.topology(0)[0])}
    perm = np.array([k2[tuple(org + sh)] for org in o1.topology(0)[0]])
    rhs2 = np.zeros_like(rhs1)
    rhs2[perm] = rhs1
    r2, st2, it2, _ = o2.solve_pcg(o2.zeros(), rhs2)
    assert st1 == st2 == 0 and it1 == it2
    assert np.allclose(r2[perm], r1, rtol=1e-5, atol=1e-6 * np.abs(r1).max())


def test_avx2_applier_matches_scalar_path():
    """The oracle's 8-lane AVX2 applier (the reference's lane layout) gives the
    scalar per-voxel path's bits in every mode, on every level, at leaf
    boundaries and in place (red/black passes)."""
    from oracle.oracle import set_simd
    sc = scenes.plain_poisson_scene(n=48, seed=5)
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    rng = np.random.default_rng(3)
    try:
        for l in range(o.num_levels):
            act = o.dof_index(l) >= 0
            x = (rng.standard_normal(act.shape) * act).astype(np.float32)
            b = (rng.standard_normal(act.shape) * act).astype(np.float32)
            for mode in ("jacobi", "residual", "laplacian", "red_gs", "black_gs", "spai0"):
                for w, wsor in ((0.8571, 1.2), (2.2473, 1.0)):
                    set_simd(True)
                    a = o.apply(l, mode, x, b, weight=w, w_sor=wsor)
                    set_simd(False)
                    c = o.apply(l, mode, x, b, weight=w, w_sor=wsor)
                    assert np.array_equal(a, c), (l, mode)
            for first in ("jacobi", "spai0"):
                set_simd(True)
                a = o.first_jacobi(l, b, 2.2473) if first == "jacobi" else o.first_spai0(l, b)
                set_simd(False)
                c = o.first_jacobi(l, b, 2.2473) if first == "jacobi" else o.first_spai0(l, b)
                assert np.array_equal(a, c), (l, first)
        set_simd(True)
        rhs = o.build_rhs(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity)
        xa, sta, ita, _ = o.solve_pcg(o.zeros(), rhs, tol=1e-7)
        set_simd(False)
        xb, stb, itb, _ = o.solve_pcg(o.zeros(), rhs, tol=1e-7)
        assert sta == stb and ita == itb and np.array_equal(xa, xb)
    finally:
        set_simd(True)
