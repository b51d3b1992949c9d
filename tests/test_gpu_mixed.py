"""GPU tests of the mixed-precision pressure solve.

The preconditioner's hierarchy is stored in FP16 or BF16 (FP32 arithmetic),
the outer CG is FP32 with FP64 dots, the true residual is recomputed every
25 iterations, and the coarsest level is solved directly in FP64.  A 16-bit
preconditioner is a different (weaker) preconditioner than the FP32 one, so
the checks are on the solution, not the bits: the mixed solve must converge
to the same relative-residual target, its error against an exact FP64 sparse
solve must stay within a small factor of the FP32 solve's error, and its
iteration count within a few of the FP32 count.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle.oracle import OraclePoisson
from uaamg_b200 import scenes

pytestmark = pytest.mark.gpu

ERR_FACTOR = 10.0   # mixed error <= 10 x the FP32 solver's error (+ 1e-6 absolute)
EXTRA_ITERS = 4     # mixed iterations <= FP32 iterations + 4


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    from uaamg_b200 import build
    build.build()
    return torch


def _setup(sc):
    from uaamg_b200.poisson import LaplacianWithLevel, PoissonSolver
    lap = LaplacianWithLevel.createPressurePoissonLaplacian(sc.phi, sc.face_weights, sc.dt, sc.dx)
    rhs = lap.createPressurePoissonRightHandSide(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity, sc.dt)
    return lap, PoissonSolver(lap), rhs


def _exact(sc):
    o = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
    r, c, v = o.triplets(0)
    n = o.ndof(0)
    A = sp.csr_matrix((v.astype(np.float64), (r, c)), shape=(n, n))
    idx = o.dof_index(0)
    m = idx >= 0
    return A, idx, m


def _vec(idx, m, leafdense, n):
    out = np.zeros(n)
    out[idx[m]] = leafdense[m]
    return out


@pytest.fixture(scope="module")
def scene48(gpu):
    sc = scenes.plain_poisson_scene(n=48, seed=0)
    A, idx, m = _exact(sc)
    return sc, A, idx, m


@pytest.mark.parametrize("precision", ["fp16", "bf16"])
def test_mixed_solution_against_fp64_exact(scene48, precision):
    sc, A, idx, m = scene48
    lap, s, rhs = _setup(sc)
    n = A.shape[0]
    b = _vec(idx, m, rhs, n)
    x64 = spla.spsolve(A.tocsc(), b)
    p32 = lap.getZeroVectorGrid()
    assert s.solveMultigridPCG(p32, rhs) == 0
    it32 = s.mIterationTaken
    pm = lap.getZeroVectorGrid()
    assert s.solveMultigridPCGMixed(pm, rhs, precision) == 0
    itm = s.mIterationTaken
    e32 = np.linalg.norm(_vec(idx, m, p32, n) - x64) / np.linalg.norm(x64)
    em = np.linalg.norm(_vec(idx, m, pm, n) - x64) / np.linalg.norm(x64)
    assert em <= ERR_FACTOR * e32 + 1e-6, (precision, em, e32)
    assert itm <= it32 + EXTRA_ITERS, (itm, it32)
    res = np.abs(b - A @ _vec(idx, m, pm, n)).max() / np.abs(b).max()
    assert res <= 1e-5, res
    assert not pm[~m].any()  # zero off the DOF


def test_fp64_true_residual_matches_scipy(scene48, gpu):
    torch = gpu
    sc, A, idx, m = scene48
    lap, s, rhs = _setup(sc)
    p = lap.getZeroVectorGrid()
    s.solveMultigridPCGMixed(p, rhs, "bf16")
    n = A.shape[0]
    rmax, bmax = s.true_residual_fp64(torch.from_numpy(p).cuda(), torch.from_numpy(rhs).cuda())
    b = _vec(idx, m, rhs, n)
    ref_r = np.abs(b - A @ _vec(idx, m, p, n)).max()
    assert bmax == pytest.approx(np.abs(b).max(), rel=1e-12)
    assert rmax == pytest.approx(ref_r, rel=1e-6, abs=1e-12 * bmax)


def test_residual_replacement_and_device_path(scene48, gpu):
    torch = gpu
    sc, A, idx, m = scene48
    lap, s, rhs = _setup(sc)
    s.mRelativeTolerance = 1e-9  # enough iterations for replacements to happen
    base = lap.getZeroVectorGrid()
    assert s.solveMultigridPCGMixed(base, rhs, "fp16") in (0, 1)
    s.set_residual_replacement(2)
    rep = lap.getZeroVectorGrid()
    s.solveMultigridPCGMixed(rep, rhs, "fp16")
    rel = np.linalg.norm(rep - base) / np.linalg.norm(base)
    assert rel <= 1e-4, rel
    s.set_residual_replacement(25)
    d_p = torch.zeros(rhs.shape, dtype=torch.float32, device="cuda")
    d_r = torch.from_numpy(rhs).cuda()
    host = lap.getZeroVectorGrid()
    s.solveMultigridPCGMixed(host, rhs, "fp16")
    s.solveMultigridPCGMixed(d_p, d_r, "fp16")
    assert np.array_equal(d_p.cpu().numpy(), host)  # deterministic: same bits on both paths


def test_one_level_hierarchy_and_precision_switch(gpu):
    sc = scenes.sdf_box_scene(12, None, [((0.5, 0.5, 0.5), 0.3)], 11)
    lap, s, rhs = _setup(sc)
    assert lap.num_levels() == 1
    A, idx, m = _exact(sc)
    x64 = spla.spsolve(A.tocsc(), _vec(idx, m, rhs, A.shape[0]))
    for prec in ("fp16", "bf16", "fp16"):
        p = lap.getZeroVectorGrid()
        assert s.solveMultigridPCGMixed(p, rhs, prec) == 0
        e = np.linalg.norm(_vec(idx, m, p, A.shape[0]) - x64) / np.linalg.norm(x64)
        assert e <= 1e-3, (prec, e)


@pytest.mark.parametrize("smoother", ["scheduled", "weighted"])
def test_fp64_reference_solve_matches_sparse_direct(scene48, gpu, smoother):
    """The FP64 reference solve (flexible FP64 PCG to a true 2-norm relative
    residual of 1e-12) against scipy's FP64 sparse direct solve of the same
    assembled matrix: relative 2-norm error <= 1e-10, the residual it reports
    is the true one, and it needs far fewer iterations than an
    unpreconditioned CG would."""
    torch = gpu
    from uaamg_b200.poisson import PoissonSolver
    sc, A, idx, m = scene48
    lap, _, rhs = _setup(sc)
    n = A.shape[0]
    xs = spla.spsolve(A.tocsc(), _vec(idx, m, rhs, n))
    s = PoissonSolver(lap)
    s.mSmoother = (PoissonSolver.SmootherOption.ScheduledRelaxedJacobi if smoother == "scheduled"
                   else PoissonSolver.SmootherOption.WeightedJacobi)
    d_b = torch.from_numpy(rhs).cuda()
    d_x = torch.full(rhs.shape, 7.0, dtype=torch.float64, device="cuda")
    st, it, rel = s.solve_fp64_reference(d_b, d_x, 1e-12, 200)
    assert st == 0 and 0 < it <= 40
    x = d_x.cpu().numpy()
    xv = np.zeros(n)
    xv[idx[m]] = x[m]
    assert np.all(x[~m] == 0.0)
    bv = _vec(idx, m, rhs, n).astype(np.float64)
    true_rel = np.linalg.norm(bv - A @ xv) / np.linalg.norm(bv)
    assert true_rel <= 1e-12 and abs(true_rel - rel) <= 1e-3 * rel + 1e-16
    assert np.linalg.norm(xv - xs) <= 1e-10 * np.linalg.norm(xs)
