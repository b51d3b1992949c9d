"""GPU tests of the batched pressure solve (many instances in one CUDA graph).

The batch runs every instance's W-cycle and CG with the same per-leaf device
code and the same reduction order as a standalone solve, so each instance's
solution must be BIT-IDENTICAL to its own PoissonSolver.solveMultigridPCG
(alone and in the mix), with the same iteration count and status, whatever
the other instances are (sizes, depths, one-level hierarchies, empty domains,
instances that converge at once).  Against the oracle the usual solve parity
holds: iterations within +-2 and relative solution difference <= 1e-5.
"""
import numpy as np
import pytest

from oracle.oracle import OraclePoisson
from uaamg_b200 import scenes
from uaamg_b200.grids import LeafGrid

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5
ITER_TOL = 2


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    from uaamg_b200 import build
    build.build()
    return torch


def _empty_scene(n=16):
    """A box with no liquid: no DOF at all."""
    sc = scenes.sdf_box_scene(n, None, [((0.5, 0.5, 0.5), 0.2)], 3)
    sc.phi.values = np.abs(sc.phi.values) + 1.0  # positive everywhere
    return sc


def _scenes():
    out = [scenes.random_balls_scene(s, sides=(16, 24, 32, 48)) for s in range(5)]
    out.append(scenes.sdf_box_scene(12, None, [((0.5, 0.5, 0.5), 0.3)], 11))  # one-level hierarchy
    out.append(scenes.plain_poisson_scene(n=40, seed=4))
    out.append(_empty_scene())
    return out


@pytest.fixture(scope="module")
def batch_scenes(gpu):
    return _scenes()


def _make(sc, smoother):
    from uaamg_b200.poisson import LaplacianWithLevel, PoissonSolver
    lap = LaplacianWithLevel.createPressurePoissonLaplacian(sc.phi, sc.face_weights, sc.dt, sc.dx)
    rhs = lap.createPressurePoissonRightHandSide(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity, sc.dt)
    s = PoissonSolver(lap)
    s.mSmoother = PoissonSolver.SmootherOption(smoother)
    return lap, s, rhs


def _standalone(scs, smoother, max_iter=100, x0=None, zero_rhs=()):
    res = []
    for i, sc in enumerate(scs):
        lap, s, rhs = _make(sc, smoother)
        if i in zero_rhs:
            rhs = np.zeros_like(rhs)
        s.mMaxIteration = max_iter
        p = lap.getZeroVectorGrid() if x0 is None else x0[i].copy()
        st = s.solveMultigridPCG(p, rhs)
        res.append((p, st, s.mIterationTaken, lap.num_levels()))
    return res


def _batched(scs, smoother, max_iter=100, device=False, use_graph=True, x0=None, zero_rhs=()):
    from uaamg_b200.batch import PoissonBatch
    made = [_make(sc, smoother) for sc in scs]
    made = [(m[0], m[1], np.zeros_like(m[2]) if i in zero_rhs else m[2]) for i, m in enumerate(made)]
    b = PoissonBatch([m[1] for m in made])
    b.mSmoother = made[0][1].mSmoother
    b.mMaxIteration = max_iter
    b.use_graph = use_graph
    ps = [m[0].getZeroVectorGrid() if x0 is None else x0[i].copy() for i, m in enumerate(made)]
    rhss = [m[2] for m in made]
    if device:
        import torch
        dps = [torch.from_numpy(p).cuda() for p in ps]
        drs = [torch.from_numpy(r).cuda() for r in rhss]
        rc = b.solveMultigridPCG(dps, drs)
        ps = [d.cpu().numpy() for d in dps]
    else:
        rc = b.solveMultigridPCG(ps, rhss)
    return rc, ps, b, made


@pytest.mark.parametrize("smoother", [0, 1, 2, 3])
def test_batch_bit_identical_to_standalone(batch_scenes, smoother):
    alone = _standalone(batch_scenes, smoother)
    assert {a[3] for a in alone} >= {1, 2}, "the mix should hold hierarchies of different depths"
    rc, ps, b, _ = _batched(batch_scenes, smoother)
    for i, (p, st, it, _) in enumerate(alone):
        assert np.array_equal(ps[i], p), (smoother, i)
        assert b.mIterationTaken[i] == it, (smoother, i, b.mIterationTaken[i], it)
        assert b.status[i] == st, (smoother, i)
    assert rc == (0 if all(a[1] == 0 for a in alone) else 1)


def test_batch_device_and_host_paths_and_graph_modes_agree(batch_scenes):
    _, p_host, b1, _ = _batched(batch_scenes, 0, use_graph=2)  # the graph from the first solve
    _, p_dev, b2, _ = _batched(batch_scenes, 0, device=True)
    _, p_eager, b3, _ = _batched(batch_scenes, 0, use_graph=False)
    for a, c, e in zip(p_host, p_dev, p_eager):
        assert np.array_equal(a, c) and np.array_equal(a, e)
    assert b1.mIterationTaken == b2.mIterationTaken == b3.mIterationTaken
    assert b1.kernel_launches > 0 and b3.kernel_launches > 0


def test_batch_against_oracle(batch_scenes):
    rc, ps, b, made = _batched(batch_scenes, 0)
    for i, sc in enumerate(batch_scenes):
        ref = OraclePoisson(sc.phi, sc.face_weights, sc.dt, sc.dx)
        if ref.ndof(0) == 0:
            assert ps[i].size == 0 and b.status[i] == 0 and b.mIterationTaken[i] == 0
            continue
        rhs = ref.build_rhs(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity)
        assert np.array_equal(rhs, made[i][2])
        x, st, it, _ = ref.solve_pcg(ref.zeros(), rhs)
        assert st == 0 and b.status[i] == 0
        assert abs(b.mIterationTaken[i] - it) <= ITER_TOL, (i, b.mIterationTaken[i], it)
        rel = np.linalg.norm(ps[i] - x) / max(np.linalg.norm(x), 1e-30)
        assert rel <= REL_TOL, (i, rel)


def test_batch_iteration_cap_and_converged_instances(batch_scenes):
    scs = batch_scenes[:4]
    alone = _standalone(scs, 0, max_iter=2)
    rc, ps, b, _ = _batched(scs, 0, max_iter=2)
    assert rc == 1
    for i, (p, st, it, _) in enumerate(alone):
        assert st == 1 and b.status[i] == 1 and b.mIterationTaken[i] == it == 2
        assert np.array_equal(ps[i], p)
    # an instance with a zero residual converges before the first iteration
    # while the others iterate; a warm-started instance stops early
    sol = [a[0] for a in _standalone(scs, 0)]
    x0 = [np.zeros_like(s) for s in sol]
    x0[2] = (sol[2] * 0.999).astype(np.float32)
    alone = _standalone(scs, 0, x0=x0, zero_rhs=(1,))
    rc, ps, b, _ = _batched(scs, 0, x0=x0, zero_rhs=(1,))
    for i, (p, st, it, _) in enumerate(alone):
        assert np.array_equal(ps[i], p) and b.mIterationTaken[i] == it and b.status[i] == st
    assert b.mIterationTaken[1] == 0 and b.status[1] == 0 and not ps[1].any()


def test_batch_results_same_alone_and_in_mix(batch_scenes):
    """Serving-style property: an instance's result does not depend on the mix."""
    _, solo, b1, _ = _batched([batch_scenes[2]], 0)
    _, mix, b2, _ = _batched(batch_scenes, 0)
    assert np.array_equal(solo[0], mix[2])
    assert b1.mIterationTaken[0] == b2.mIterationTaken[2]
