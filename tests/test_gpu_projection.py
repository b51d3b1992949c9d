"""GPU parity of the steps either side of the pressure solve against the
oracle (projection_oracle.c): the solid face weights on the liquid's dilated
topology, and the pressure-gradient update of every velocity channel with the
GPU's pressure solution, with and without boundary friction.  Both are
per-voxel float work in the reference's operation order: bit-exact."""
import numpy as np
import pytest

from oracle import oracle as orc
from oracle.oracle import OraclePoisson
from uaamg_b200 import scenes
from uaamg_b200.grids import LeafGrid, dense_to_leaves, unpack_masks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    from uaamg_b200 import build
    build.build()
    return torch


def solid_box_with_obstacle(n: int, dx: float) -> LeafGrid:
    """Solid SDF over [-8, n+8)^3: walls 1.5 voxels thick and a sphere of radius
    n/8 at (n/2, n/4, n/2) (negative inside the solid)."""
    lo, size = -8, n + 16
    c = np.arange(size, dtype=np.float64) + lo
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    wall = np.minimum.reduce([X - 1.5, n - 1.5 - X, Y - 1.5, n - 1.5 - Y, Z - 1.5, n - 1.5 - Z])
    sph = np.sqrt((X - n / 2) ** 2 + (Y - n / 4) ** 2 + (Z - n / 2) ** 2) - n / 8
    return dense_to_leaves((np.minimum(wall, sph) * dx).astype(np.float32), origin=(lo, lo, lo),
                           background=-3.0 * dx)


@pytest.fixture(scope="module")
def setup(gpu):
    from uaamg_b200.poisson import LaplacianWithLevel, PoissonSolver
    from uaamg_b200.projection import calculate_face_weights, face_weight_topology
    sc = scenes.plain_poisson_scene(n=48, seed=3)
    solid = solid_box_with_obstacle(sc.n, sc.dx)
    origins, masks = face_weight_topology(sc.phi)
    w = calculate_face_weights(solid, origins, masks)
    fw = LeafGrid(origins=origins, values=w, background=np.ones(3, np.float32), masks=masks)
    lap = LaplacianWithLevel.createPressurePoissonLaplacian(sc.phi, fw, sc.dt, sc.dx)
    ref = OraclePoisson(sc.phi, fw, sc.dt, sc.dx, hierarchy=False)
    rhs = lap.createPressurePoissonRightHandSide(fw, sc.vx, sc.vy, sc.vz, sc.solid_velocity, sc.dt)
    p = lap.getZeroVectorGrid()
    assert PoissonSolver(lap).solveMultigridPCG(p, rhs) == 0
    m = sc.n + 1
    sv = dense_to_leaves(np.random.default_rng(11).uniform(-1, 1, (m, m, m, 3)).astype(np.float32),
                         background=np.zeros(3, np.float32))
    return sc, solid, origins, masks, w, fw, lap, ref, p, sv


def test_face_weights_bit_exact(setup):
    sc, solid, origins, masks, w, fw, lap, ref, p, sv = setup
    wo = orc.face_weights(solid, origins, masks)
    assert np.array_equal(w, wo)
    act = unpack_masks(masks)
    frac = w[act]
    assert np.any((frac > 0) & (frac < 1)) and np.any(frac == 0) and np.any(frac == 1)
    assert np.all(w[~act] == 1.0)


@pytest.mark.parametrize("friction", [0.0, 0.5])
def test_pressure_gradient_bit_exact(setup, friction):
    from uaamg_b200.projection import apply_pressure_gradient
    sc, solid, origins, masks, w, fw, lap, ref, p, sv = setup
    p_org, p_masks = ref.topology(0)
    assert np.array_equal(lap.dof_index(0) >= 0, ref.dof_index(0) >= 0)
    partial = 0
    for c, vel in enumerate((sc.vx, sc.vy, sc.vz)):
        g = apply_pressure_gradient(lap, sc.phi, fw, sv, p, sc.dt, c, vel, friction=friction)
        o = orc.pressure_gradient(sc.phi, fw, sv, p_org, p_masks, p, sc.dt, sc.dx, friction, c, vel)
        for a, b, name in zip(g, o, ("velocity", "mask", "update", "reflected")):
            assert np.array_equal(a, b), (c, name)
        on = unpack_masks(g[1])
        assert on.sum() > 0 and on.sum() < unpack_masks(vel.masks).sum()
        # faces with a fractional weight and an update take the friction branch
        where = {tuple(o): i for i, o in enumerate(origins.tolist())}
        for i in np.nonzero(on.any(axis=1))[0]:
            lf = where.get(tuple(vel.origins[i].tolist()))
            if lf is not None:
                wv = w[lf, on[i], c]
                partial += int(np.count_nonzero((wv > 0) & (wv < 1)))
    assert partial > 0


def test_pressure_gradient_device_path_matches_host(setup, gpu):
    import ctypes as C
    from uaamg_b200 import _lib
    from uaamg_b200.poisson import _as_c
    from uaamg_b200.projection import apply_pressure_gradient
    torch = gpu
    sc, solid, origins, masks, w, fw, lap, ref, p, sv = setup
    vel = sc.vy
    host = apply_pressure_gradient(lap, sc.phi, fw, sv, p, sc.dt, 1, vel, friction=0.5)
    keep = []
    d_vel = torch.from_numpy(vel.values.copy()).cuda()
    d_p = torch.from_numpy(p).cuda()
    n = vel.leaf_count
    d_mask = torch.zeros(n * 8, dtype=torch.int64, device="cuda")
    d_upd = torch.zeros((n, 512), dtype=torch.float32, device="cuda")
    d_refl = torch.zeros((n, 512), dtype=torch.float32, device="cuda")
    gphi, gfw, gsv, gv = (_as_c(x, keep) for x in (sc.phi, fw, sv, vel))
    torch.cuda.synchronize()  # the buffers above are ready before the library's stream reads them
    rc = _lib.lib().uaamg_poisson_apply_pressure_gradient_device(
        lap._h, C.byref(gphi), C.byref(gfw), C.byref(gsv), d_p.data_ptr(), float(sc.dt), 0.5, 1, C.byref(gv),
        d_vel.data_ptr(), d_mask.data_ptr(), d_upd.data_ptr(), d_refl.data_ptr())
    _lib.check(rc, "apply_pressure_gradient_device")
    torch.cuda.synchronize()
    assert np.array_equal(d_vel.cpu().numpy(), host[0])
    assert np.array_equal(d_mask.cpu().numpy().view(np.uint64).reshape(n, 8), host[1])
    assert np.array_equal(d_upd.cpu().numpy(), host[2])
    assert np.array_equal(d_refl.cpu().numpy(), host[3])
