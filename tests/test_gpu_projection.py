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
from uaamg_b200.grids import LeafGrid, dense_to_leaves, pack_masks, unpack_masks

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


@pytest.fixture(scope="module")
def immersion_case(gpu):
    """The walled box with a sphere obstacle around the liquid of the plain
    scene, and a copy of the solid without its leaves at x >= n/2 (the pass
    gate: no solid leaf, no change, although samples there read the solid's
    negative background)."""
    sc = scenes.plain_poisson_scene(n=48, seed=3)
    solid = solid_box_with_obstacle(sc.n, sc.dx)
    keep = solid.origins[:, 0] < sc.n // 2
    half = LeafGrid(origins=solid.origins[keep], values=solid.values[keep], background=solid.background,
                    masks=solid.masks[keep])
    # isolated liquid voxels (1 %) in the air: negative values with no negative face neighbour
    v = sc.phi.values.copy()
    drop = (np.random.default_rng(12).random(v.shape) < 0.01) & (v > sc.dx)
    v[drop] = -0.25 * sc.dx
    # a narrow band, as a level set's active voxels: inactive voxels next to the band are visited after the
    # 26-neighbour dilation
    sc.phi = LeafGrid(origins=sc.phi.origins, values=v, background=sc.phi.background,
                      masks=pack_masks(np.abs(v) < 4 * sc.dx))
    return sc, solid, half


@pytest.mark.parametrize("which", ["full", "half"])
def test_immersion_bit_exact(immersion_case, which):
    from uaamg_b200.projection import immerse_liquid_phi_values
    sc, solid, half = immersion_case
    s = solid if which == "full" else half
    g = immerse_liquid_phi_values(sc.phi, s, sc.dx)
    o = orc.immerse_liquid_phi(sc.phi, s, sc.dx)
    assert np.array_equal(g, o)
    before = sc.phi.values
    changed = g != before
    assert changed.any()
    # every branch of the second pass is taken somewhere: a value moved to a negative neighbour's, a value
    # clamped to max(background, -solid), and pass 1's shift kept
    assert np.any(changed & (g < 0) & (before >= 0))
    assert np.any(changed & (g > 0) & (before < 0))
    assert np.any(changed & ~unpack_masks(sc.phi.masks))  # reached through the 26-neighbour dilation
    if which == "half":
        right = sc.phi.origins[:, 0] >= sc.n // 2
        assert np.array_equal(g[right], before[right])


def test_immersion_topology_and_device_path(immersion_case, gpu):
    import ctypes as C
    from uaamg_b200 import _lib
    from uaamg_b200.poisson import _as_c
    from uaamg_b200.projection import immerse_liquid_phi_in_solids, immerse_liquid_phi_values
    from uaamg_b200.topology import dilate, topology_coords
    torch = gpu
    sc, solid, half = immersion_case
    out = immerse_liquid_phi_in_solids(sc.phi, solid, sc.dx)
    n = sc.phi.leaf_count
    host = immerse_liquid_phi_values(sc.phi, solid, sc.dx)
    assert np.array_equal(out.values[:n], host)
    assert np.all(out.values[n:] == sc.phi.background[0])
    want = {tuple(p) for p in topology_coords(dilate(dilate(sc.phi, 1, 26), 1, 6)).tolist()}
    assert {tuple(p) for p in topology_coords(out).tolist()} == want
    # device form, in place over the liquid's device values
    keep = []
    d = LeafGrid(origins=sc.phi.origins, values=sc.phi.values, background=sc.phi.background, masks=sc.phi.masks)
    d.values = torch.from_numpy(sc.phi.values.copy()).cuda()
    gs, gl = _as_c(solid, keep), _as_c(d, keep)
    torch.cuda.synchronize()
    rc = _lib.lib().uaamg_immerse_liquid_phi_device(C.byref(gs), C.byref(gl), float(sc.dx), d.values.data_ptr(), None)
    _lib.check(rc, "immerse_liquid_phi_device")
    torch.cuda.synchronize()
    assert np.array_equal(d.values.cpu().numpy(), host)
