"""The oracle's restatement of the steps either side of the pressure solve
(projection_oracle.c) on CPU: fraction_inside over a square against closed
forms, its symmetries, the face-weight topology (the liquid SDF dilated
by two voxels), and the extrapolation's union topology and layers."""
import numpy as np
import pytest

from oracle.oracle import face_weights, fraction_inside4
from uaamg_b200.grids import LeafGrid, dense_to_leaves, unpack_masks
from uaamg_b200.projection import face_weight_topology


@pytest.mark.parametrize("corners,area", [
    ((-1, -1, -1, -1), 1.0),        # all inside
    ((1, 1, 1, 1), 0.0),            # all outside
    ((-1, 1, 1, 1), 0.125),         # one corner: triangle with legs 1/2
    ((-1, -1, 1, 1), 0.5),          # bottom edge inside (bl, br)
    ((-1, 1, -1, 1), 0.5),          # left edge inside (bl, tl)
    ((-1, -1, -1, 1), 0.875),       # three corners
    ((-1, 1, 1, -1), 0.25),         # opposite corners, centre outside: two triangles
    ((-3, 1, 1, -3), 0.9375),       # opposite corners, centre inside: 1 - two triangles of legs 1/4
    ((-1, 3, 3, 3), 0.5 * 0.25 * 0.25),
])
def test_fraction_inside4_closed_forms(corners, area):
    assert fraction_inside4(*corners) == pytest.approx(area, abs=1e-7)


def test_fraction_inside4_rotations_and_linear_fields():
    rng = np.random.default_rng(5)
    for _ in range(200):
        bl, br, tl, tr = (rng.standard_normal(4)).astype(np.float32)
        a = fraction_inside4(bl, br, tl, tr)
        assert 0.0 <= a <= 1.0
        # a quarter turn of the square (bl -> br -> tr -> tl) keeps the area
        assert fraction_inside4(tl, bl, tr, br) == pytest.approx(a, abs=1e-6)
    # a linear field phi = x - s on the unit square: the inside area is s
    for s in (0.1, 0.25, 0.6, 0.9):
        assert fraction_inside4(-s, 1 - s, -s, 1 - s) == pytest.approx(s, abs=1e-6)


def test_face_weights_without_solid_are_one():
    solid = dense_to_leaves(np.full((16, 16, 16), 1.0, np.float32), background=1.0)
    org = np.array([[0, 0, 0], [8, 8, 8]], np.int32)
    w = face_weights(solid, org)
    assert np.all(w == 1.0)


def test_face_weight_topology_is_a_two_voxel_dilation():
    act = np.zeros((24, 24, 24), bool)
    act[10, 11, 12] = True
    phi = dense_to_leaves(np.ones((24, 24, 24), np.float32), background=1.0, active=act)
    org, masks = face_weight_topology(phi)
    on = unpack_masks(masks)
    pts = set()
    for i in range(org.shape[0]):
        for off in np.nonzero(on[i])[0]:
            pts.add((org[i][0] + (off >> 6), org[i][1] + ((off >> 3) & 7), org[i][2] + (off & 7)))
    expect = {(10 + a, 11 + b, 12 + c) for a in range(-2, 3) for b in range(-2, 3) for c in range(-2, 3)}
    assert pts == expect


def test_union_topology_is_a_face_dilation():
    from uaamg_b200.extrapolate import topology_coords, union_topology
    act = np.zeros((16, 16, 16), bool)
    act[5, 6, 7] = True
    g = dense_to_leaves(np.zeros((16, 16, 16), np.float32), active=act)
    pts = {tuple(p) for p in topology_coords(union_topology((g, g, g), 2)).tolist()}
    expect = {(5 + a, 6 + b, 7 + c) for a in range(-2, 3) for b in range(-2, 3) for c in range(-2, 3)
              if abs(a) + abs(b) + abs(c) <= 2}
    assert pts == expect and len(pts) == 25


def test_oracle_extrapolation_of_a_single_value():
    """One active voxel of value 3: two layers fill the face-connected diamond
    of radius 2 with 3 (every filled voxel averages filled neighbours only)."""
    from oracle.oracle import extrapolate_channel
    from uaamg_b200.extrapolate import prepare_channel, union_topology
    act = np.zeros((16, 16, 16), bool)
    act[5, 6, 7] = True
    dense = np.zeros((16, 16, 16), np.float32)
    dense[5, 6, 7] = 3.0
    g = dense_to_leaves(dense, active=act)
    u = union_topology((g,), 2)
    org, vals, masks, fl, fm = prepare_channel(g, u)
    v, m = extrapolate_channel(2, org, vals, masks, fl, fm)
    on = unpack_masks(m)
    assert on.sum() == 25
    assert np.all(v[on] == 3.0)


@pytest.mark.parametrize("n_layer", [1, 2, 3, 9])
def test_leaf_level_dilation_matches_voxel_dilation(n_layer):
    """The leaf-mask dilation (shifts within a leaf, planes from the 6
    neighbour leaves) against scipy's voxel dilation over a ragged random set
    spanning many leaves and negative coordinates (9 layers cross a whole
    leaf)."""
    from scipy.ndimage import binary_dilation, generate_binary_structure
    from uaamg_b200.extrapolate import topology_coords, union_topology
    rng = np.random.default_rng(n_layer)
    shape = (40, 33, 27)
    dense_a = rng.random(shape) < 0.004
    dense_b = np.zeros(shape, bool)
    dense_b[3:9, 20:22, 5:26] = True
    ga = dense_to_leaves(np.zeros(shape, np.float32), origin=(-16, 8, -8), active=dense_a)
    gb = dense_to_leaves(np.zeros(shape, np.float32), origin=(-16, 8, -8), active=dense_b)
    got = {tuple(p) for p in topology_coords(union_topology((ga, gb), n_layer)).tolist()}
    pad = n_layer + 1
    vol = np.pad(dense_a | dense_b, pad)
    vol = binary_dilation(vol, structure=generate_binary_structure(3, 1), iterations=n_layer)
    want = {(int(x) - pad - 16, int(y) - pad + 8, int(z) - pad - 8) for x, y, z in np.argwhere(vol)}
    assert got == want


@pytest.mark.parametrize("n_layer", [1, 2, 9])
def test_leaf_level_box_dilation_matches_voxel_dilation(n_layer):
    """The 26-neighbour dilation (z, y, x 1-D passes at leaf level) against
    scipy's voxel dilation with a full 3x3x3 structure."""
    from scipy.ndimage import binary_dilation
    from uaamg_b200.topology import dilate, topology_coords
    rng = np.random.default_rng(10 + n_layer)
    shape = (35, 41, 30)
    dense = rng.random(shape) < 0.003
    dense[30:33, 2:4, 20:29] = True
    g = dense_to_leaves(np.zeros(shape, np.float32), origin=(8, -24, -16), active=dense)
    got = {tuple(p) for p in topology_coords(dilate(g, n_layer, neighbours=26)).tolist()}
    pad = n_layer + 1
    vol = binary_dilation(np.pad(dense, pad), structure=np.ones((3, 3, 3), bool), iterations=n_layer)
    want = {(int(x) - pad + 8, int(y) - pad - 24, int(z) - pad - 16) for x, y, z in np.argwhere(vol)}
    assert got == want


def test_oracle_immersion_known_answers():
    """immerse_liquid_phi_in_solids' value passes on a hand-made case: solid
    everywhere (SDF -1), dx 0.5, liquid background 1.5; leaf 0 (with a solid
    leaf) has phi 1 except -1 at (3,3,3) and is active for x < 4; leaf 1 at
    (8,0,0) has no solid leaf and is left alone."""
    from oracle.oracle import immerse_liquid_phi
    solid = dense_to_leaves(np.full((8, 8, 8), -1.0, np.float32), background=-1.0)
    phi = np.ones((16, 8, 8), np.float32)
    phi[3, 3, 3] = -1.0
    act = np.zeros((16, 8, 8), bool)
    act[:4] = True
    act[8:] = True
    liq = dense_to_leaves(phi, background=1.5, active=act)
    assert liq.leaf_count == 2
    out = immerse_liquid_phi(liq, solid, 0.5)

    def at(x, y, z):
        return out[x >> 3, ((x & 7) << 6) | (y << 3) | z]

    assert at(3, 3, 3) == 1.5     # no negative neighbour: max(background, -solid) = max(1.5, 1)
    assert at(4, 3, 3) == -1.25   # inactive, next to an active voxel: its -x neighbour (corrected)
    assert at(2, 3, 3) == -1.25   # +x neighbour first
    assert at(3, 3, 2) == -1.25   # +z neighbour, after four positive ones
    assert at(1, 1, 1) == 0.75    # pass 1 only: 1 - dx/2
    assert at(4, 0, 0) == 1.0     # processed in pass 2, no negative neighbour, positive: unchanged
    assert at(6, 6, 6) == 1.0     # not active after the dilation
    assert np.all(out[1] == 1.0)  # no solid leaf at (8,0,0)


def test_topology_edge_cases():
    from uaamg_b200.topology import dilate, topology_coords, union
    empty = (np.zeros((0, 3), np.int32), np.zeros((0, 8), np.uint64))
    assert union([empty, empty])[0].shape == (0, 3)
    assert dilate(empty, 3, 6)[0].shape == (0, 3) and dilate(empty, 2, 26)[0].shape == (0, 3)
    org = np.array([[0, 0, 0], [8, 0, 0]], np.int32)
    masks = np.zeros((2, 8), np.uint64)
    masks[0, 3] = np.uint64(1 << 9)  # voxel (3, 1, 1)
    o, m = dilate((org, masks), 0, 6)  # no layers: the non-empty leaves as they are
    assert np.array_equal(o, org[:1]) and np.array_equal(m, masks[:1])
    with pytest.raises(ValueError):
        dilate((org, masks), 1, 18)
    assert {tuple(p) for p in topology_coords(dilate((org, masks), 1, 26)).tolist()} == {
        (3 + a, 1 + b, 1 + c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)}


def test_prepare_channel_touches_target_leaves():
    """touchLeaf semantics: every target leaf the channel lacks becomes an
    inactive leaf of background values, also one with no voxel to fill; a
    target leaf whose voxels the channel already has gets no fill entry."""
    from uaamg_b200.extrapolate import prepare_channel
    ch = LeafGrid(origins=np.array([[0, 0, 0]], np.int32), values=np.full((1, 512), 2.0, np.float32),
                  background=np.float32(-7.0), masks=np.full((1, 8), np.uint64(0xFFFFFFFFFFFFFFFF)))
    torg = np.array([[0, 0, 0], [8, 0, 0], [16, 0, 0]], np.int32)
    tmask = np.zeros((3, 8), np.uint64)
    tmask[0] = np.uint64(0xFF)        # covered by the channel
    tmask[1, 0] = np.uint64(0x3)       # two voxels to fill
    org, vals, masks, fl, fm = prepare_channel(ch, (torg, tmask))  # leaf 2: empty target leaf
    assert np.array_equal(org, torg) and vals.shape == (3, 512)
    assert np.all(vals[0] == 2.0) and np.all(vals[1:] == -7.0)
    assert np.all(masks[1:] == 0)
    assert fl.tolist() == [1] and fm[0, 0] == np.uint64(0x3) and not fm[0, 1:].any()
    # an empty channel: every target leaf is new and every active target voxel is filled
    e = LeafGrid(origins=np.zeros((0, 3), np.int32), values=np.zeros((0, 512), np.float32),
                 background=np.float32(0.0), masks=np.zeros((0, 8), np.uint64))
    org, vals, masks, fl, fm = prepare_channel(e, (torg, tmask))
    assert org.shape == (3, 3) and fl.tolist() == [0, 1] and not masks.any()


def test_extrapolation_abi_rejects_bad_input_on_the_host():
    """The C ABI checks the leaf list and the fill set before any device work."""
    from uaamg_b200 import _lib
    from uaamg_b200.extrapolate import run_layers
    org = np.array([[0, 0, 0], [8, 0, 0]], np.int32)
    vals = np.zeros((2, 512), np.float32)
    masks = np.zeros((2, 8), np.uint64)
    fm = np.ones((2, 8), np.uint64)
    bad = [
        (np.array([[0, 0, 0], [4, 0, 0]], np.int32), np.array([0], np.int32)),   # origin not a multiple of 8
        (org, np.array([2], np.int32)),                                           # fill leaf out of range
        (org, np.array([1, 1], np.int32)),                                        # a leaf listed twice
        (np.array([[0, 0, 0], [0, 0, 0]], np.int32), np.array([0], np.int32)),   # duplicate output origin
    ]
    for o, fl in bad:
        with pytest.raises(_lib.UaamgError):
            run_layers(2, o, vals.copy(), masks.copy(), fl, np.ascontiguousarray(fm[: fl.size]))
    run_layers(2, org, vals, masks, np.zeros(0, np.int32), np.zeros((0, 8), np.uint64))  # nothing to fill


@pytest.mark.parametrize("neighbours,n_layer", [(6, 3), (26, 2), (6, 10)])
def test_dense_and_sorted_dilation_agree(monkeypatch, neighbours, n_layer):
    """The dense bounding-box dilation and the sorted-leaf one (used for huge
    sparse boxes) give the same leaves, in the same order, and masks."""
    from uaamg_b200 import topology as T
    rng = np.random.default_rng(neighbours + n_layer)
    shape = (37, 29, 44)
    g = dense_to_leaves(np.zeros(shape, np.float32), origin=(-24, 0, 8), active=rng.random(shape) < 0.002)
    a = T.dilate(g, n_layer, neighbours)
    monkeypatch.setattr(T, "_DENSE_MAX_CELLS", 0)
    b = T.dilate(g, n_layer, neighbours)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
