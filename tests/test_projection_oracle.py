"""The oracle's restatement of the steps either side of the pressure solve
(projection_oracle.c) on CPU: fraction_inside over a square against closed
forms, its symmetries, and the face-weight topology (the liquid SDF dilated
by two voxels)."""
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
