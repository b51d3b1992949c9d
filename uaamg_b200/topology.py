"""Leaf-level topology operations on flattened grids (host side).

A topology is a pair (origins int32 [m, 3], masks uint64 [m, 8]) in the
OpenVDB leaf layout: voxel offset 64x + 8y + z, so mask word x holds the
8 x 8 (y, z) plane with bit 8y + z.  The operations restate the OpenVDB tree
operations the reference applies to grid topologies -- topologyUnion and
dilateActiveValues with NN_FACE (6 neighbours) or NN_FACE_EDGE_VERTEX
(26 neighbours) -- as shifts inside each leaf plus the boundary planes of the
neighbour leaves, vectorised over all leaves.  Leaves without an active
voxel are dropped from dilation results.
"""
from __future__ import annotations

import numpy as np

from .grids import LeafGrid, offsets_xyz, unpack_masks

_U = np.uint64
_Z_LO = _U(0x0101010101010101)  # bits with z = 0
_Z_HI = _U(0x8080808080808080)  # bits with z = 7
_DIRS = np.array([[-8, 0, 0], [8, 0, 0], [0, -8, 0], [0, 8, 0], [0, 0, -8], [0, 0, 8]], np.int64)
_BIAS = 1 << 20


def leaf_keys(org: np.ndarray) -> np.ndarray:
    """One int64 key per leaf origin (leaf coordinates biased into 21 bits);
    keys sort in x-major, then y, then z order."""
    o = (np.asarray(org, np.int64).reshape(-1, 3) >> 3) + _BIAS
    return (o[:, 0] << 42) | (o[:, 1] << 21) | o[:, 2]


class LeafIndex:
    """Leaf lookup by origin over one leaf list (sorted keys)."""

    def __init__(self, org: np.ndarray):
        k = leaf_keys(org)
        self.order = np.argsort(k, kind="stable")
        self.sorted = k[self.order]

    def find(self, org: np.ndarray) -> np.ndarray:
        """Index of each queried origin in the leaf list, -1 where absent."""
        q = leaf_keys(org)
        if self.sorted.size == 0:
            return np.full(q.shape, -1, np.int64)
        pos = np.minimum(np.searchsorted(self.sorted, q), self.sorted.size - 1)
        return np.where(self.sorted[pos] == q, self.order[pos], -1)


def topology_of(g) -> tuple[np.ndarray, np.ndarray]:
    """The (origins, masks) topology of a LeafGrid, or a topology itself."""
    if isinstance(g, LeafGrid):
        return g.origins.astype(np.int32), g.masks
    org, masks = g
    return (np.ascontiguousarray(org, np.int32).reshape(-1, 3),
            np.ascontiguousarray(masks, np.uint64).reshape(-1, 8))


def topology_coords(topo) -> np.ndarray:
    """Active voxel coordinates [k, 3] (int64) of a topology or LeafGrid."""
    org, masks = topology_of(topo)
    li, off = np.nonzero(unpack_masks(masks))
    return org[li].astype(np.int64) + offsets_xyz()[off]


def union(topos) -> tuple[np.ndarray, np.ndarray]:
    """topologyUnion of several topologies: leaves sorted by origin (x-major),
    masks OR-ed."""
    topos = [topology_of(t) for t in topos]
    org = np.concatenate([t[0] for t in topos], axis=0).reshape(-1, 3)
    masks = np.concatenate([t[1] for t in topos], axis=0).reshape(-1, 8)
    if org.shape[0] == 0:
        return org.astype(np.int32), masks.astype(np.uint64)
    k = leaf_keys(org)
    order = np.argsort(k, kind="stable")
    ks = k[order]
    starts = np.flatnonzero(np.r_[True, ks[1:] != ks[:-1]])
    out = np.bitwise_or.reduceat(masks[order], starts, axis=0)
    return org[order[starts]].astype(np.int32), np.ascontiguousarray(out, dtype=np.uint64)


def _nonempty(org, masks):
    live = masks.any(axis=1)
    return org[live], masks[live]


def _with_neighbours(org, masks, dirs):
    """The leaves plus their neighbours in the given directions, and a gather
    of the original masks at an offset from each of those leaves."""
    nb = (org[:, None, :].astype(np.int64) + dirs[None]).reshape(-1, 3)
    org2, _ = union([(org, masks), (nb, np.zeros((nb.shape[0], 8), np.uint64))])
    idx = LeafIndex(org)

    def gather(shift):
        j = idx.find(org2.astype(np.int64) + shift)
        out = np.zeros((org2.shape[0], 8), np.uint64)
        out[j >= 0] = masks[j[j >= 0]]
        return out

    return org2, gather


def _z_pass(M, mn, mp):
    return M | ((M << _U(1)) & ~_Z_LO) | ((M >> _U(1)) & ~_Z_HI) | ((mn >> _U(7)) & _Z_LO) | ((mp << _U(7)) & _Z_HI)


def _y_pass(M, mn, mp):
    return M | (M << _U(8)) | (M >> _U(8)) | (mn >> _U(56)) | (mp << _U(56))


def _x_pass(M, mn, mp):
    D = M.copy()
    D[:, 1:] |= M[:, :-1]
    D[:, :-1] |= M[:, 1:]
    D[:, 0] |= mn[:, 7]
    D[:, 7] |= mp[:, 0]
    return D


_PASSES = (_x_pass, _y_pass, _z_pass)


def dilate_face_once(org, masks):
    """One NN_FACE dilation (the 6 face neighbours)."""
    org, masks = _nonempty(org, masks)
    if org.shape[0] == 0:
        return org, masks
    org2, gather = _with_neighbours(org, masks, _DIRS)
    M = gather(np.zeros(3, np.int64))
    D = M.copy()
    for axis in range(3):
        D |= _PASSES[axis](M, gather(_DIRS[2 * axis]), gather(_DIRS[2 * axis + 1]))
    return _nonempty(org2.astype(np.int32), D)


def dilate_box_once(org, masks):
    """One NN_FACE_EDGE_VERTEX dilation (the 26 neighbours): the 1-D
    dilations along z, y and x applied in turn."""
    org, masks = _nonempty(org, masks)
    for axis in (2, 1, 0):
        if org.shape[0] == 0:
            break
        org2, gather = _with_neighbours(org, masks, _DIRS[2 * axis: 2 * axis + 2])
        M = gather(np.zeros(3, np.int64))
        org, masks = _nonempty(org2.astype(np.int32),
                               _PASSES[axis](M, gather(_DIRS[2 * axis]), gather(_DIRS[2 * axis + 1])))
    return org, masks


# ---------------------------------------------------------------------------
# Dense form: the masks of every leaf cell of the bounding box (plus a margin)
# in one [X, Y, Z, 8] array, where a 1-D pass is a few whole-array shifts and
# the neighbour planes come from the adjacent cells.  Used when the box is
# small enough; same results and leaf order (x-major) as the sorted form.
_DENSE_MAX_CELLS = 1 << 24


def _dense_z(V):
    D = V | ((V << _U(1)) & ~_Z_LO) | ((V >> _U(1)) & ~_Z_HI)
    D[:, :, 1:] |= (V[:, :, :-1] >> _U(7)) & _Z_LO
    D[:, :, :-1] |= (V[:, :, 1:] << _U(7)) & _Z_HI
    return D


def _dense_y(V):
    D = V | (V << _U(8)) | (V >> _U(8))
    D[:, 1:] |= V[:, :-1] >> _U(56)
    D[:, :-1] |= V[:, 1:] << _U(56)
    return D


def _dense_x(V):
    D = V.copy()
    D[..., 1:] |= V[..., :-1]
    D[..., :-1] |= V[..., 1:]
    D[1:, :, :, 0] |= V[:-1, :, :, 7]
    D[:-1, :, :, 7] |= V[1:, :, :, 0]
    return D


def _dilate_dense(org, masks, n, neighbours):
    lc = org.astype(np.int64) >> 3
    pad = 1 + (int(n) + 7) // 8
    lo = lc.min(axis=0) - pad
    dims = lc.max(axis=0) + pad + 1 - lo
    V = np.zeros((int(dims[0]), int(dims[1]), int(dims[2]), 8), np.uint64)
    c = lc - lo
    V[c[:, 0], c[:, 1], c[:, 2]] = masks
    for _ in range(int(n)):
        if neighbours == 6:
            V = _dense_x(V) | _dense_y(V) | _dense_z(V)
        else:
            V = _dense_x(_dense_y(_dense_z(V)))
    live = V.any(axis=3)
    cells = np.argwhere(live)
    return ((cells + lo) * 8).astype(np.int32), np.ascontiguousarray(V[live])


def dilate(topo, n: int, neighbours: int = 6) -> tuple[np.ndarray, np.ndarray]:
    """dilateActiveValues(n, NN_FACE) (neighbours=6) or
    (n, NN_FACE_EDGE_VERTEX) (neighbours=26) of a topology."""
    if neighbours not in (6, 26):
        raise ValueError("neighbours must be 6 or 26")
    org, masks = _nonempty(*topology_of(topo))
    if org.shape[0] == 0 or int(n) <= 0:
        return org, masks
    org, masks = union([(org, masks)])  # one entry per leaf
    lc = org.astype(np.int64) >> 3
    pad = 1 + (int(n) + 7) // 8
    cells = int(np.prod(lc.max(axis=0) - lc.min(axis=0) + 1 + 2 * pad))
    if cells <= _DENSE_MAX_CELLS:
        return _dilate_dense(org, masks, n, neighbours)
    step = dilate_face_once if neighbours == 6 else dilate_box_once
    for _ in range(int(n)):
        org, masks = step(org, masks)
    return org, masks
