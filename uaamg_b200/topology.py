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
    uk, first, inv = np.unique(leaf_keys(org), return_index=True, return_inverse=True)
    out = np.zeros((uk.size, 8), np.uint64)
    np.bitwise_or.at(out, inv.reshape(-1), masks)
    return org[first].astype(np.int32), out


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


def dilate(topo, n: int, neighbours: int = 6) -> tuple[np.ndarray, np.ndarray]:
    """dilateActiveValues(n, NN_FACE) (neighbours=6) or
    (n, NN_FACE_EDGE_VERTEX) (neighbours=26) of a topology."""
    if neighbours not in (6, 26):
        raise ValueError("neighbours must be 6 or 26")
    org, masks = _nonempty(*topology_of(topo))
    step = dilate_face_once if neighbours == 6 else dilate_box_once
    for _ in range(int(n)):
        org, masks = step(org, masks)
    return org, masks
