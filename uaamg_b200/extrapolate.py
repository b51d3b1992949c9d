"""Velocity extrapolation into new voxels (vdb_velocity_extrapolator::
union_extrapolate, FLIP_vdb/vdb_velocity_extrapolator.cpp:585-662).

The topology steps of the reference run here on the host, at leaf level on the
flattened grids' masks (word x, bit 8y + z of each 8^3 leaf):

* the union of the three channels' active voxels dilated ``n_layer`` times over
  the 6 face neighbours (topologyUnion + dilateActiveValues(NN_FACE), :589-595),
  or a given target topology (:597);
* per channel, the voxels of that topology the channel lacks
  (topologyDifference, :602), and the channel's leaves extended by the target
  leaves it does not have (touchLeaf: background values, inactive, :609-611).

The layers (:614-658) then run on the GPU through ``uaamg_extrapolate_channel``
(host arrays) or ``uaamg_extrapolate_channel_device`` (values and masks in
device memory).  A topology is a pair (origins int32 [m, 3], masks uint64
[m, 8]).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .grids import LeafGrid, offsets_xyz, unpack_masks

_U = np.uint64
_Z_LO = _U(0x0101010101010101)  # bits with z = 0
_Z_HI = _U(0x8080808080808080)  # bits with z = 7
_DIRS = np.array([[-8, 0, 0], [8, 0, 0], [0, -8, 0], [0, 8, 0], [0, 0, -8], [0, 0, 8]], np.int64)
_BIAS = 1 << 20


def _keys(org: np.ndarray) -> np.ndarray:
    """One int64 key per leaf origin (leaf coordinates biased into 21 bits)."""
    o = (np.asarray(org, np.int64).reshape(-1, 3) >> 3) + _BIAS
    return (o[:, 0] << 42) | (o[:, 1] << 21) | o[:, 2]


class _Index:
    """Leaf lookup by origin over one leaf list (sorted keys)."""

    def __init__(self, org: np.ndarray):
        k = _keys(org)
        self.order = np.argsort(k, kind="stable")
        self.sorted = k[self.order]

    def find(self, org: np.ndarray) -> np.ndarray:
        """Index of each queried origin in the leaf list, -1 where absent."""
        q = _keys(org)
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


def _union(topos) -> tuple[np.ndarray, np.ndarray]:
    org = np.concatenate([t[0] for t in topos], axis=0).reshape(-1, 3)
    masks = np.concatenate([t[1] for t in topos], axis=0).reshape(-1, 8)
    if org.shape[0] == 0:
        return org.astype(np.int32), masks.astype(np.uint64)
    uk, first, inv = np.unique(_keys(org), return_index=True, return_inverse=True)
    out = np.zeros((uk.size, 8), np.uint64)
    np.bitwise_or.at(out, inv.reshape(-1), masks)
    return org[first].astype(np.int32), out


def _dilate_face(org: np.ndarray, masks: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """One face-neighbour dilation of a topology of non-empty leaves; leaves
    with no active voxel are dropped from the result."""
    if org.shape[0] == 0:
        return org, masks
    # the leaves a dilation can reach: every leaf and its 6 face neighbours
    nb = (org[:, None, :].astype(np.int64) + _DIRS[None]).reshape(-1, 3)
    org2, _ = _union([(org, masks), (nb, np.zeros((nb.shape[0], 8), np.uint64))])
    idx = _Index(org)

    def gather(shift):
        j = idx.find(org2.astype(np.int64) + shift)
        out = np.zeros((org2.shape[0], 8), np.uint64)
        out[j >= 0] = masks[j[j >= 0]]
        return out

    M = gather(np.zeros(3, np.int64))
    D = M.copy()
    D |= (M << _U(1)) & ~_Z_LO          # z + 1 within the leaf
    D |= (M >> _U(1)) & ~_Z_HI          # z - 1
    D |= M << _U(8)                     # y + 1
    D |= M >> _U(8)                     # y - 1
    D[:, 1:] |= M[:, :-1]               # x + 1
    D[:, :-1] |= M[:, 1:]               # x - 1
    mnx, mpx, mny, mpy, mnz, mpz = (gather(_DIRS[d]) for d in range(6))
    D[:, 0] |= mnx[:, 7]                # from the -x leaf's x = 7 plane
    D[:, 7] |= mpx[:, 0]                # from the +x leaf's x = 0 plane
    D |= mny >> _U(56)                  # -y leaf's y = 7 row -> y = 0
    D |= mpy << _U(56)                  # +y leaf's y = 0 row -> y = 7
    D |= (mnz >> _U(7)) & _Z_LO         # -z leaf's z = 7 -> z = 0
    D |= (mpz << _U(7)) & _Z_HI         # +z leaf's z = 0 -> z = 7
    keep = D.any(axis=1)
    return org2[keep].astype(np.int32), D[keep]


def union_topology(grids, n_layer: int) -> tuple[np.ndarray, np.ndarray]:
    """Topology (origins, masks) of the union of the grids' active voxels
    dilated n_layer times over the 6 face neighbours."""
    org, masks = _union([topology_of(g) for g in grids])
    live = masks.any(axis=1)
    org, masks = org[live], masks[live]
    for _ in range(int(n_layer)):
        org, masks = _dilate_face(org, masks)
    return org, masks


def prepare_channel(channel: LeafGrid, topology):
    """The inputs of the extrapolation layers for one channel: the output
    leaves (the channel's, then the topology's leaves the channel lacks), their
    values (background in new leaves) and active masks, and the fill set (output
    leaf index and, per leaf, the topology's voxels the channel lacks)."""
    torg, tmask = topology_of(topology)
    n_c = channel.leaf_count
    j = _Index(channel.origins).find(torg)
    have = np.zeros_like(tmask)
    have[j >= 0] = channel.masks[j[j >= 0]]
    extra = tmask & ~have
    new = j < 0
    out_org = np.ascontiguousarray(np.concatenate([channel.origins.astype(np.int32), torg[new]], axis=0))
    n_out = out_org.shape[0]
    vals = np.empty((n_out, 512), np.float32)
    vals[:n_c] = channel.values
    vals[n_c:] = channel.background.reshape(-1)[0]
    masks = np.zeros((n_out, 8), np.uint64)
    masks[:n_c] = channel.masks
    out_index = j.copy()
    out_index[new] = n_c + np.arange(int(new.sum()))
    fill = extra.any(axis=1)
    return (out_org, vals, masks, np.ascontiguousarray(out_index[fill], dtype=np.int32),
            np.ascontiguousarray(extra[fill], dtype=np.uint64))


def run_layers(n_layer: int, out_org, vals, masks, fill_leaf, fill_masks) -> None:
    """The extrapolation layers on the GPU (vals and masks updated in place)."""
    n_out = int(out_org.shape[0])
    nf = int(fill_leaf.size)
    rc = _lib.lib().uaamg_extrapolate_channel(
        int(n_layer), n_out, out_org.ctypes.data if n_out else None, vals.ctypes.data if n_out else None,
        masks.ctypes.data if n_out else None, nf, fill_leaf.ctypes.data if nf else None,
        fill_masks.ctypes.data if nf else None)
    _lib.check(rc, "extrapolate_channel")


def run_layers_device(n_layer: int, out_org, vals_dev, masks_dev, fill_leaf, fill_masks, stream=None) -> None:
    """The layers on device tensors (values [n_out, 512] float32 and masks
    [n_out, 8] int64, updated in place), enqueued on ``stream`` (a
    cudaStream_t handle; None: the legacy default stream).  The topology
    arrays are host arrays."""
    n_out = int(out_org.shape[0])
    nf = int(fill_leaf.size)
    rc = _lib.lib().uaamg_extrapolate_channel_device(
        int(n_layer), n_out, out_org.ctypes.data if n_out else None, vals_dev.data_ptr() if n_out else None,
        masks_dev.data_ptr() if n_out else None, nf, fill_leaf.ctypes.data if nf else None,
        fill_masks.ctypes.data if nf else None, stream)
    _lib.check(rc, "extrapolate_channel_device")


def extrapolate_channel(channel: LeafGrid, topology, n_layer: int) -> LeafGrid:
    """One channel extrapolated n_layer layers into ``topology``."""
    out_org, vals, masks, fill_leaf, fill_masks = prepare_channel(channel, topology)
    run_layers(n_layer, out_org, vals, masks, fill_leaf, fill_masks)
    return LeafGrid(origins=out_org, values=vals, background=channel.background.copy(), masks=masks)


def union_extrapolate(n_layer: int, vx: LeafGrid, vy: LeafGrid, vz: LeafGrid, target_topology=None):
    """The three channels extrapolated n_layer layers into the union topology
    (or ``target_topology``: a LeafGrid whose active voxels are the target, as
    the reference's target tree, or an (origins, masks) pair); returns new
    grids."""
    topo = union_topology((vx, vy, vz), n_layer) if target_topology is None else topology_of(target_topology)
    return tuple(extrapolate_channel(g, topo, n_layer) for g in (vx, vy, vz))
