"""Velocity extrapolation into new voxels (vdb_velocity_extrapolator::
union_extrapolate, FLIP_vdb/vdb_velocity_extrapolator.cpp:585-662).

The topology steps of the reference run here on the host, at leaf level on the
flattened grids' masks (``uaamg_b200.topology``):

* the union of the three channels' active voxels dilated ``n_layer`` times over
  the 6 face neighbours (topologyUnion + dilateActiveValues(NN_FACE), :589-595),
  or a given target topology (:597);
* per channel, the voxels of that topology the channel lacks
  (topologyDifference, :602), and the channel's leaves extended by the target
  leaves it does not have (touchLeaf: background values, inactive, :609-611).

The layers (:614-658) then run on the GPU through ``uaamg_extrapolate_channel``
(host arrays) or ``uaamg_extrapolate_channel_device`` (values and masks in
device memory).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .grids import LeafGrid
from .topology import LeafIndex, dilate, topology_coords, topology_of, union  # noqa: F401  (re-exported)


def union_topology(grids, n_layer: int) -> tuple[np.ndarray, np.ndarray]:
    """Topology (origins, masks) of the union of the grids' active voxels
    dilated n_layer times over the 6 face neighbours."""
    return dilate(union(grids), n_layer, neighbours=6)


def prepare_channel(channel: LeafGrid, topology):
    """The inputs of the extrapolation layers for one channel: the output
    leaves (the channel's, then the topology's leaves the channel lacks), their
    values (background in new leaves) and active masks, and the fill set (output
    leaf index and, per leaf, the topology's voxels the channel lacks)."""
    torg, tmask = topology_of(topology)
    n_c = channel.leaf_count
    j = LeafIndex(channel.origins).find(torg)
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
