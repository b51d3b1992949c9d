"""CPU oracle of packed_FloatGrid3 (SIMD_UAAMG/packed3grids.cpp:11-83).

Test infrastructure: imported only by tests/ as the checker of the
uaamg_packed3_* kernels, never by the library.  The reference has no test or
fixture for this file; the restatement follows the source lines cited, and the
tests add the round trip (to_vec3 of from_vec3 gives back the active values).
"""
from __future__ import annotations

import numpy as np


def tree_order(origins: np.ndarray) -> np.ndarray:
    """Indices that sort leaf origins into OpenVDB tree order for the
    Tree4<float, 5, 4, 3> layout: the root's tiles (4096^3) by (x, y, z), then
    the 32^3 children of the upper internal node, then the 16^3 leaves of the
    lower one, each by its linear offset (x-major)."""
    o = np.asarray(origins, np.int64).reshape(-1, 3)
    tile = o & ~np.int64(4095)
    off5 = (((o[:, 0] & 4095) >> 7) << 10) | (((o[:, 1] & 4095) >> 7) << 5) | ((o[:, 2] & 4095) >> 7)
    off4 = (((o[:, 0] & 127) >> 3) << 8) | (((o[:, 1] & 127) >> 3) << 4) | ((o[:, 2] & 127) >> 3)
    return np.lexsort((off4, off5, tile[:, 2], tile[:, 1], tile[:, 0]))


def _active(masks, n):
    if masks is None:
        return np.ones((n, 512), bool)
    m = np.asarray(masks, np.uint64).reshape(n, 8)
    return np.unpackbits(m.view(np.uint8), axis=1, bitorder="little").astype(bool)


def from_vec3(origins, masks, values, background):
    """from_vec3 (:11-43): per channel, the topology copy holds the background
    everywhere (Tree(other, background, TopologyCopy)), then the converter
    sets component c at every active voxel (:30-39)."""
    v = np.asarray(values, np.float32)
    n = v.shape[0]
    act = _active(masks, n)
    bg = np.asarray(background, np.float32).reshape(3)
    return [np.where(act, v[:, :, c], bg[c]).astype(np.float32) for c in range(3)]


def to_vec3(channels):
    """to_vec3 (:46-83): channels = three (origins, masks, values) triples.
    The output tree (background (0,0,0)) takes the union of the channels'
    topologies (:54-59), then component c is set at the active voxels of
    channel c (:63-76).  Returns (origins, masks, values [n][512][3]) in tree
    order."""
    allorg = np.concatenate([np.asarray(o, np.int32).reshape(-1, 3) for o, _, _ in channels], axis=0)
    if allorg.shape[0] == 0:
        return np.zeros((0, 3), np.int32), np.zeros((0, 8), np.uint64), np.zeros((0, 512, 3), np.float32)
    uniq = np.unique(allorg, axis=0)
    uniq = uniq[tree_order(uniq)]
    index = {tuple(o): i for i, o in enumerate(uniq.tolist())}
    n = uniq.shape[0]
    act_u = np.zeros((n, 512), bool)
    vals = np.zeros((n, 512, 3), np.float32)
    for c, (org, masks, v) in enumerate(channels):
        org = np.asarray(org, np.int32).reshape(-1, 3)
        act = _active(masks, org.shape[0])
        v = np.asarray(v, np.float32).reshape(-1, 512)
        for i, o in enumerate(org.tolist()):
            j = index[tuple(o)]
            act_u[j] |= act[i]
            vals[j, act[i], c] = v[i, act[i]]
    masks_u = np.packbits(act_u, axis=1, bitorder="little").view(np.uint64).reshape(n, 8)
    return uniq, masks_u, vals
