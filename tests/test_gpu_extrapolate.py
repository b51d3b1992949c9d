"""GPU parity of the velocity extrapolation (union_extrapolate's layers,
vdb_velocity_extrapolator.cpp:611-659) against the oracle: velocities known on
the liquid and one band around it, extrapolated three layers into the union
topology and into a given target topology.  Per-voxel float means in the
reference's order: bit-exact."""
import numpy as np
import pytest

from oracle.oracle import extrapolate_channel as orc_extrapolate
from uaamg_b200 import scenes
from uaamg_b200.grids import dense_to_leaves, unpack_masks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    from uaamg_b200 import build
    build.build()
    return torch


@pytest.fixture(scope="module")
def channels(gpu):
    sc = scenes.plain_poisson_scene(n=48, seed=4)
    n = sc.n
    c = (np.arange(n + 1) + 0.5) / n
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    liquid = (Y < 0.4) | ((X - 0.5) ** 2 + (Y - 0.7) ** 2 + (Z - 0.5) ** 2 < 0.15 ** 2)
    rng = np.random.default_rng(9)
    out = []
    for k in range(3):
        known = liquid.copy()
        known[:, :, :] &= rng.random(known.shape) < 0.97  # holes the layers also fill
        vals = rng.uniform(-1, 1, known.shape).astype(np.float32)
        out.append(dense_to_leaves(vals, background=0.0, active=known))
    return out


@pytest.mark.parametrize("n_layer", [1, 3])
def test_extrapolation_bit_exact(channels, n_layer):
    from uaamg_b200.extrapolate import prepare_channel, run_layers, union_topology
    u = union_topology(channels, n_layer)
    for g in channels:
        org, vals, masks, fl, fm = prepare_channel(g, u)
        gv, gm = vals.copy(), masks.copy()
        run_layers(n_layer, org, gv, gm, fl, fm)
        ov, om = orc_extrapolate(n_layer, org, vals, masks, fl, fm)
        assert np.array_equal(gm, om)
        assert np.array_equal(gv, ov)
        grown = unpack_masks(gm).sum() - unpack_masks(g.masks).sum()
        assert grown > 0
        assert org.shape[0] > g.leaf_count  # touchLeaf: new leaves around the band


def test_union_extrapolate_into_target_topology(channels):
    from uaamg_b200.extrapolate import topology_coords, union_extrapolate, union_topology
    target = union_topology(channels[:1], 2)
    out = union_extrapolate(2, *channels, target_topology=target)
    for g_in, g_out in zip(channels, out):
        on = unpack_masks(g_out.masks)
        assert on.sum() >= unpack_masks(g_in.masks).sum()
        # every active voxel is either an input voxel or in the target topology
        act = {tuple(p) for p in topology_coords(target).tolist()}
        from uaamg_b200.grids import offsets_xyz
        xyz = offsets_xyz()
        before = unpack_masks(g_in.masks)
        idx = {tuple(o): i for i, o in enumerate(g_in.origins.tolist())}
        for i in range(g_out.leaf_count):
            j = idx.get(tuple(g_out.origins[i].tolist()))
            new = on[i] & ~(before[j] if j is not None else np.zeros(512, bool))
            for off in np.nonzero(new)[0][:16]:
                assert tuple((g_out.origins[i] + xyz[off]).tolist()) in act


def test_device_path_matches_host(channels, gpu):
    from uaamg_b200.extrapolate import prepare_channel, run_layers, run_layers_device, union_topology
    torch = gpu
    u = union_topology(channels, 2)
    for n_layer in (1, 2, 3):  # odd layer counts end in the scratch mask buffer
        org, vals, masks, fl, fm = prepare_channel(channels[1], u)
        hv, hm = vals.copy(), masks.copy()
        run_layers(n_layer, org, hv, hm, fl, fm)
        dv = torch.from_numpy(vals.copy()).cuda()
        dm = torch.from_numpy(masks.view(np.int64).copy()).cuda()
        torch.cuda.synchronize()
        run_layers_device(n_layer, org, dv, dm, fl, fm)
        torch.cuda.synchronize()
        assert np.array_equal(dv.cpu().numpy(), hv)
        assert np.array_equal(dm.cpu().numpy().view(np.uint64), hm)
