"""packed_FloatGrid3 (SIMD_UAAMG/packed3grids.cpp:11-83): the oracle's
semantics on the CPU, and the uaamg_packed3_* kernels against it bit for bit
on the GPU (host and device paths, masks, non-zero backgrounds, negative
origins, channels of different topologies, the round trip)."""
import numpy as np
import pytest

from oracle import packed3 as orc
from uaamg_b200.grids import LeafGrid


def _rand_vec3(rng, n=40, span=6, neg=True):
    lo = -span // 2 if neg else 0
    cells = rng.choice(span ** 3, size=n, replace=False)
    org = np.stack(np.unravel_index(cells, (span, span, span)), axis=1).astype(np.int32) * 8 + lo * 8
    masks = rng.integers(0, 2 ** 63, size=(n, 8), dtype=np.int64).astype(np.uint64)
    vals = rng.standard_normal((n, 512, 3)).astype(np.float32)
    return LeafGrid(origins=org, values=vals, background=np.array([0.5, -1.5, 2.0], np.float32), masks=masks)


def test_tree_order_matches_openvdb_layout():
    # leaves in one 128^3 lower node sort x-major by leaf offset; the upper node and the root tile come first
    org = np.array([[8, 0, 0], [0, 8, 0], [0, 0, 8], [0, 0, 0], [128, 0, 0], [-8, 0, 0], [0, 0, 4096]], np.int32)
    got = org[orc.tree_order(org)].tolist()
    assert got == [[-8, 0, 0], [0, 0, 0], [0, 0, 8], [0, 8, 0], [8, 0, 0], [128, 0, 0], [0, 0, 4096]]


def test_oracle_round_trip_and_union():
    rng = np.random.default_rng(0)
    g = _rand_vec3(rng)
    ch = orc.from_vec3(g.origins, g.masks, g.values, g.background)
    act = np.unpackbits(g.masks.view(np.uint8), axis=1, bitorder="little").astype(bool)
    for c in range(3):
        assert np.array_equal(ch[c][act], g.values[:, :, c][act]) and np.all(ch[c][~act] == g.background[c])
    org, masks, vals = orc.to_vec3([(g.origins, g.masks, ch[c]) for c in range(3)])
    order = orc.tree_order(g.origins)
    assert np.array_equal(org, g.origins[order]) and np.array_equal(masks, g.masks[order])
    exp = np.where(act[order][:, :, None], g.values[order], 0.0)
    assert np.array_equal(vals, exp)
    # channels of different topologies: the union; a component is 0 where its channel is inactive or absent
    a = (g.origins[:10], g.masks[:10], ch[0][:10])
    b = (g.origins[5:20], None, ch[1][5:20])
    c = (np.zeros((0, 3), np.int32), None, np.zeros((0, 512), np.float32))
    org, masks, vals = orc.to_vec3([a, b, c])
    assert org.shape[0] == 20 and np.all(vals[:, :, 2] == 0)


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    from uaamg_b200 import build
    build.build()
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("device", [False, True])
def test_from_vec3_bit_exact(gpu, device):
    torch = gpu
    from uaamg_b200.packed3 import packed_FloatGrid3
    rng = np.random.default_rng(1)
    g = _rand_vec3(rng, n=300, span=10)
    ref = orc.from_vec3(g.origins, g.masks, g.values, g.background)
    inp = g
    if device:
        inp = LeafGrid(origins=g.origins, values=g.values, background=g.background, masks=g.masks)
        inp.values = torch.from_numpy(g.values).cuda()
    p = packed_FloatGrid3()
    p.from_vec3(inp)
    for c in range(3):
        got = p.v[c].values.cpu().numpy() if device else p.v[c].values
        assert np.array_equal(got, ref[c]), c
        assert np.array_equal(p.v[c].origins, g.origins) and np.array_equal(p.v[c].masks, g.masks)
        assert float(p.v[c].background[0]) == float(g.background[c])
    p.from_vec3(inp, topologycopy=True)
    for c in range(3):
        got = p.v[c].values.cpu().numpy() if device else p.v[c].values
        assert np.all(got == g.background[c])


@pytest.mark.gpu
@pytest.mark.parametrize("device", [False, True])
def test_to_vec3_bit_exact_and_round_trip(gpu, device):
    torch = gpu
    from uaamg_b200.packed3 import packed_FloatGrid3
    rng = np.random.default_rng(2)
    g = _rand_vec3(rng, n=300, span=10)
    chans = orc.from_vec3(g.origins, g.masks, g.values, g.background)
    # channel 0: the first 200 leaves; 1: leaves 100-299 with all voxels active; 2: 150 leaves, shuffled
    sel = [np.arange(200), np.arange(100, 300), rng.permutation(300)[:150]]
    p = packed_FloatGrid3()
    trip = []
    for c in range(3):
        idx = sel[c]
        m = None if c == 1 else g.masks[idx]
        lg = LeafGrid(origins=g.origins[idx], values=chans[c][idx], background=g.background[c], masks=m)
        if c == 1:
            lg.masks = None
        if device:
            lg.values = torch.from_numpy(np.ascontiguousarray(chans[c][idx])).cuda()
        p.v[c] = lg
        trip.append((g.origins[idx], m, chans[c][idx]))
    out = p.to_vec3()
    org, masks, vals = orc.to_vec3(trip)
    got = out.values.cpu().numpy() if device else out.values
    assert np.array_equal(out.origins, org) and np.array_equal(out.masks, masks) and np.array_equal(got, vals)
    # round trip of one grid: the active values come back, the rest is 0
    q = packed_FloatGrid3()
    inp = LeafGrid(origins=g.origins, values=g.values, background=g.background, masks=g.masks)
    if device:
        inp.values = torch.from_numpy(g.values).cuda()
    q.from_vec3(inp)
    back = q.to_vec3()
    order = orc.tree_order(g.origins)
    act = np.unpackbits(g.masks[order].view(np.uint8), axis=1, bitorder="little").astype(bool)
    got = back.values.cpu().numpy() if device else back.values
    assert np.array_equal(back.origins, g.origins[order])
    assert np.array_equal(got, np.where(act[:, :, None], g.values[order], 0.0))
