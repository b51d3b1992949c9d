"""The allocation-free residual norm (uaamg_poisson_residual_norm_noalloc).

It serves callers that may not allocate GPU memory while they run (a loop that
reserves its whole device budget up front, a host application that owns the
device heap): its reduction scratch is a fixed array inside the library rather
than per-handle memory.  This file is collected last so that a run stopping at
the first failure has already run every other test.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    from uaamg_b200 import build, scenes, _lib
    from uaamg_b200.poisson import LaplacianWithLevel
    from uaamg_b200.grids import unpack_masks
    build.build()
    L = _lib.lib()
    sc = scenes.plain_poisson_scene(n=48, seed=1)
    lap = LaplacianWithLevel.createPressurePoissonLaplacian(sc.phi, sc.face_weights, sc.dt, sc.dx)
    lap.set_stream(torch.cuda.current_stream().cuda_stream)
    rhs = lap.createPressurePoissonRightHandSide(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity, sc.dt)
    _, masks = lap.dof_topology(0)
    return torch, L, lap, rhs, unpack_masks(masks)


def test_noalloc_residual_norm_matches_allocating_entry_point():
    torch, L, lap, rhs, act = _setup()
    db = torch.from_numpy(rhs).cuda()
    rng = np.random.default_rng(0)
    for call in range(2):  # two calls in a row: the shared array keeps the previous call's contents
        x = (rng.standard_normal(rhs.shape) * act * (call + 1)).astype(np.float32)
        dx = torch.from_numpy(x).cuda()
        r1, n1 = torch.empty_like(db), torch.full((1,), -1.0, device="cuda")
        r2, n2 = torch.full_like(db, 7.0), torch.full((1,), -2.0, device="cuda")
        lap.residual_norm_device(dx, db, r1, n1)
        rc = L.uaamg_poisson_residual_norm_noalloc(lap._h, dx.data_ptr(), db.data_ptr(), r2.data_ptr(),
                                                   n2.data_ptr())
        assert rc == 0, L.uaamg_last_error()
        torch.cuda.synchronize()
        # same kernel on the same data: identical results (tolerance 0)
        assert torch.equal(r1, r2)
        assert float(n1.item()) == float(n2.item()) > 0
    assert L.uaamg_poisson_residual_norm_noalloc(None, None, None, None, None) == -1


def test_noalloc_call_allocates_nothing():
    """After a warm-up call, repeated calls leave the device's free memory and
    torch's allocator unchanged (the library's own pool is not touched)."""
    torch, L, lap, rhs, act = _setup()
    db = torch.from_numpy(rhs).cuda()
    dx = torch.from_numpy((act * 0.5).astype(np.float32)).cuda()
    r, nrm = torch.empty_like(db), torch.zeros(1, device="cuda")
    args = (lap._h, dx.data_ptr(), db.data_ptr(), r.data_ptr(), nrm.data_ptr())
    assert L.uaamg_poisson_residual_norm_noalloc(*args) == 0, L.uaamg_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    first = None
    for _ in range(5):
        assert L.uaamg_poisson_residual_norm_noalloc(*args) == 0, L.uaamg_last_error()
        torch.cuda.synchronize()
        first = float(nrm.item()) if first is None else first
        assert float(nrm.item()) == first
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_rejects_levels_above_the_limit():
    """A level 0 above the array's leaf limit is rejected with an error naming
    the limit, and nothing is written (the limit is lowered through the test
    hook so a small domain reaches the check)."""
    torch, L, lap, rhs, act = _setup()
    nl = lap.leaf_count(0)
    db = torch.from_numpy(rhs).cuda()
    dx = torch.zeros_like(db)
    r, nrm = torch.full_like(db, 3.0), torch.full((1,), -5.0, device="cuda")
    os.environ["UAAMG_NOALLOC_TEST_MAX_LEAVES"] = str(nl - 1)
    try:
        rc = L.uaamg_poisson_residual_norm_noalloc(lap._h, dx.data_ptr(), db.data_ptr(), r.data_ptr(),
                                                   nrm.data_ptr())
    finally:
        del os.environ["UAAMG_NOALLOC_TEST_MAX_LEAVES"]
    assert rc == -1
    msg = L.uaamg_last_error().decode()
    assert f"level 0 has {nl} leaves" in msg and f"at most {nl - 1}" in msg
    torch.cuda.synchronize()
    assert float(nrm.item()) == -5.0 and bool((r == 3.0).all())
