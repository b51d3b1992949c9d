"""The allocation-free residual norm (uaamg_poisson_residual_norm_noalloc).

It serves callers that may not allocate GPU memory while they run (a loop that
reserves its whole device budget up front, a host application that owns the
device heap): its reduction scratch is a fixed array inside the library rather
than per-handle memory.  This file is collected last so that a run stopping at
the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_residual_norm_matches_allocating_entry_point():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    from uaamg_b200 import build, scenes, _lib
    from uaamg_b200.poisson import LaplacianWithLevel
    build.build()
    L = _lib.lib()
    sc = scenes.plain_poisson_scene(n=48, seed=1)
    lap = LaplacianWithLevel.createPressurePoissonLaplacian(sc.phi, sc.face_weights, sc.dt, sc.dx)
    lap.set_stream(torch.cuda.current_stream().cuda_stream)
    rhs = lap.createPressurePoissonRightHandSide(sc.face_weights, sc.vx, sc.vy, sc.vz, sc.solid_velocity, sc.dt)
    _, masks = lap.dof_topology(0)
    from uaamg_b200.grids import unpack_masks
    act = unpack_masks(masks)
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
