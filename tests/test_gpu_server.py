"""GPU tests of the native served form (uaamg_server_* through
uaamg_b200.server.NativeServer): every substep's result is the same, bit for
bit, as the same request solved alone through the plain API (pressure warm-
started from the previous substep's pressure; viscosity warm-started from the
velocity), whether the pressure rounds are batched or not and whatever else is
in the mix; each pressure result carries its FP64 residual; the budget limits
what is resident."""
import numpy as np
import pytest

from uaamg_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    from uaamg_b200 import build
    build.build()
    return torch


POIS = [(32, 11, 3), (48, 12, 2), (40, 13, 4)]  # (side, seed, substeps)
VISC = [(32, 21, 2)]


def _vel(torch, side, seed, k):
    return scenes.device_face_velocities(side, seed * 1000003 + k, torch.device("cuda"))


def _alone_poisson(torch, side, seed, substeps):
    from uaamg_b200.poisson import LaplacianWithLevel, PoissonSolver
    phi, fw, sv, dt, dx = scenes.device_poisson_instance(side, seed, torch.device("cuda"))
    lap = LaplacianWithLevel.createPressurePoissonLaplacian(phi, fw, dt, dx)
    s = PoissonSolver(lap)
    x = torch.zeros((lap.leaf_count(0), 512), device="cuda")
    rhs = torch.empty_like(x)
    out = []
    for k in range(substeps):
        vx, vy, vz = _vel(torch, side, seed, k)
        lap.createPressurePoissonRightHandSide(fw, vx, vy, vz, sv, dt, out=rhs)
        st = s.solveMultigridPCG(x, rhs)
        out.append((st, s.mIterationTaken, x.cpu().numpy().copy()))
    return out


def _alone_viscosity(torch, side, seed, substeps):
    from uaamg_b200.viscosity import L_with_level, simd_viscosity3d
    liq, sol, mu, sv, dt, rho, dx = scenes.device_viscosity_instance(side, seed, torch.device("cuda"))
    lv = L_with_level.create_viscosity_matrix(mu, liq, sol, dt, rho, dx)
    n = lv.leaf_count(0)
    rhs = torch.empty((3, n, 512), device="cuda")
    x = torch.empty_like(rhs)
    out = []
    for k in range(substeps):
        u, v, w = _vel(torch, side, seed, k)
        lv.build_rhs(u, v, w, sv, out=rhs)
        lv.gather_velocity(u, v, w, out=x)
        s = simd_viscosity3d(lv)
        st = s.pcg_solve(x, 1e-6, rhs)
        out.append((st, s.m_iteration, x.cpu().numpy().copy()))
    return out


def _served(torch, batching, budget=None, interleave=True):
    from uaamg_b200.server import NativeServer, POISSON, VISCOSITY
    srv = NativeServer(batching=batching, keep_results=True, budget_bytes=budget)
    reqs = []
    for side, seed, sub in POIS:
        phi, fw, sv, dt, dx = scenes.device_poisson_instance(side, seed, torch.device("cuda"))
        reqs.append((srv.submit_poisson(phi, fw, sv, dt, dx, sub), POISSON, side, seed, sub))
    for side, seed, sub in VISC:
        liq, sol, mu, sv, dt, rho, dx = scenes.device_viscosity_instance(side, seed, torch.device("cuda"))
        reqs.append((srv.submit_viscosity(mu, liq, sol, sv, dt, rho, dx, sub), VISCOSITY, side, seed, sub))
    # velocities pushed substep by substep across all requests (or request by request)
    order = ([(i, k) for k in range(max(r[4] for r in reqs)) for i in range(len(reqs))] if interleave
             else [(i, k) for i in range(len(reqs)) for k in range(reqs[i][4])])
    for i, k in order:
        rid, kind, side, seed, sub = reqs[i]
        if k < sub:
            srv.push_velocity(rid, *_vel(torch, side, seed, k))
    res = []
    for rid, kind, side, seed, sub in reqs:
        per = []
        for k in range(sub):
            w = srv.wait(rid, k, 120.0)
            per.append((w, srv.result(rid, k, kind)))
        res.append(per)
    stats = srv.stats()
    srv.close()
    return reqs, res, stats


@pytest.mark.parametrize("batching", [True, False])
def test_served_results_identical_to_alone(gpu, batching):
    torch = gpu
    reqs, res, stats = _served(torch, batching)
    alone = [_alone_poisson(torch, *p) for p in POIS] + [_alone_viscosity(torch, *v) for v in VISC]
    for (rid, kind, side, seed, sub), got, ref in zip(reqs, res, alone):
        for k in range(sub):
            w, x = got[k]
            st, it, xr = ref[k]
            assert w["status"] == st == 0 and w["iterations"] == it, (kind, side, k, w, it)
            assert np.array_equal(x, xr), (kind, side, k)
            if kind == 0:
                assert 0.0 < w["fp64_residual"] < 1e-5
            assert w["latency_s"] > 0
    assert stats["done"] == len(reqs) and stats["failed"] == 0
    assert stats["solves"] == sum(r[4] for r in reqs)
    if batching:
        # how many substeps share a round depends on when their velocities arrive
        assert stats["batch_builds"] >= 1 and stats["rounds"] <= sum(p[2] for p in POIS)


def test_served_under_a_tight_budget(gpu):
    """A budget that holds about one request at a time: requests are admitted
    as others complete, and the results do not change."""
    torch = gpu
    from uaamg_b200.server import NativeServer
    dev = torch.device("cuda")
    # the server's own estimate (leaf arrays of the largest input grid, plus
    # 64 MiB) for the largest request, plus a little
    ests = []
    for side, seed, _ in POIS:
        phi, fw, sv, dt, dx = scenes.device_poisson_instance(side, seed, dev)
        ests.append(max(phi.leaf_count, fw.leaf_count) * 512 * 4 * 20 + (64 << 20))
    for side, seed, _ in VISC:
        liq, sol, mu, sv, dt, rho, dx = scenes.device_viscosity_instance(side, seed, dev)
        ests.append(max(liq.leaf_count, sol.leaf_count) * 512 * 4 * 110 + (64 << 20))
    est = max(ests)
    reqs, res, stats = _served(torch, True, budget=int(est * 1.2), interleave=False)
    assert stats["peak_bytes"] <= int(est * 1.2) and stats["done"] == len(reqs)
    alone = [_alone_poisson(torch, *p) for p in POIS] + [_alone_viscosity(torch, *v) for v in VISC]
    for (rid, kind, side, seed, sub), got, ref in zip(reqs, res, alone):
        for k in range(sub):
            assert np.array_equal(got[k][1], ref[k][2])


def test_server_argument_errors(gpu):
    torch = gpu
    from uaamg_b200 import _lib
    from uaamg_b200.server import NativeServer
    with NativeServer(budget_bytes=1 << 20) as srv:  # 1 MiB: no request fits
        phi, fw, sv, dt, dx = scenes.device_poisson_instance(32, 1, torch.device("cuda"))
        with pytest.raises(_lib.UaamgError, match="budget"):
            srv.submit_poisson(phi, fw, sv, dt, dx, 1)
    with NativeServer() as srv:
        rid = srv.submit_poisson(phi, fw, sv, dt, dx, 1)
        u, v, w = _vel(torch, 32, 1, 0)
        srv.push_velocity(rid, u, v, w)
        with pytest.raises(_lib.UaamgError, match="already has all"):
            srv.push_velocity(rid, u, v, w)
        with pytest.raises(_lib.UaamgError, match="unknown request"):
            srv.push_velocity(rid + 99, u, v, w)
        assert srv.wait(rid, 0, 60.0)["status"] == 0
        with pytest.raises(_lib.UaamgError, match="keeps no solutions"):
            srv.result(rid, 0)
