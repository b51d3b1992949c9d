"""Seeded synthetic fluid domains for the UAAMG-PCG workloads.

The reference's benchmark scenes are procedural (CG_benchmarks/main.cpp:108-221,
1559-1614) and use std::mt19937 whose output is implementation-defined through
std::uniform_real_distribution, so the same shapes are regenerated here with a
portable counter-based generator (SplitMix64 outputs, top 24 bits -> [0,1)).

Poisson inputs follow FLIP_vdb's pressure call site (FLIP_vdb.cpp:3118-3168):
liquid SDF sampled at voxel centres, solid face fractions (FLIP_vdb.cpp:2669-2752,
here: 1 in the interior, 0 on the domain walls), three staggered face-velocity
channels (packed3grids) and a zero solid velocity.
"""
from __future__ import annotations

import functools
from dataclasses import dataclass

import numpy as np

from .grids import LeafGrid, dense_to_leaves

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int, start: int = 0) -> np.ndarray:
    """Outputs ``start .. start+count-1`` of SplitMix64 seeded with ``seed``."""
    with np.errstate(over="ignore"):
        k = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + k * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, count: int, lo: float, hi: float, start: int = 0) -> np.ndarray:
    u = (splitmix64(seed, count, start) >> np.uint64(40)).astype(np.float64) * (1.0 / (1 << 24))
    return (lo + (hi - lo) * u).astype(np.float32)


@dataclass
class PoissonScene:
    name: str
    n: int
    dx: float
    dt: float
    phi: LeafGrid
    face_weights: LeafGrid
    vx: LeafGrid
    vy: LeafGrid
    vz: LeafGrid
    solid_velocity: LeafGrid


def _walls_face_weights(n: int) -> np.ndarray:
    """Face fractions on the (n+1)^3 face lattice: component k of voxel c is the
    face between c-e_k and c; faces on the six domain walls are solid (0)."""
    w = np.ones((n + 1, n + 1, n + 1, 3), dtype=np.float32)
    w[0, :, :, 0] = 0.0; w[n, :, :, 0] = 0.0
    w[:, 0, :, 1] = 0.0; w[:, n, :, 1] = 0.0
    w[:, :, 0, 2] = 0.0; w[:, :, n, 2] = 0.0
    return w


def sdf_box_scene(n: int, slab_height: float | None, spheres, seed: int, dt: float = 1.0,
                  name: str = "poisson") -> PoissonScene:
    """Liquid = {y < slab_height} U spheres inside the unit box at n^3 voxels;
    face velocities U[-1,1] from ``seed``; walls solid."""
    dx = 1.0 / n
    c = ((np.arange(n, dtype=np.float64) + 0.5) * dx)
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    phi = np.full((n, n, n), np.inf, dtype=np.float64)
    if slab_height is not None:
        phi = np.minimum(phi, Y - slab_height)
    for cen, r in spheres:
        phi = np.minimum(phi, np.sqrt((X - cen[0]) ** 2 + (Y - cen[1]) ** 2 + (Z - cen[2]) ** 2) - r)
    phi = np.minimum(phi, 3.0 * 4 * n * dx)  # finite everywhere
    bg = 3.0 * dx
    phi_g = dense_to_leaves(phi.astype(np.float32), background=bg)
    fw_g = dense_to_leaves(_walls_face_weights(n), background=np.ones(3, np.float32))
    m = n + 1
    vel = uniform(seed, 3 * m * m * m, -1.0, 1.0).reshape(3, m, m, m)
    vx = dense_to_leaves(vel[0], background=0.0)
    vy = dense_to_leaves(vel[1], background=0.0)
    vz = dense_to_leaves(vel[2], background=0.0)
    sv = LeafGrid(origins=np.zeros((0, 3), np.int32), values=np.zeros((0, 512, 3), np.float32),
                  background=np.zeros(3, np.float32))
    return PoissonScene(name=name, n=n, dx=dx, dt=dt, phi=phi_g, face_weights=fw_g,
                        vx=vx, vy=vy, vz=vz, solid_velocity=sv)


def plain_poisson_scene(n: int = 128, seed: int = 0) -> PoissonScene:
    """Plain Poisson projection workload: n^3 (128^3), dx = 1/n, liquid = y < 0.4
    plus a sphere of radius 0.15 at (0.5, 0.7, 0.5), walls solid, face
    velocities U[-1,1] from seed 0, dt = 1."""
    return sdf_box_scene(n, 0.4, [((0.5, 0.7, 0.5), 0.15)], seed, 1.0,
                         name=f"slab0.4+sphere0.15 {n}^3 seed{seed}")


def large_poisson_scene(n: int = 512, seed: int = 2) -> PoissonScene:
    """512^3: liquid = y < 0.45 plus 4 spheres of radius 0.1 (centres from seed)."""
    u = uniform(seed + 1000, 12, 0.15, 0.85).reshape(4, 3)
    spheres = [((float(a), float(b) * 0.4 + 0.5, float(c)), 0.1) for a, b, c in u]
    return sdf_box_scene(n, 0.45, spheres, seed, 1.0, name=f"slab0.45+4spheres {n}^3 seed{seed}")


def random_balls_scene(seed: int, sides=(32, 64, 96, 128, 192)) -> PoissonScene:
    """Batched-Poisson instance ``seed``: a cubic box whose side is drawn from
    ``sides``, 1-6 spheres with radii log-uniform in [0.05, 0.3] (box units)
    and centres uniform in the box, walls solid."""
    u = uniform(seed + 7919, 32, 0.0, 1.0).astype(np.float64)
    n = int(sides[min(int(u[0] * len(sides)), len(sides) - 1)])
    k = 1 + min(int(u[1] * 6), 5)
    spheres = []
    for s in range(k):
        r = float(np.exp(np.log(0.05) + (np.log(0.3) - np.log(0.05)) * u[2 + 4 * s]))
        spheres.append(((float(u[3 + 4 * s]), float(u[4 + 4 * s]), float(u[5 + 4 * s])), r))
    return sdf_box_scene(n, None, spheres, seed, 1.0, name=f"balls{k} {n}^3 seed{seed}")


@dataclass
class ViscosityScene:
    name: str
    n: int
    dx: float
    dt: float
    rho: float
    liquid_phi: LeafGrid
    solid_phi: LeafGrid
    viscosity: LeafGrid
    u: LeafGrid
    v: LeafGrid
    w: LeafGrid
    solid_velocity: LeafGrid


def viscosity_box_scene(n: int, slab_height: float | None, spheres, seed: int, mu: float = 1e3,
                        dt: float = 1.0 / 240.0, rho: float = 1.0, name: str = "viscosity") -> ViscosityScene:
    """Viscosity inputs in the convention of simd_viscosity3d's call site
    (FLIP_vdb.cpp:3170-3204): every grid shares one index space, voxel i of
    the n^3 box centred at world (i + 1/2) dx.

    * liquid SDF: {y < slab_height} U spheres, all n^3 voxels active,
      background 3 dx (air);
    * solid SDF on the box plus one leaf of margin: distance to the nearest
      domain wall minus dx/4, so that the faces on the walls sample < 0 (solid,
      like the Poisson workload's zero wall fractions) and the first interior
      faces do not; background -3 dx (solid);
    * constant dynamic viscosity ``mu`` (a grid with no leaves);
    * face velocities U[-1, 1] from ``seed`` on the (n+1)^3 face lattice of
      each channel, zero solid velocity."""
    dx = 1.0 / n
    c = (np.arange(n, dtype=np.float64) + 0.5) * dx
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    phi = np.full((n, n, n), np.inf, dtype=np.float64)
    if slab_height is not None:
        phi = np.minimum(phi, Y - slab_height)
    for cen, r in spheres:
        phi = np.minimum(phi, np.sqrt((X - cen[0]) ** 2 + (Y - cen[1]) ** 2 + (Z - cen[2]) ** 2) - r)
    phi = np.minimum(phi, 3.0 * 4 * n * dx)
    liquid = dense_to_leaves(phi.astype(np.float32), background=3.0 * dx)
    m = n + 16
    cs = (np.arange(m, dtype=np.float64) - 8 + 0.5) * dx
    SX, SY, SZ = np.meshgrid(cs, cs, cs, indexing="ij")
    wall = np.minimum.reduce([SX, 1.0 - SX, SY, 1.0 - SY, SZ, 1.0 - SZ]) - 0.25 * dx
    solid = dense_to_leaves(wall.astype(np.float32), origin=(-8, -8, -8), background=-3.0 * dx)
    visc = LeafGrid(origins=np.zeros((0, 3), np.int32), values=np.zeros((0, 512), np.float32),
                    background=np.float32(mu))
    f = n + 1
    vel = uniform(seed, 3 * f * f * f, -1.0, 1.0).reshape(3, f, f, f)
    u = dense_to_leaves(vel[0], background=0.0)
    v = dense_to_leaves(vel[1], background=0.0)
    w = dense_to_leaves(vel[2], background=0.0)
    sv = LeafGrid(origins=np.zeros((0, 3), np.int32), values=np.zeros((0, 512, 3), np.float32),
                  background=np.zeros(3, np.float32))
    return ViscosityScene(name=name, n=n, dx=dx, dt=dt, rho=rho, liquid_phi=liquid, solid_phi=solid,
                          viscosity=visc, u=u, v=v, w=w, solid_velocity=sv)


def plain_viscosity_scene(n: int = 128, seed: int = 1, mu: float = 1e3) -> ViscosityScene:
    """Plain variational viscosity workload: the Poisson geometry at n^3
    (128^3; liquid y < 0.4 plus a sphere of radius 0.15 at (0.5, 0.7, 0.5)),
    walls solid, face velocities U[-1,1] from seed 1, mu = 1e3, dt = 1/240,
    rho = 1."""
    return viscosity_box_scene(n, 0.4, [((0.5, 0.7, 0.5), 0.15)], seed, mu,
                               name=f"slab0.4+sphere0.15 {n}^3 mu{mu:g} seed{seed}")


# ---------------------------------------------------------------------------
# Device-side scene construction (served request stream).  Large requests
# (up to 384^3 voxels) are built directly in HBM with torch: the leaf values
# live on the device (values_on_device = 1 at the C ABI), origins and masks
# on the host.

def served_side(seed: int, lo: int = 48, hi: int = 384) -> int:
    """Domain side log-uniform in [lo, hi] voxels (rounded to a multiple of 8)."""
    u = float(uniform(seed + 104729, 1, 0.0, 1.0)[0])
    s = float(np.exp(np.log(lo) + (np.log(hi) - np.log(lo)) * u))
    return int(max(lo, min(hi, 8 * round(s / 8))))


def balls_spheres(seed: int):
    """1-6 spheres, radii log-uniform in [0.05, 0.3] and centres uniform in the
    unit box (the geometry of random_balls_scene, box units)."""
    u = uniform(seed + 7919, 32, 0.0, 1.0).astype(np.float64)
    k = 1 + min(int(u[1] * 6), 5)
    out = []
    for s in range(k):
        r = float(np.exp(np.log(0.05) + (np.log(0.3) - np.log(0.05)) * u[2 + 4 * s]))
        out.append(((float(u[3 + 4 * s]), float(u[4 + 4 * s]), float(u[5 + 4 * s])), r))
    return out


def _device_leaf_grid(dense, origin: int, background, components: int) -> LeafGrid:
    """A dense torch CUDA array [X, Y, Z(, C)] with X, Y, Z multiples of 8 and
    voxel (0,0,0) at index ``origin`` (all three axes) cut into 8^3 leaves in
    the order of dense_to_leaves; all voxels active (masks None)."""
    X, Y, Z = dense.shape[:3]
    nx, ny, nz = X // 8, Y // 8, Z // 8
    if components == 1:
        vals = dense.reshape(nx, 8, ny, 8, nz, 8).permute(0, 2, 4, 1, 3, 5).reshape(-1, LEAF)
    else:
        vals = dense.reshape(nx, 8, ny, 8, nz, 8, components).permute(0, 2, 4, 1, 3, 5, 6).reshape(
            -1, LEAF, components)
    org = _leaf_origins(nx, ny, nz, origin)
    g = LeafGrid(origins=np.zeros((0, 3), np.int32),
                 values=np.zeros((0, LEAF) if components == 1 else (0, LEAF, components), np.float32),
                 background=background)
    g.origins = org
    g.masks = None  # all voxels active (nothing to upload)
    g.values = vals.contiguous()
    return g


LEAF = 512


@functools.lru_cache(maxsize=64)
def _leaf_origins(nx: int, ny: int, nz: int, origin: int) -> np.ndarray:
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    org = (np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1) * 8 + origin).astype(np.int32)
    org.setflags(write=False)
    return org


def _device_sdf(n: int, spheres, device, slab_height=None):
    import torch
    c = (torch.arange(n, device=device, dtype=torch.float64) + 0.5) / n
    X, Y, Z = c.view(n, 1, 1), c.view(1, n, 1), c.view(1, 1, n)
    phi = torch.full((n, n, n), float("inf"), device=device, dtype=torch.float64)
    if slab_height is not None:
        phi = torch.minimum(phi, (Y - slab_height).expand(n, n, n))
    for cen, r in spheres:
        phi = torch.minimum(phi, torch.sqrt((X - cen[0]) ** 2 + (Y - cen[1]) ** 2 + (Z - cen[2]) ** 2) - r)
    return torch.clamp(phi, max=3.0 * 4).to(torch.float32)


def device_face_velocities(n: int, seed: int, device):
    """Three face-velocity channels U[-1,1] on the (n+1)^3 face lattice (zero
    padding up to the next leaf), from a torch generator seeded with ``seed``."""
    import torch
    m = n + 8
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed) & 0x7FFFFFFFFFFFFFFF)
    out = []
    for _ in range(3):
        v = torch.zeros((m, m, m), device=device, dtype=torch.float32)
        v[: n + 1, : n + 1, : n + 1] = torch.rand((n + 1, n + 1, n + 1), generator=gen, device=device) * 2 - 1
        out.append(_device_leaf_grid(v, 0, 0.0, 1))
    return out


def device_poisson_instance(n: int, seed: int, device):
    """Pressure inputs of a served request built in HBM: liquid = union of the
    seeded spheres in an n^3 box (dx = 1/n, dt = 1), walls solid.  Returns
    (phi, face_weights, solid_velocity, dt, dx)."""
    import torch
    assert n % 8 == 0
    dx = 1.0 / n
    phi = _device_sdf(n, balls_spheres(seed), device)
    m = n + 8
    w = torch.ones((m, m, m, 3), device=device, dtype=torch.float32)
    f = n + 1  # the face lattice; the padding beyond it keeps the background 1
    w[0, :f, :f, 0] = 0.0; w[n, :f, :f, 0] = 0.0
    w[:f, 0, :f, 1] = 0.0; w[:f, n, :f, 1] = 0.0
    w[:f, :f, 0, 2] = 0.0; w[:f, :f, n, 2] = 0.0
    phi_g = _device_leaf_grid(phi, 0, np.float32(3.0 * dx), 1)
    fw_g = _device_leaf_grid(w, 0, np.ones(3, np.float32), 3)
    sv = LeafGrid(origins=np.zeros((0, 3), np.int32), values=np.zeros((0, 512, 3), np.float32),
                  background=np.zeros(3, np.float32))
    return phi_g, fw_g, sv, 1.0, dx


def device_viscosity_instance(n: int, seed: int, device, mu: float = 1e3, dt: float = 1.0 / 240.0,
                              rho: float = 1.0):
    """Viscosity inputs of a served request built in HBM, in the convention of
    viscosity_box_scene: liquid SDF (bg 3 dx), solid SDF on the box plus one
    leaf of margin (nearest wall distance - dx/4, bg -3 dx), constant mu.
    Returns (liquid_phi, solid_phi, viscosity, solid_velocity, dt, rho, dx)."""
    import torch
    assert n % 8 == 0
    dx = 1.0 / n
    phi = _device_sdf(n, balls_spheres(seed), device)
    m = n + 16
    cs = (torch.arange(m, device=device, dtype=torch.float64) - 8 + 0.5) * dx
    SX, SY, SZ = cs.view(m, 1, 1), cs.view(1, m, 1), cs.view(1, 1, m)
    wall = torch.minimum(torch.minimum(torch.minimum(SX, 1.0 - SX), torch.minimum(SY, 1.0 - SY)),
                         torch.minimum(SZ, 1.0 - SZ)) - 0.25 * dx
    liquid = _device_leaf_grid(phi, 0, np.float32(3.0 * dx), 1)
    solid = _device_leaf_grid(wall.to(torch.float32).contiguous(), -8, np.float32(-3.0 * dx), 1)
    visc = LeafGrid(origins=np.zeros((0, 3), np.int32), values=np.zeros((0, 512), np.float32),
                    background=np.float32(mu))
    sv = LeafGrid(origins=np.zeros((0, 3), np.int32), values=np.zeros((0, 512, 3), np.float32),
                  background=np.zeros(3, np.float32))
    return liquid, solid, visc, sv, dt, rho, dx


def device_large_poisson(n: int = 512, seed: int = 2, device="cuda"):
    """Mixed-precision workload built in HBM: n^3 (512^3), dx = 1/n, liquid =
    {y < 0.45} U 4 spheres of radius 0.1 (centres from ``seed``, as
    large_poisson_scene), walls solid, face velocities U[-1,1] (seed), dt = 1.
    Returns (phi, face_weights, vx, vy, vz, solid_velocity, dt, dx)."""
    import torch
    assert n % 8 == 0
    u = uniform(seed + 1000, 12, 0.15, 0.85).reshape(4, 3)
    spheres = [((float(a), float(b) * 0.4 + 0.5, float(c)), 0.1) for a, b, c in u]
    dx = 1.0 / n
    phi = _device_sdf(n, spheres, device, slab_height=0.45)
    m = n + 8
    w = torch.ones((m, m, m, 3), device=device, dtype=torch.float32)
    f = n + 1
    w[0, :f, :f, 0] = 0.0; w[n, :f, :f, 0] = 0.0
    w[:f, 0, :f, 1] = 0.0; w[:f, n, :f, 1] = 0.0
    w[:f, :f, 0, 2] = 0.0; w[:f, :f, n, 2] = 0.0
    phi_g = _device_leaf_grid(phi, 0, np.float32(3.0 * dx), 1)
    del phi
    fw_g = _device_leaf_grid(w, 0, np.ones(3, np.float32), 3)
    del w
    vx, vy, vz = device_face_velocities(n, seed, device)
    sv = LeafGrid(origins=np.zeros((0, 3), np.int32), values=np.zeros((0, 512, 3), np.float32),
                  background=np.zeros(3, np.float32))
    return phi_g, fw_g, vx, vy, vz, sv, 1.0, dx
