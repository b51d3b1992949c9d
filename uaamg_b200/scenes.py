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
