"""Seeded synthetic workloads with the shapes of the reference's configurations.

* :func:`taylor_green` — triply periodic Taylor-Green vortex (D3Q19 BGK), the
  velocity field u0*(sin x cos y cos z, -cos x sin y cos z, 0) at cell centres
  x = 2*pi*(i+1/2)/N plus seeded uniform noise, rho = 1, equilibrium
  populations (as examples/turbulence/tgv3d/tgv3d.cpp sets it up, with
  setPeriodicity({true,true,true}) at :550).
* :func:`cavity` — lid-driven cavity geometry as cavity3dBenchmark builds it
  (examples/laminar/cavity3dBenchmark/cavity3d.cpp:40-59): bounce-back walls on
  the box surface, a moving lid on the y = max face.
* :func:`porous_spheres` — x-periodic channel with bounce-back walls at the y/z
  faces and seeded non-overlapping spheres up to a solid fraction.
* :func:`square_cylinder_channel` — channel with bounce-back y/z walls, an inlet
  plane at x = 0, an outlet plane at x = nx-1 and a square cylinder spanning z.
"""
from __future__ import annotations

import numpy as np

from .descriptors import D3Q19, descriptor


def tgv_velocity(n: int, u0: float = 0.05, noise: float = 1e-4, seed: int = 0,
                 dtype=np.float32) -> np.ndarray:
    """Velocity field of the TGV on an n^3 box, shape (3, n^3), z fastest."""
    x = (np.arange(n, dtype=np.float64) + 0.5) * (2.0 * np.pi / n)
    sx, cx = np.sin(x), np.cos(x)
    rng = np.random.default_rng(seed)
    u = np.empty((3, n, n, n), dtype=dtype)
    u[0] = (u0 * sx[:, None, None] * cx[None, :, None] * cx[None, None, :]).astype(dtype)
    u[1] = (-u0 * cx[:, None, None] * sx[None, :, None] * cx[None, None, :]).astype(dtype)
    u[2] = 0
    if noise:
        for d in range(3):
            u[d] += rng.uniform(-noise, noise, size=(n, n, n)).astype(dtype)
    return u.reshape(3, -1)


def taylor_green(n: int, u0: float = 0.05, nu: float = 0.0125, noise: float = 1e-4, seed: int = 0,
                 dtype=np.float32, lattice="D3Q19"):
    """Returns (omega, populations (q, n^3)) of the TGV workload."""
    desc = descriptor(lattice)
    u = tgv_velocity(n, u0, noise, seed, dtype)
    rho = np.ones(n ** 3, dtype=dtype)
    # equilibrium in slabs to bound host memory for large n
    pops = np.empty((desc.q, n ** 3), dtype=dtype)
    slab = n * n * max(1, (1 << 22) // (n * n))
    for s in range(0, n ** 3, slab):
        e = min(n ** 3, s + slab)
        pops[:, s:e] = desc.equilibrium(rho[s:e], u[:, s:e], dtype)
    tau = 0.5 + 3.0 * nu
    return 1.0 / tau, pops


def tgv_energy(u: np.ndarray) -> float:
    """Mean kinetic energy 1/2 <|u|^2>."""
    u = u.reshape(3, -1).astype(np.float64)
    return 0.5 * float(np.mean(np.sum(u * u, axis=0)))


def tgv_energy_decay(t: float, n: int, nu: float) -> float:
    """Linear-limit decay factor E(t)/E(0) = exp(-2*nu*|k|^2*t), |k|^2 = 3*(2*pi/n)^2."""
    k2 = 3.0 * (2.0 * np.pi / n) ** 2
    return float(np.exp(-2.0 * nu * k2 * t))


def cavity(size):
    """Per-cell ids for a lid-driven cavity: 0 fluid, 1 wall, 2 lid."""
    nx, ny, nz = size
    ids = np.zeros((nx, ny, nz), np.uint8)
    ids[0, :, :] = 1
    ids[-1, :, :] = 1
    ids[:, 0, :] = 1
    ids[:, :, 0] = 1
    ids[:, :, -1] = 1
    ids[1:-1, -1, 1:-1] = 2
    return ids.reshape(-1)


def porous_spheres(size, r_range=(6.0, 14.0), solid_fraction=0.35, seed: int = 0, max_tries: int = 400000):
    """Per-cell ids (0 fluid, 1 solid) of an x-periodic channel: bounce-back
    walls on the y/z faces and spheres of radius uniform in r_range, centres
    uniform in the box (periodic in x), overlaps rejected, added until the
    solid fraction reaches ``solid_fraction`` (or ``max_tries`` candidates).
    Returns (ids, number of spheres, solid fraction)."""
    nx, ny, nz = size
    solid = np.zeros(size, bool)
    solid[:, 0, :] = solid[:, -1, :] = True
    solid[:, :, 0] = solid[:, :, -1] = True
    rng = np.random.default_rng(seed)
    centres = np.zeros((0, 3))
    radii = np.zeros(0)
    count = int(solid.sum())
    target = solid_fraction * solid.size
    tries = 0
    while count < target and tries < max_tries:
        tries += 1
        r = rng.uniform(*r_range)
        c = rng.uniform([0.0, 1.0 + r, 1.0 + r], [nx, ny - 1.0 - r, nz - 1.0 - r])
        if len(radii):
            d = np.abs(centres - c)
            d[:, 0] = np.minimum(d[:, 0], nx - d[:, 0])
            if np.any(np.sum(d * d, axis=1) < (radii + r) ** 2):
                continue
        centres = np.vstack([centres, c])
        radii = np.append(radii, r)
        lo = np.floor(c - r).astype(int)
        hi = np.ceil(c + r).astype(int) + 1
        xs = np.arange(lo[0], hi[0])
        ys = np.arange(max(lo[1], 0), min(hi[1], ny))
        zs = np.arange(max(lo[2], 0), min(hi[2], nz))
        X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
        inside = (X + 0.5 - c[0]) ** 2 + (Y + 0.5 - c[1]) ** 2 + (Z + 0.5 - c[2]) ** 2 <= r * r
        xi = np.mod(X[inside], nx)
        block = solid[xi, Y[inside], Z[inside]]
        count += int((~block).sum())
        solid[xi, Y[inside], Z[inside]] = True
    return solid.astype(np.uint8).reshape(-1), len(radii), count / solid.size


def square_cylinder_channel(size, side: int = 32, x_centre: float | None = None):
    """Per-cell ids of a channel: 0 fluid, 1 bounce-back (y/z walls and a
    side x side square cylinder spanning z between the walls), 2 inlet plane
    (x = 0, interior y/z), 3 outlet plane (x = nx-1, interior y/z)."""
    nx, ny, nz = size
    ids = np.zeros(size, np.uint8)
    ids[:, 0, :] = ids[:, -1, :] = 1
    ids[:, :, 0] = ids[:, :, -1] = 1
    ids[0, 1:-1, 1:-1] = 2
    ids[-1, 1:-1, 1:-1] = 3
    xc = nx / 4 if x_centre is None else x_centre
    x0, y0 = int(round(xc - side / 2)), ny // 2 - side // 2
    ids[x0:x0 + side, y0:y0 + side, 1:-1] = 1
    return ids.reshape(-1)


__all__ = ["taylor_green", "tgv_velocity", "tgv_energy", "tgv_energy_decay", "cavity", "porous_spheres",
           "square_cylinder_channel", "D3Q19"]
