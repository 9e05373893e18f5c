"""Seeded synthetic workloads with the shapes of the reference's configurations.

* :func:`taylor_green` — triply periodic Taylor-Green vortex (D3Q19 BGK), the
  velocity field u0*(sin x cos y cos z, -cos x sin y cos z, 0) at cell centres
  x = 2*pi*(i+1/2)/N plus seeded uniform noise, rho = 1, equilibrium
  populations (as examples/turbulence/tgv3d/tgv3d.cpp sets it up, with
  setPeriodicity({true,true,true}) at :550).
* :func:`cavity` — lid-driven cavity geometry as cavity3dBenchmark builds it
  (examples/laminar/cavity3dBenchmark/cavity3d.cpp:40-59): bounce-back walls on
  the box surface, a moving lid on the y = max face.
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


__all__ = ["taylor_green", "tgv_velocity", "tgv_energy", "tgv_energy_decay", "cavity", "D3Q19"]
