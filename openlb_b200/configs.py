"""Full-size runs of the reference's configurations on one GPU, with reports.

    python -m openlb_b200.configs c2 [--steps 5000]
    python -m openlb_b200.configs c3 [--max-steps 50000]
    python -m openlb_b200.configs c4 [--steps 20000]

Each prints one JSON line.  The FP64 comparison run at full size is this
library's exact build in FP64 (``variant="exact"``: ``-fmad=false``, the
reference's operation order); the GPU tests show that build bit-identical to
the CPU restatement of the reference, which is itself pinned to OpenLB's own
CPU build, so it stands in for the FP64 oracle at sizes the CPU cannot run.

* c2 — Taylor-Green vortex, 256^3 periodic, D3Q19 BGK, nu = 0.0125, u0 = 0.05,
  seeded +-1e-4 noise, 5000 steps: MLUPS per storage type, kinetic energy
  against the linear-limit decay, velocity L2 of FP32 / FP16 / BF16 against FP64.
* c3 — porous channel 384x192x192, D3Q19 forced TRT (magic 3/16), g = 1e-6,
  x periodic, bounce-back y/z walls and spheres of radius U[6,14] up to 35 %
  solid; runs to a velocity-change residual < 1e-7 (checked every 1000 steps)
  or the step limit: velocity L2 and permeability error of FP16 / FP32 storage
  against FP64.
* c4 — square-cylinder channel 512x256x256, D3Q27 Smagorinsky-BGK (Cs = 0.1),
  interpolated velocity inlet u = 0.05 with 2 % per-step fluctuations
  (olb_b200_set_boundary_noise), interpolated pressure outlet, bounce-back
  walls and a 32x32 cylinder spanning z: MLUPS against the roofline and the
  time-averaged velocity error of BF16 / FP16 storage against FP64.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import _abi
from .descriptors import descriptor
from .lattice import (BounceBack, Dynamics, ForcedTRTdynamics, InterpolatedPressureBoundary,
                      InterpolatedVelocityBoundary, Lattice, SmagorinskyBGKdynamics)
from .workloads import porous_spheres, square_cylinder_channel, taylor_green, tgv_energy, tgv_energy_decay

BYTES = {"f32": 4, "f64": 8, "f16": 2, "bf16": 2}


def peak_gbs() -> float:
    from .tune import peak_gbs as p
    return p()


def _l2(a: np.ndarray, b: np.ndarray, sel=None) -> float:
    a = a.reshape(3, -1).astype(np.float64)
    b = b.reshape(3, -1).astype(np.float64)
    if sel is not None:
        a, b = a[:, sel], b[:, sel]
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _mlups(cells: int, steps: int, ms: float) -> float:
    return cells * steps / (ms * 1e-3) / 1e6


def c2(steps: int = 5000, n: int = 256, chunk: int = 500) -> dict:
    nu, u0 = 0.0125, 0.05
    cells = n ** 3
    out = {"config": "c2_tgv", "size": [n, n, n], "steps": steps, "nu": nu, "u0": u0, "runs": {}}
    fields = {}
    for name, storage, variant in (("f64", "f64", "exact"), ("f32", "f32", "fast"), ("f32_reference_order", "f32", "exact"),
                                   ("f16", "f16", "fast"), ("bf16", "bf16", "fast")):
        dtype = np.float64 if storage == "f64" else np.float32
        omega, pops = taylor_green(n, u0=u0, nu=nu, dtype=dtype)
        lat = Lattice(19, (n, n, n), (True, True, True), storage=storage, variant=variant)
        try:
            lat.set_dynamics([Dynamics(_abi.DYN_BGK, omega=omega)])
            lat.set_populations(pops)
            del pops
            e0 = tgv_energy(lat.get_moments()[1])
            ms, energy, done = 0.0, [], 0
            while done < steps:
                k = min(chunk, steps - done)
                ms += lat.time_steps(k)
                done += k
                energy.append((done, tgv_energy(lat.get_moments()[1]) / e0))
            fields[name] = lat.get_moments()[1].astype(np.float64)
        finally:
            lat.close()
        bpc = 2 * 19 * BYTES[storage]
        mlups = _mlups(cells, steps, ms)
        out["runs"][name] = {
            "build": variant, "mlups": round(mlups, 1),
            "roofline_frac": round(mlups * 1e6 * bpc / 1e9 / peak_gbs(), 4),
            "energy_ratio_end": energy[-1][1], "energy_ratio_linear_theory": tgv_energy_decay(steps, n, nu),
            "energy_curve": energy,
        }
    for name in ("f32", "f32_reference_order", "f16", "bf16"):
        out["runs"][name]["u_l2_vs_f64"] = _l2(fields[name], fields["f64"])
    return out


def _forced_trt_lattice(size, ids, storage, variant, omega, g):
    lat = Lattice(19, size, (True, False, False), storage=storage, variant=variant)
    lat.set_dynamics([ForcedTRTdynamics(omega=omega, magic=3 / 16, force=(g, 0.0, 0.0)), BounceBack()], ids)
    return lat


def c3(max_steps: int = 50000, size=(384, 192, 192), tol: float = 1e-7, check: int = 1000, seed: int = 3,
       storages=("f64", "f32", "f16"), r_range=(6.0, 14.0)) -> dict:
    tau, g = 0.8, 1e-6
    omega, nu = 1.0 / tau, (tau - 0.5) / 3.0
    ids, n_spheres, frac = porous_spheres(size, r_range=r_range, seed=seed)
    cells = int(np.prod(size))
    fluid = ids == 0
    out = {"config": "c3_porous", "size": list(size), "spheres": n_spheres, "solid_fraction": frac,
           "tau": tau, "g": g, "tol": tol, "check_interval": check, "runs": {}}
    fields = {}
    for storage in storages:
        variant = "exact" if storage == "f64" else "fast"
        dtype = np.float64 if storage == "f64" else np.float32
        lat = _forced_trt_lattice(size, ids, storage, variant, omega, g)
        try:
            lat.set_populations(np.zeros(19 * cells, dtype))
            lat.velocity_residual()
            ms, steps, res = 0.0, 0, math.inf
            while steps < max_steps:
                ms += lat.time_steps(check)
                steps += check
                res = lat.velocity_residual()
                if res < tol:
                    break
            u = lat.get_moments()[1].astype(np.float64)
        finally:
            lat.close()
        fields[storage] = u
        mean_ux = float(u[0].sum() / cells)            # superficial (Darcy) velocity
        bpc = 2 * 19 * BYTES[storage]
        mlups = _mlups(cells, steps, ms)
        out["runs"][storage] = {"build": variant, "steps": steps, "residual": res, "mlups": round(mlups, 1),
                                "roofline_frac": round(mlups * 1e6 * bpc / 1e9 / peak_gbs(), 4),
                                "permeability": nu * mean_ux / g}
    k64 = out["runs"]["f64"]["permeability"]
    for storage in storages:
        if storage == "f64":
            continue
        out["runs"][storage]["u_l2_vs_f64"] = _l2(fields[storage], fields["f64"], fluid)
        out["runs"][storage]["permeability_rel_err"] = abs(out["runs"][storage]["permeability"] - k64) / k64
    return out


def c4(steps: int = 20000, size=(512, 256, 256), side: int = 32, u_in: float = 0.05, re: float = 1000.0,
       noise: float = 0.02, seed: int = 11, sample: int = 100,
       storages=("f64", "f64_other_seed", "bf16", "f16")) -> dict:
    nx, ny, nz = size
    cells = nx * ny * nz
    nu = u_in * side / re
    omega = 1.0 / (3.0 * nu + 0.5)
    ids = square_cylinder_channel(size, side)
    mix = SmagorinskyBGKdynamics(omega=omega, smagorinsky=0.1)
    table = [mix, BounceBack(), InterpolatedVelocityBoundary(mix, 0, -1), InterpolatedPressureBoundary(mix, 0, 1)]
    inlet = np.flatnonzero(ids == 2)
    outlet = np.flatnonzero(ids == 3)
    values = np.zeros((len(inlet) + len(outlet), 4))
    values[:, 0] = 1.0
    values[:len(inlet), 1] = u_in
    bcells = np.concatenate([inlet, outlet])
    fluid = ids == 0
    desc = descriptor(27)
    out = {"config": "c4_square_cylinder", "size": list(size), "cylinder": side, "re": re, "nu": nu,
           "omega": omega, "smagorinsky": 0.1, "inlet_u": u_in, "inlet_noise": noise, "steps": steps,
           "average_over_last": steps // 2, "sample_interval": sample, "runs": {}}
    means = {}
    for name in storages:
        # "f64_other_seed": FP64 with another fluctuation seed, the spread of the
        # time averages between two equally valid runs
        storage = "f64" if name.startswith("f64") else name
        variant = "exact" if storage == "f64" else "fast"
        dtype = np.float64 if storage == "f64" else np.float32
        lat = Lattice(27, size, (False, False, False), storage=storage, variant=variant)
        try:
            lat.set_dynamics(table, ids)
            lat.set_boundary_values(bcells, values)
            lat.set_boundary_noise(noise, seed + 1 if name == "f64_other_seed" else seed)
            # uniform flow u_in everywhere (rest in the walls), equilibrium populations
            feq = desc.equilibrium(np.ones(1, dtype), np.array([[u_in], [0.0], [0.0]], dtype), dtype)[:, 0]
            pops = np.empty((27, cells), dtype)
            pops[:] = feq[:, None]
            pops[:, ids == 1] = 0
            lat.set_populations(pops)
            del pops
            ms, done, acc, count = 0.0, 0, None, 0
            while done < steps:
                k = min(sample, steps - done)
                ms += lat.time_steps(k)
                done += k
                if done > steps - steps // 2:
                    u = lat.get_moments()[1]
                    acc = u.astype(np.float64) if acc is None else acc + u
                    count += 1
            means[name] = acc / count
        finally:
            lat.close()
        bpc = 2 * 27 * BYTES[storage]
        mlups = _mlups(cells, steps, ms)
        out["runs"][name] = {"build": variant, "mlups": round(mlups, 1),
                             "roofline_frac": round(mlups * 1e6 * bpc / 1e9 / peak_gbs(), 4),
                             "samples": count, "mean_ux_fluid": float(means[name][0, fluid].mean())}
    for name in storages:
        if name != "f64":
            out["runs"][name]["time_avg_u_l2_vs_f64"] = _l2(means[name], means["f64"], fluid)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=["c2", "c3", "c4"])
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--max-steps", type=int, default=50000)
    ap.add_argument("--n", type=int, default=None, help="scale the domain: c2 side, c3/c4 nx (others in proportion)")
    args = ap.parse_args(argv)
    t0 = time.time()
    if args.config == "c2":
        out = c2(steps=args.steps or 5000, n=args.n or 256)
    elif args.config == "c3":
        size = (384, 192, 192) if not args.n else (args.n, args.n // 2, args.n // 2)
        scale = size[0] / 384
        out = c3(max_steps=args.max_steps, size=size, r_range=(6.0 * scale, 14.0 * scale))
    else:
        size = (512, 256, 256) if not args.n else (args.n, args.n // 2, args.n // 2)
        side = 32 if not args.n else max(4, args.n // 16)
        out = c4(steps=args.steps or 20000, size=size, side=side)
    out["wall_s"] = round(time.time() - t0, 1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
