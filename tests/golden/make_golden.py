#!/usr/bin/env python3
"""Generates the golden fixtures in this directory by running OpenLB itself.

Each fixture is the output of the reference's own CPU_SISD build
(oracle/_ref/olb_ref_sisd_*, built by oracle/ref/Makefile from the reference
sources with OpenLB's public API) on a small seeded case: the inputs (geometry
ids, dynamics table, initial populations) and the reference's populations,
Density3D / Velocity3D fields and per-step LatticeStatistics after the stated
number of collideAndStream steps (after the lattice's initialize(), which
applies the PostStream post-processors once to the initial state).

    python tests/golden/make_golden.py [prefix]   # needs oracle/_ref (make -C oracle/ref)

The checkpoint_* fixtures hold a file OpenLB saved (SuperLattice::save), the
populations it dumped for the same state, this library's file for that state
and OpenLB's run resumed from this library's file (SuperLattice::load), which
the generator checks against OpenLB's uninterrupted run bit for bit.

The C oracle is pinned against these fixtures in tests/test_oracle_golden.py.
"""
from __future__ import annotations

import hashlib
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from openlb_b200 import checkpoint as CK  # noqa: E402
from tests import cases as C  # noqa: E402


def fixture_cases():
    rng = np.random.default_rng(20261203)
    out = []
    # periodic boxes, every collision, random near-equilibrium state
    for q in (19, 27):
        for dtype in (np.float32, np.float64):
            for kind in (O.BGK, O.TRT, O.SMAGORINSKY, O.FORCED_TRT):
                case = C.periodic_case(q, (7, 6, 5), kind=kind)
                f0 = C.random_state(q, case.n, dtype, rng)
                variants = ["sisd"]
                if q == 19 and dtype == np.float32:
                    variants.append("nocse")
                for variant in variants:
                    name = f"periodic_q{q}_{np.dtype(dtype).name}_{O.KIND_NAMES[kind]}_{variant}"
                    out.append((name, case, f0, 4, dtype, variant, False))
    # lid-driven cavity: bounce-back walls, moving lid, rest start
    for q in (19, 27):
        for dtype in (np.float32, np.float64):
            case = C.cavity_case(q, (9, 8, 7))
            f0 = C.rest_state(q, case.n, dtype)
            for variant in (["sisd", "nocse"] if (q == 19 and dtype == np.float32) else ["sisd"]):
                out.append((f"cavity_q{q}_{np.dtype(dtype).name}_{variant}", case, f0, 25, dtype, variant, True))
    # porous channel: Guo-forced TRT + bounce-back spheres, x periodic
    case = C.porous_case(19, (12, 9, 8), np.random.default_rng(7), g=1e-4)
    f0 = C.rest_state(19, case.n, np.float32)
    for variant in ("sisd", "nocse"):
        out.append((f"porous_q19_float32_{variant}", case, f0, 15, np.float32, variant, True))
    # D3Q27 Smagorinsky channel with a square cylinder
    case = C.channel_cylinder_case(27, (12, 8, 6), side=2)
    n = case.n
    u = np.zeros((3, n), np.float32)
    u[0] = 0.05
    f0 = O.equilibrium(27, np.ones(n, np.float32), u)
    out.append(("channel_q27_float32_sisd", case, f0, 10, np.float32, "sisd", True))
    # interpolated velocity inlet / pressure outlet (PlaneFdBoundaryProcessor3D)
    for q, dtype, mixin, side in ((19, np.float32, O.BGK, 0), (19, np.float64, O.BGK, 2),
                                  (19, np.float64, O.TRT, 0), (27, np.float32, O.SMAGORINSKY, 2),
                                  (27, np.float64, O.SMAGORINSKY, 0)):
        case = C.interpolated_channel_case(q, (12, 8, 7), mixin=mixin, side=side, seed=q + side)
        f0 = C.rest_state(q, case.n, dtype)
        name = f"interp_channel_q{q}_{np.dtype(dtype).name}_{O.KIND_NAMES[mixin]}_sisd"
        out.append((name, case, f0, 30, dtype, "sisd", True))
    # cavity3dBenchmark's default: LocalVelocity walls and lid (flat faces,
    # external edges and corners, OuterVelocityEdge/CornerProcessor3D)
    for q, dtype, variants in ((19, np.float32, ("sisd", "nocse")), (19, np.float64, ("sisd",)),
                               (27, np.float32, ("sisd",)), (27, np.float64, ("sisd",))):
        case = C.local_velocity_cavity_case(q, (9, 8, 7))
        f0 = C.rest_state(q, case.n, dtype)
        for variant in variants:
            out.append((f"local_cavity_q{q}_{np.dtype(dtype).name}_{variant}", case, f0, 20, dtype, variant, True))
    # an interpolated velocity inlet over a whole face: its rim is external
    # edges and corners of the inlet
    for q, dtype, mixin in ((19, np.float32, O.BGK), (19, np.float64, O.BGK), (27, np.float64, O.TRT)):
        case = C.open_inlet_channel_case(q, (10, 7, 6), mixin=mixin, seed=q)
        f0 = C.rest_state(q, case.n, dtype)
        for variant in (("sisd", "nocse") if (q == 19 and dtype == np.float32) else ("sisd",)):
            name = f"open_inlet_q{q}_{np.dtype(dtype).name}_{O.KIND_NAMES[mixin]}_{variant}"
            out.append((name, case, f0, 15, dtype, variant, True))
    # a block standing in cavity3dBenchmark's cavity: its surface adds the
    # internal edges and corners of the velocity boundary (local and interpolated)
    for q, dtype, setter, variants in ((19, np.float32, O.LOCAL_VELOCITY, ("sisd", "nocse")),
                                       (19, np.float64, O.LOCAL_VELOCITY, ("sisd",)),
                                       (27, np.float64, O.LOCAL_VELOCITY, ("sisd",)),
                                       (19, np.float64, O.INTERP_VELOCITY, ("sisd",))):
        case = C.concave_cavity_case(q, (12, 11, 10), setter=setter)
        f0 = C.rest_state(q, case.n, dtype)
        tag = "local" if setter == O.LOCAL_VELOCITY else "interp"
        for variant in variants:
            out.append((f"concave_{tag}_q{q}_{np.dtype(dtype).name}_{variant}", case, f0, 20, dtype, variant, True))
    # LocalVelocity inlet and LocalPressure outlet (regularised flat faces)
    for q, dtype, mixin, side, variants in ((19, np.float32, O.BGK, 0, ("sisd", "nocse")),
                                            (19, np.float64, O.TRT, 2, ("sisd",)),
                                            (27, np.float64, O.BGK, 2, ("sisd",)),
                                            (27, np.float32, O.TRT, 0, ("sisd",))):
        case = C.local_channel_case(q, (12, 8, 7), mixin=mixin, side=side, seed=q + side)
        f0 = C.rest_state(q, case.n, dtype)
        for variant in variants:
            name = f"local_channel_q{q}_{np.dtype(dtype).name}_{O.KIND_NAMES[mixin]}_{variant}"
            out.append((name, case, f0, 30, dtype, variant, True))
    # a FORCE value per cell (setField<FORCE> cell by cell) for the Guo-forced
    # dynamics: porous channel with forced TRT, periodic D3Q27 forced BGK
    frng = np.random.default_rng(31)
    for q, dtype, variants in ((19, np.float32, ("sisd", "nocse")), (19, np.float64, ("sisd",)),
                               (27, np.float32, ("sisd",))):
        case = C.with_force_field(C.porous_case(q, (12, 9, 8), np.random.default_rng(7), g=1e-4), dtype, frng)
        f0 = C.rest_state(q, case.n, dtype)
        for variant in variants:
            out.append((f"forcefield_porous_q{q}_{np.dtype(dtype).name}_{variant}", case, f0, 15, dtype, variant,
                        True))
    case = C.with_force_field(C.periodic_case(27, (7, 6, 5), kind=O.FORCED_BGK), np.float64, frng)
    f0 = C.random_state(27, case.n, np.float64, frng)
    out.append(("forcefield_periodic_q27_float64_forced_bgk_sisd", case, f0, 4, np.float64, "sisd", True))
    return out


def checkpoint_cases():
    """(name, case, initial state, steps before the save, steps after it, dtype,
    descriptor fields) for the checkpoint fixtures."""
    rng = np.random.default_rng(99)
    out = []
    case = C.periodic_case(19, (7, 6, 5), kind=O.BGK)
    out.append(("checkpoint_periodic_q19_float32_bgk", case, C.random_state(19, case.n, np.float32, rng),
                5, 4, np.float32, ("FORCE",)))
    case = C.periodic_case(27, (6, 5, 4), kind=O.TRT)
    out.append(("checkpoint_periodic_q27_float64_trt", case, C.random_state(27, case.n, np.float64, rng),
                3, 3, np.float64, ("FORCE",)))
    case = C.cavity_case(19, (9, 8, 7))
    out.append(("checkpoint_cavity_q19_float64", case, C.rest_state(19, case.n, np.float64),
                12, 8, np.float64, ("FORCE",)))
    case = C.porous_case(19, (12, 9, 8), np.random.default_rng(7), g=1e-4)
    out.append(("checkpoint_porous_q19_float32", case, C.rest_state(19, case.n, np.float32),
                10, 6, np.float32, ("FORCE",)))
    # interpolated velocity inlet / pressure outlet: momenta fields per boundary normal
    case = C.interpolated_channel_case(19, (12, 8, 7), mixin=O.BGK, side=2, seed=5)
    out.append(("checkpoint_interp_channel_q19_float32_bgk", case, C.rest_state(19, case.n, np.float32),
                14, 10, np.float32, ("FORCE",)))
    case = C.interpolated_channel_case(27, (10, 7, 6), mixin=O.SMAGORINSKY, side=0, seed=6)
    out.append(("checkpoint_interp_channel_q27_float64_smagorinsky", case, C.rest_state(27, case.n, np.float64),
                9, 7, np.float64, ("FORCE",)))
    return out


def checkpoint_fixture(name, case, f0, steps, resume, dtype, dfields):
    """OpenLB saves after `steps`; this library's file for that state is written
    and OpenLB resumes from it for `resume` steps, which must equal OpenLB's
    own run of steps + resume."""
    fields, setup = CK.setup_fields(case.q, case.dyn_id if case.dyn_id is not None else np.zeros(case.n, np.uint8),
                                    case.table, dfields, case.bc_values)
    saved = O.run_reference(case, steps, dtype, init=f0, threads=1, save_checkpoint=True)
    arrays, overlap = CK.load_bytes(saved["checkpoint"], case.q, case.size, dtype, fields)
    if not np.array_equal(arrays["POPULATION"].reshape(-1), saved["pops"]):
        raise AssertionError(f"{name}: the file's populations differ from OpenLB's own dump")
    for k, v in setup.items():
        if not np.array_equal(v.astype(dtype), arrays[k]):
            raise AssertionError(f"{name}: field {k} of the set-up differs from OpenLB's")
    ours = CK.encode_fields(arrays, case.q, case.size, case.periodic, dtype, overlap, fields)
    resumed = O.run_reference(case, resume, dtype, init=f0, threads=1, load_checkpoint=ours)
    straight = O.run_reference(case, steps + resume, dtype, init=f0, threads=1)
    # slots fed from OpenLB's non-periodic padding (the outward slots of walls
    # on the box faces) hold what OpenLB streamed out earlier, which only
    # OpenLB's own file carries; the oracle marks them NaN and no fluid cell
    # ever reads them
    probe = np.ascontiguousarray(arrays["POPULATION"].reshape(-1)).copy()
    O.step(case, probe, resume)
    live = np.isfinite(probe)
    if not np.array_equal(resumed["pops"][live], straight["pops"][live]):
        raise AssertionError(f"{name}: OpenLB resumed from this library's file differs from its own run")
    payload = {
        "q": np.int32(case.q), "size": np.array(case.size, np.int32),
        "periodic": np.array(case.periodic, np.int32), "overlap": np.int32(overlap),
        "steps": np.int32(steps), "resume_steps": np.int32(resume),
        "dyn_id": case.dyn_id if case.dyn_id is not None else np.zeros(case.n, np.uint8),
        "table": np.array([[d.kind, d.omega, d.magic, d.smagorinsky, *d.force, *d.wall_u, d.wall_rho,
                            d.mixin, d.direction, d.orientation] for d in case.table], np.float64),
        "descriptor_fields": np.array(dfields, dtype="U24"),
        "extra_fields": np.array([f.name for f in fields if f.name != "POPULATION" and f.name not in dfields],
                                 dtype="U24"),
        "init": f0, "pops_saved": saved["pops"], "pops_resumed": resumed["pops"],
        "checkpoint_ref": np.frombuffer(saved["checkpoint"], np.uint8),
        "checkpoint_ours": np.frombuffer(ours, np.uint8),
        # the oracle restates the generic templates: bit-identical except the
        # CSE-generated D3Q19 BGK / Smagorinsky and the in-place boundary loop,
        # which agree to rounding
        "tolerance": np.float64(2e-6 if dtype == np.float32 else 1e-10),
    }
    if case.bc_values is not None:
        payload["bc_values"] = case.bc_values
    for k, v in arrays.items():
        if k != "POPULATION":
            payload[f"field_{k}"] = v
    return payload


def normals_geometries():
    """Material layouts whose boundary cells (material 3) cover flat faces,
    edges and corners; fluid is material 1, walls 2, outside 0."""
    out = []
    # channel with inlet/outlet planes bounded by walls and a square cylinder
    case = C.interpolated_channel_case(19, (12, 8, 7), side=2)
    mats = case.dyn_id.reshape(case.size).astype(np.int32) + 1
    mats[mats == 4] = 3
    out.append(("normals_channel", mats, (0, 0, 0)))
    # inlet spanning the whole x = 0 face (its rim touches the outside), x periodic
    mats = np.full((9, 8, 7), 1, np.int32)
    mats[:, 0, :] = mats[:, -1, :] = 2
    mats[0, :, :] = 3
    out.append(("normals_open_face", mats, (0, 0, 1)))
    # random fluid boxes in a wall block, boundary cells sampled next to fluid,
    # an outside pocket
    rng = np.random.default_rng(11)
    for k in range(3):
        size = (14, 12, 10)
        mats = np.full(size, 2, np.int32)
        for _ in range(4):
            lo = rng.integers(1, np.array(size) - 4)
            hi = np.minimum(lo + rng.integers(3, 7, 3), np.array(size) - 1)
            mats[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = 1
        fluid = mats == 1
        near = np.zeros(size, bool)
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    near |= np.roll(fluid, (dx, dy, dz), axis=(0, 1, 2))
        cand = near & ~fluid
        mats[cand & (rng.random(size) < 0.7)] = 3
        mats[-3:, -3:, :] = np.where(mats[-3:, -3:, :] == 1, 1, 0)
        out.append((f"normals_random{k}", mats, (0, 0, 0)))
    return out


def main(only: str | None = None):
    """Regenerates every fixture, or only those whose name starts with `only`
    (the manifest keeps the other entries)."""
    mf = HERE / "MANIFEST.json"
    manifest = json.loads(mf.read_text())["fixtures"] if (only and mf.exists()) else {}

    def wanted(name):
        return only is None or name.startswith(only)

    for name, mats, periodic in normals_geometries():
        if not wanted(name):
            continue
        ref = O.reference_normals(mats, periodic, boundary_materials=(3,))
        path = HERE / f"{name}.npz"
        np.savez_compressed(path, materials=mats, periodic=np.array(periodic, np.int32), normals=ref)
        manifest[name] = {"variant": "sisd", "dtype": "int32", "steps": 0,
                          "sha256": hashlib.sha256(path.read_bytes()).hexdigest()}
        print(name, path.stat().st_size, "types", np.unique(ref[0][ref[0] >= 0], return_counts=True))
    for name, case, f0, steps, dtype, variant, stats in fixture_cases():
        if not wanted(name):
            continue
        # one thread: the reference applies post-processors in an OpenMP loop
        # in place, so neighbouring pressure-boundary cells race otherwise
        ref = O.run_reference(case, steps, dtype, init=f0, variant=variant, stats=stats, threads=1)
        payload = {
            "q": np.int32(case.q), "size": np.array(case.size, np.int32),
            "periodic": np.array(case.periodic, np.int32), "steps": np.int32(steps),
            "dyn_id": case.dyn_id if case.dyn_id is not None else np.zeros(case.n, np.uint8),
            "table": np.array([[d.kind, d.omega, d.magic, d.smagorinsky, *d.force, *d.wall_u, d.wall_rho,
                                d.mixin, d.direction, d.orientation, *d.normal, d.boundary]
                               for d in case.table], np.float64),
            "init": f0, "pops": ref["pops"], "rho": ref["rho"], "u": ref["u"],
        }
        if stats:
            payload["stats"] = ref["stats"]
        if case.bc_values is not None:
            payload["bc_values"] = case.bc_values
        if case.force_field is not None:
            payload["force_field"] = case.force_field
        path = HERE / f"{name}.npz"
        np.savez_compressed(path, **payload)
        manifest[name] = {"variant": variant, "dtype": np.dtype(dtype).name, "steps": steps,
                          "sha256": hashlib.sha256(path.read_bytes()).hexdigest()}
        print(name, path.stat().st_size)
    for name, case, f0, steps, resume, dtype, dfields in checkpoint_cases():
        if not wanted(name):
            continue
        payload = checkpoint_fixture(name, case, f0, steps, resume, dtype, dfields)
        path = HERE / f"{name}.npz"
        np.savez_compressed(path, **payload)
        manifest[name] = {"variant": "sisd", "dtype": np.dtype(dtype).name, "steps": steps + resume,
                          "sha256": hashlib.sha256(path.read_bytes()).hexdigest()}
        print(name, path.stat().st_size)
    gxx = subprocess.run(["g++", "--version"], capture_output=True, text=True).stdout.splitlines()[0]
    (HERE / "MANIFEST.json").write_text(json.dumps(
        {"generator": "tests/golden/make_golden.py", "reference_build": "oracle/ref/Makefile",
         "compiler": gxx, "flags": "-O3 -std=c++20 -march=x86-64-v2 -ffp-contract=off -fopenmp",
         "threads": 1,
         "fixtures": manifest}, indent=1) + "\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
