"""Step-kernel variant sweep and autotuning report.

    python -m openlb_b200.tune [--n 256] [--steps 20] [--repeat 3]

For each lattice class (D3Q19 FP32 periodic, D3Q19 FP32 cavity with walls and
a lid, D3Q19 FP16/BF16, D3Q19 FP64, D3Q27 FP32/FP16, forced TRT and
Smagorinsky-BGK in FP32 and 16-bit storage) it times every
step-kernel variant at every launch shape with CUDA events (best of
`--repeat` runs of `--steps` steps), then runs the autotuner and prints one
JSON line per measurement and a markdown summary of the fraction of the
measured HBM copy bandwidth (MEASURED_PEAKS.json) each one reaches.
"""
from __future__ import annotations

import argparse
import json
from pathlib import Path

import numpy as np

from . import _abi
from .lattice import (BGKdynamics, BounceBack, BounceBackVelocity, ForcedTRTdynamics, Lattice,
                      SmagorinskyBGKdynamics)
from .workloads import cavity, porous_spheres

BYTES = {"f32": 4, "f64": 8, "f16": 2, "bf16": 2}
CLASSES = [
    ("D3Q19 f32", 19, "f32", False, "bgk"),
    ("D3Q19 f32 cavity", 19, "f32", True, "bgk"),
    ("D3Q19 f16", 19, "f16", False, "bgk"),
    ("D3Q19 bf16", 19, "bf16", False, "bgk"),
    ("D3Q19 f64", 19, "f64", False, "bgk"),
    ("D3Q27 f32", 27, "f32", False, "bgk"),
    ("D3Q27 f16", 27, "f16", False, "bgk"),
    ("D3Q19 f32 forced TRT", 19, "f32", False, "forced_trt"),
    ("D3Q19 f16 forced TRT", 19, "f16", False, "forced_trt"),
    ("D3Q27 f32 Smagorinsky", 27, "f32", False, "smagorinsky"),
    ("D3Q27 bf16 Smagorinsky", 27, "bf16", False, "smagorinsky"),
]


def fluid(collision: str):
    if collision == "smagorinsky":
        return SmagorinskyBGKdynamics(omega=1.9, smagorinsky=0.1)
    if collision == "forced_trt":
        return ForcedTRTdynamics(omega=1.25, magic=3 / 16, force=(1e-6, 0.0, 0.0))
    return BGKdynamics(omega=1.6)


def peak_gbs() -> float:
    p = Path(__file__).resolve().parents[1] / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def make_porous(size, storage, q=19):
    """The porous channel: x-periodic, bounce-back y/z walls and spheres of
    radius U[6,14] up to 35 % solid, forced TRT (tau 0.8, magic 3/16, g 1e-6)."""
    ids, _, _ = porous_spheres(size, seed=3)
    lat = Lattice(q, size, (True, False, False), storage=storage)
    lat.set_dynamics([ForcedTRTdynamics(omega=1 / 0.8, magic=3 / 16, force=(1e-6, 0.0, 0.0)), BounceBack()], ids)
    return lat


def make_lattice(q, n, storage, masked, collision="bgk"):
    lat = Lattice(q, (n, n, n), (not masked,) * 3, storage=storage)
    if masked:
        lat.set_dynamics([fluid(collision), BounceBack(), BounceBackVelocity((0.1, 0.0, 0.0))],
                         cavity((n, n, n)))
    else:
        lat.set_dynamics([fluid(collision)])
    return lat


def time_config(lat, steps, repeat):
    lat.collide_and_stream(4)
    lat.synchronize()
    return min(lat.time_steps(steps) for _ in range(repeat)) / steps


def run_single(args):
    """Fixed configurations: for each variant of `--variant` (comma-separated)
    and each launch shape of `--shape` (';'-separated), warm-up, then
    `--steps` steps (for profilers; one JSON line each)."""
    if args.porous:
        size = tuple(int(v) for v in args.porous.split(","))
        lat = make_porous(size, args.storage, args.lattice)
    else:
        size = (args.n,) * 3
        lat = make_lattice(args.lattice, args.n, args.storage, args.masked)
    cells = int(np.prod(size))
    bpc = 2 * args.lattice * BYTES[args.storage]
    try:
        for variant in (int(v) for v in str(args.variant).split(",")):
            for shape in args.shape.split(";"):
                lat.set_step_variant(variant)
                bz, by = (int(v) for v in shape.split(","))
                lat.set_launch_shape(bz, by)
                lat.collide_and_stream(args.warmup)
                lat.synchronize()
                ms = lat.time_steps(args.steps)
                print(json.dumps({"lattice": args.lattice, "size": list(size), "storage": args.storage,
                                  "workload": "porous" if args.porous else ("cavity" if args.masked else "periodic"),
                                  "tuning": lat.tuning(), "ms_per_step": ms / args.steps,
                                  "mlups": round(cells * args.steps / (ms * 1e-3) / 1e6),
                                  "frac": round(cells * bpc * args.steps / (ms * 1e-3) / 1e9 / peak_gbs(), 3)}),
                      flush=True)
    finally:
        lat.close()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--single", action="store_true",
                    help="run one fixed configuration (--lattice/--storage/--masked/--variant/--shape)")
    ap.add_argument("--lattice", type=int, default=19, choices=[19, 27])
    ap.add_argument("--storage", default="f32", choices=list(BYTES))
    ap.add_argument("--masked", action="store_true", help="lid-driven cavity (walls and a moving lid)")
    ap.add_argument("--porous", default="", metavar="NX,NY,NZ",
                    help="--single: the porous channel of this size instead of a cube")
    ap.add_argument("--variant", default="-1", help="--single: variant(s), comma-separated (-1: default)")
    ap.add_argument("--shape", default="128,2", help="--single: launch shape(s) bz,by; ';'-separated")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--classes", default="", help="';'-separated substrings of the class labels to run")
    args = ap.parse_args(argv)
    if args.single:
        return run_single(args)
    peak = peak_gbs()
    summary = {}
    for label, q, storage, masked, collision in CLASSES:
        if args.classes and not any(c in label for c in args.classes.split(";")):
            continue
        lat = make_lattice(q, args.n, storage, masked, collision)
        cells = args.n ** 3
        bpc = 2 * q * BYTES[storage]
        best_fixed = {}
        try:
            for variant in range(4):
                lat.set_step_variant(variant)
                t = lat.tuning()
                for bz in (256, 128, 64, 32):
                    lat.set_launch_shape(bz, 256 // bz)
                    ms = time_config(lat, args.steps, args.repeat)
                    frac = cells * bpc / (ms * 1e-3) / 1e9 / peak
                    rec = {"class": label, "variant": variant, "cells_per_thread": t["cells_per_thread"],
                           "min_blocks": t["min_blocks_per_sm"], "shape": [bz, 256 // bz],
                           "mlups": round(cells / (ms * 1e-3) / 1e6), "frac": round(frac, 3)}
                    print(json.dumps(rec), flush=True)
                    key = (t["cells_per_thread"], t["min_blocks_per_sm"])
                    best_fixed[key] = max(best_fixed.get(key, 0.0), frac)
            tuned = lat.autotune(4)
            ms = time_config(lat, args.steps, args.repeat)
            frac = cells * bpc / (ms * 1e-3) / 1e9 / peak
            print(json.dumps({"class": label, "autotuned": tuned, "mlups": round(cells / (ms * 1e-3) / 1e6),
                              "frac": round(frac, 3)}), flush=True)
            summary[label] = (best_fixed, tuned, frac, cells / (ms * 1e-3) / 1e6)
        finally:
            lat.close()
    keys = sorted({k for v in summary.values() for k in v[0]})
    print(f"\n| class | " + " | ".join(f"C{c},B{b}" for c, b in keys) + " | autotuned (C,B,shape) | autotuned GLUPS |")
    print("|---|" + "---|" * (len(keys) + 2))
    for label, (best, tuned, frac, mlups) in summary.items():
        cells = " | ".join(f"{best.get(k, float('nan')):.3f}" for k in keys)
        print(f"| {label} | {cells} | {tuned['cells_per_thread']},{tuned['min_blocks_per_sm']},"
              f"({tuned['block_z']},{tuned['block_y']}) {frac:.3f} | {mlups / 1e3:.1f} |")


if __name__ == "__main__":
    main()
