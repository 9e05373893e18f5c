#!/usr/bin/env python3
"""Benchmark of the fused collide-and-stream step (one JSON line on rank 0).

Workload: periodic Taylor-Green vortex, D3Q19 BGK, FP32, 256^3 cells,
u0 = 0.05, nu = 0.0125 (tau = 0.5375), seeded +-1e-4 velocity noise, rho = 1,
equilibrium start.  A "step" is one collide-and-stream over all cells.

Metric: MLUPS = cells * steps / seconds (all cells are fluid, matching OpenLB's
getNvoxel count).  The population array (1.37 GB) is larger than L2 (126 MB),
so no L2 flush is needed between steps.

  value     device time of K back-to-back steps (CUDA events on the lattice's
            stream), state resident in HBM.
  e2e       the same K steps through the C ABI as a user drives them, host
            buffers included: upload of the initial state from pinned memory
            (the density and velocity fields, expanded to populations on the
            device as iniEquilibrium does), K x collide_and_stream(1,
            statistics) each reading its FP64
            statistics back to the host, and the download of the density and
            velocity fields; MLUPS over the wall time of all of it.
  roofline  HBM bound: algorithmic bytes per launch (2*q*4 B per cell) over the
            mean step-kernel duration, against MEASURED_PEAKS.json hbm_gbs.

--impl reference times OpenLB's own CPU path (CPU_SIMD + OpenMP build in
oracle/_ref, all host threads) on the same workload and metric.
N > 1 (torchrun): every rank runs an independent replica of the workload
(weak scaling); value is the total cells*steps over the slowest rank's time.

--workload serve runs the served ensemble instead (the serving layer,
openlb_b200/serving.py): 2000 lid-driven cavities, sides U{24..96}, Re
log-uniform in [10, 400], lid speed U[0.05, 0.1], each until its
velocity-change residual < 1e-7 or 20000 steps, Poisson arrivals, 150 GB
admission budget.  One JSON line: solves/s and p50/p99 latency of the batched
server, the same requests through the two plain one-at-a-time loops (one
collideAndStream per step with statistics, as an OpenLB example drives a
lattice; and this library's multi-step call per 100 steps) and the ratios.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = {"name": "tgv256_d3q19_bgk_f32", "n": 256, "q": 19, "storage": "f32", "u0": 0.05,
            "nu": 0.0125, "noise": 1e-4, "seed": 1234}
METRIC = "MLUPS"
BYTES_PER_CELL = {"f32": 4, "f64": 8, "f16": 2, "bf16": 2}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=WORKLOAD["n"], help="cube side (default 256)")
    ap.add_argument("--storage", default=WORKLOAD["storage"], choices=list(BYTES_PER_CELL))
    ap.add_argument("--lattice", type=int, default=WORKLOAD["q"], choices=[19, 27])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="step", choices=["step", "serve"],
                    help="step: the fused step on the 256^3 TGV (default); serve: the served "
                         "ensemble of cavities against both plain loops")
    ap.add_argument("--requests", type=int, default=2000, help="serve: number of requests")
    ap.add_argument("--rate", type=float, default=50.0, help="serve: Poisson arrival rate per s")
    ap.add_argument("--max-steps", type=int, default=20000, help="serve: step limit per request")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serve: HBM admission budget")
    ap.add_argument("--no-plain", action="store_true", help="serve: skip the two plain loops")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing

def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world, device=None):
    if world > 1:
        import torch.distributed as dist
        if device is not None:
            dist.barrier(device_ids=[device])
        else:
            dist.barrier()


def allreduce_max(world, value: float, device=None) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{device}" if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for name, flag in zip(names, parts[4:8]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        under_load = sorted(sm)[len(sm) // 4:] or sm
        return {"sm_mhz": float(np.median(under_load)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# our implementation

def measured_hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


def ncu_traffic(kernel_tag: str):
    """dram bytes per launch from a committed ncu summary, or None."""
    p = ROOT / "profiles" / f"{kernel_tag}.txt"
    if not p.exists():
        p = p.with_suffix(".md")
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def run_ours(args, world, rank, local):
    import openlb_b200 as ob
    from openlb_b200.workloads import taylor_green

    n, q, storage = args.n, args.lattice, args.storage
    dtype = np.float64 if storage == "f64" else np.float32
    omega, pops = taylor_green(n, WORKLOAD["u0"], WORKLOAD["nu"], WORKLOAD["noise"],
                               WORKLOAD["seed"] + rank, dtype, f"D3Q{q}")
    cells = n ** 3
    lat = ob.Lattice(q, (n, n, n), (True, True, True), storage=storage, device=local)
    lat.set_dynamics([ob.BGKdynamics(omega=omega)])
    lat.set_populations(pops)
    # pick the step-kernel variant and launch shape on this lattice (state restored)
    tuning = lat.autotune(4)
    lat.collide_and_stream(args.warmup)
    lat.synchronize()

    # ---- device-timed region (value) ----
    barrier(world, local)
    lat.synchronize()
    with ClockSampler(local) as clk:
        ms = lat.time_steps(args.steps)
    lat.synchronize()
    barrier(world, local)
    sec = ms * 1e-3
    sec_max = allreduce_max(world, sec, local)
    value = world * cells * args.steps / sec_max / 1e6

    # ---- end-to-end through the C ABI with host buffers (e2e) ----
    e2e = None
    if not args.no_e2e:
        import torch
        from openlb_b200.workloads import tgv_velocity
        tdt = torch.float64 if storage == "f64" else torch.float32
        # the initial state as the example defines it: rho and u fields
        # (iniEquilibrium), expanded to populations on the device
        u_init = torch.from_numpy(np.ascontiguousarray(
            tgv_velocity(n, WORKLOAD["u0"], WORKLOAD["noise"], WORKLOAD["seed"] + rank, dtype).reshape(-1))).pin_memory()
        rho_init = torch.ones(cells, dtype=tdt).pin_memory()
        rho_h = torch.empty(cells, dtype=tdt).pin_memory()
        u_h = torch.empty(3 * cells, dtype=tdt).pin_memory()
        barrier(world, local)
        t0 = time.perf_counter()
        lat.ini_equilibrium(rho_init.numpy(), u_init.numpy())
        for _ in range(args.steps):
            lat.collide_and_stream(1, stats=True)
        lat.get_moments(out=(rho_h.numpy(), u_h.numpy()))
        t1 = time.perf_counter()
        barrier(world, local)
        e2e_sec = allreduce_max(world, t1 - t0, local)
        real = 8 if storage == "f64" else 4
        e2e = {"value": world * cells * args.steps / e2e_sec / 1e6, "unit": METRIC,
               "h2d_bytes_per_step": 4 * cells * real / args.steps,
               "d2h_bytes_per_step": (40 * args.steps + 4 * cells * real) / args.steps,
               "note": "per step: fused step + FP64 statistics read back; the initial rho, u fields "
                       "(iniEquilibrium, expanded to populations on the device) and the final rho/u "
                       "download amortised over the steps"}
    info = lat.info()
    lat.close()

    peak, peak_kind = measured_hbm_peak()
    bpc = 2 * q * BYTES_PER_CELL[storage]
    achieved = cells * bpc / (sec / args.steps) / 1e9
    # the committed ncu summaries of the kernels the two bench arms time
    tag = {(256, 19, "f32"): f"aa_step_kernel_{WORKLOAD['name']}",
           (256, 19, "f16"): "aa_step_paired_kernel_f16_256"}.get((n, q, storage))
    traffic = ncu_traffic(tag) if tag else None
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                "bytes_per_cell": bpc, "roofline_mlups": round(peak * 1e9 / bpc / 1e6, 1)}
    return {
        "value": value, "ms_per_step": sec_max * 1e3 / args.steps, "clocks": clk.summary(),
        "e2e": e2e, "roofline": roofline, "gpu_launches": args.steps,
        "launch_shape": [info["block_z"], info["block_y"]], "cells": cells,
        "tuning": {k: tuning[k] for k in ("variant", "cells_per_thread", "min_blocks_per_sm", "candidates")},
    }


# ---------------------------------------------------------------------------
# the reference's CPU implementation (OpenLB CPU_SIMD + OpenMP)

def reference_binary():
    flags = open("/proc/cpuinfo").read()
    isa = "avx512" if " avx512f" in flags else "avx2"
    return ROOT / "oracle" / "_ref" / f"olb_ref_simd_q19_f32_{isa}", isa


def run_reference_cpu(n: int, steps: int, warmup: int, threads: int):
    """Times OpenLB's own collideAndStream (CPU_SIMD + OpenMP) on the TGV."""
    from openlb_b200.workloads import tgv_velocity
    binary, isa = reference_binary()
    if not binary.exists():
        return None, f"reference build missing ({binary.name}); run make -C oracle/ref"
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        cells = n ** 3
        np.ones(cells, np.int32).tofile(d / "materials.i32")
        rhou = np.empty((4, cells), np.float32)
        rhou[0] = 1.0
        rhou[1:] = tgv_velocity(n, WORKLOAD["u0"], WORKLOAD["noise"], WORKLOAD["seed"], np.float32)
        rhou.tofile(d / "rhou.bin")
        tau = 0.5 + 3 * WORKLOAD["nu"]
        (d / "case.txt").write_text(
            f"size {n} {n} {n}\nperiodic 1 1 1\ndyn 1 bgk\nomega {1.0 / tau!r}\ninit eq\n"
            f"bench {warmup} {steps}\n")
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
        r = subprocess.run([str(binary), str(d)], capture_output=True, text=True, env=env)
        if r.returncode != 0:
            return None, f"reference run failed: {r.stderr[-300:]}"
        line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
        out = json.loads(line)
        out["isa"] = isa
        return out, None


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# the served ensemble (continuous batching) against the plain loops

SERVE = {"name": "serve_cavities", "sides": (24, 96), "re": (10.0, 400.0), "lid": (0.05, 0.1), "tol": 1e-7,
         "check": 100, "seed": 5}


def run_serve(args, world, rank, local):
    """One JSON line: solves/s and p50/p99 latency of the batched server, the
    same requests through both plain one-at-a-time loops, and the ratios.
    Every rank serves its own request stream (replicas); rank 0 reports its
    own line with the total solves/s of all ranks as value."""
    from openlb_b200 import serving
    reqs = serving.make_requests(args.requests, args.rate, SERVE["seed"] + rank, SERVE["sides"], SERVE["re"],
                                 SERVE["lid"], SERVE["tol"], args.max_steps, tables=True)
    b = serving.serve_batched(reqs, int(args.budget_gb * 2 ** 30), 4096, SERVE["check"], device=local)
    steps = {r.rid: r.steps for r in b["results"]}
    cell_steps = float(sum(r.cells * steps[r.rid] for r in reqs))
    out = {"batched": {k: v for k, v in b.items() if k != "results"}}
    out["batched"]["mlups"] = cell_steps / b["wall_s"] / 1e6
    if not args.no_plain:
        for style, key in (("per_step", "plain_per_step"), ("chunked", "plain_chunked")):
            p = serving.serve_plain(reqs, SERVE["check"], device=local, style=style)
            out[key] = {k: v for k, v in p.items() if k != "results"}
            out[key]["mlups"] = cell_steps / p["wall_s"] / 1e6
            out[f"speedup_vs_{key}"] = b["solves_per_s"] / p["solves_per_s"]
    total = b["solves_per_s"]
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([total], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t)
        total = float(t.item())
    return total, out, cell_steps


def main():
    args = parse()
    world, rank, local = dist_init(args)
    if args.workload == "serve":
        return main_serve(args, world, rank, local)
    config = {"workload": WORKLOAD["name"] if (args.n, args.lattice, args.storage) == (256, 19, "f32")
              else f"tgv{args.n}_d3q{args.lattice}_bgk_{args.storage}",
              "lattice": f"D3Q{args.lattice}", "cells": args.n ** 3, "size": [args.n] * 3,
              "collision": "BGK", "periodic": [True, True, True], "storage": args.storage,
              "u0": WORKLOAD["u0"], "nu": WORKLOAD["nu"], "l2": "inputs larger than L2 (no flush)",
              "parallelism": f"replicas{world}" if world > 1 else "single-gpu"}
    line = {"metric": METRIC, "unit": METRIC, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic",
            "dtype": {"f32": "f32", "f64": "f64", "f16": "f32 math, f16 storage",
                      "bf16": "f32 math, bf16 storage"}[args.storage],
            "config": config}

    if args.impl == "reference":
        if rank != 0:
            return
        threads = cpu_threads()
        # bounded sample: 2 warm-up + min(steps, 40) steps of the 256^3 workload
        nsteps = max(1, min(args.steps, 40))
        res, err = run_reference_cpu(args.n, nsteps, min(args.warmup, 2), threads)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return
        v = res["mlups"]
        line.update({"impl": "reference", "value": v, "ms_per_step": res["seconds"] * 1e3 / res["steps"],
                     "cpu_baseline": {"value": v, "unit": METRIC, "cores": res["threads"], "kind": "reference",
                                      "sample": f"OpenLB CPU_SIMD({res['isa']})+OpenMP collideAndStream on the "
                                                f"{args.n}^3 TGV, {res['steps']} steps after 2 warm-up"},
                     "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        line["steps"] = res["steps"]
        print(json.dumps(line))
        return

    res = run_ours(args, world, rank, local)
    line.update({"value": res["value"], "ms_per_step": res["ms_per_step"], "e2e": res["e2e"],
                 "roofline": res["roofline"], "clocks": res["clocks"], "gpu_launches": res["gpu_launches"]})
    line["config"]["launch_shape"] = res["launch_shape"]
    line["config"]["step_variant"] = res["tuning"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = cpu_threads()
        ref, err = run_reference_cpu(args.n, 30, 2, threads)
        if ref is not None:
            line["cpu_baseline"] = {"value": ref["mlups"], "unit": METRIC, "cores": ref["threads"],
                                    "kind": "reference",
                                    "sample": f"OpenLB CPU_SIMD({ref['isa']})+OpenMP collideAndStream, "
                                              f"{args.n}^3 TGV, {ref['steps']} steps after 2 warm-up"}
        else:
            line["cpu_baseline"] = {"value": None, "unavailable": err}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main_serve(args, world, rank, local):
    config = {"workload": SERVE["name"], "requests": args.requests, "sides": list(SERVE["sides"]),
              "re_log_uniform": list(SERVE["re"]), "lid": list(SERVE["lid"]), "tol": SERVE["tol"],
              "max_steps": args.max_steps, "budget_gb": args.budget_gb, "arrivals": f"poisson {args.rate}/s",
              "seed": SERVE["seed"], "check_interval": SERVE["check"], "geometry": "per-instance tables",
              "lattice": "D3Q19", "collision": "BGK",
              "storage": "f32", "parallelism": f"replicas{world}" if world > 1 else "single-gpu"}
    line = {"metric": "solves/s", "unit": "solves/s", "n_gpus": world, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic", "dtype": "f32", "config": config}
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "OpenLB has no serving layer; its "
                              "one-request-at-a-time loop is the plain_per_step arm of this line"}))
        return
    total, out, cell_steps = run_serve(args, world, rank, local)
    if rank == 0:
        b = out["batched"]
        line.update({"value": total, "p50_latency_s": b["p50_latency_s"], "p99_latency_s": b["p99_latency_s"],
                     "e2e": {"value": total, "unit": "solves/s", "note": "host-driven server, wall clock "
                             "from the first arrival to the last completion"},
                     "cell_steps": cell_steps, **out})
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
