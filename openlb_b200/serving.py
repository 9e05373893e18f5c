"""Serving layer: many cavity / channel solves on one GPU with continuous batching.

Requests arrive over time (seeded Poisson process).  The batched server keeps
an :class:`Ensemble` on the device; after every chunk of `check_interval` steps
it retires the instances whose velocity-change residual fell below the
tolerance (or that reached their step limit) and admits queued requests while
instance slots and pool memory (the HBM admission budget) allow — requests that
arrive while others run join the next chunk.  The plain loop solves the same
requests one at a time, in arrival order, through the single-lattice API with
the same convergence check: once as an OpenLB example's time loop drives a
lattice (one collideAndStream per step, statistics on), once with this
library's multi-step call.  All report solves/s and the p50/p99 latency
(completion minus arrival).

    python -m openlb_b200.serving --requests 2000 --rate 50 --budget-gb 150 --plain

Every instance carries its geometry as a table (one class byte per cell:
fluid, bounce-back wall, moving wall) unless --procedural names the built-in
cavity instead.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _abi
from .lattice import BGKdynamics, BounceBack, BounceBackVelocity, ForcedBGKdynamics, Lattice
from .workloads import cavity


@dataclass
class Request:
    """One solve: a lid-driven cavity (or channel) of side n at Reynolds number re."""
    rid: int
    arrival: float          # seconds after the start of the run
    n: int
    re: float
    lid: float
    kind: int = _abi.ENSEMBLE_CAVITY
    tol: float = 1e-7
    max_steps: int = 20000
    force: float = 0.0
    geometry: np.ndarray | None = None  # kind ENSEMBLE_GEOMETRY: n^3 cell classes (0 fluid, 1 wall, 2 lid), z fastest

    @property
    def nu(self) -> float:
        """Lattice viscosity from Re = lid * n / nu."""
        return self.lid * self.n / self.re

    @property
    def omega(self) -> float:
        return 1.0 / (3.0 * self.nu + 0.5)

    @property
    def cells(self) -> int:
        return self.n ** 3


@dataclass
class Result:
    rid: int
    steps: int
    residual: float
    start: float
    finish: float
    arrival: float
    u: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


def make_requests(count: int, rate: float, seed: int = 0, n_range=(24, 96), re_range=(10.0, 400.0),
                  lid_range=(0.05, 0.1), tol: float = 1e-7, max_steps: int = 20000,
                  tables: bool = False) -> list:
    """Cavity requests: side uniform in n_range, Re log-uniform, lid speed
    uniform, Poisson arrivals at `rate` per second (0: all at t = 0).
    tables: each request carries its geometry as a table (kind
    ENSEMBLE_GEOMETRY) instead of naming the procedural cavity."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, count) if rate > 0 else np.zeros(count)
    arrivals = np.cumsum(gaps) - (gaps[0] if count else 0.0)
    out = []
    for k in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        re = float(math.exp(rng.uniform(math.log(re_range[0]), math.log(re_range[1]))))
        lid = float(rng.uniform(*lid_range))
        req = Request(k, float(arrivals[k]), n, re, lid, tol=tol, max_steps=max_steps)
        if tables:
            req.kind = _abi.ENSEMBLE_GEOMETRY
            req.geometry = cavity((n, n, n))
        out.append(req)
    return out


class Ensemble:
    """Binding of the ensemble C ABI (olb_b200_ensemble_*)."""

    def __init__(self, pool_bytes: int, max_instances: int = 1024, device: int = 0):
        self._lib = _abi.load()
        d = _abi.EnsembleDesc()
        d.q, d.storage, d.device = 19, _abi.STORAGE["f32"], device
        d.max_instances, d.pool_bytes = max_instances, int(pool_bytes)
        h = ctypes.c_void_p()
        _abi.check(self._lib, self._lib.olb_b200_ensemble_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        self.max_instances = max_instances
        self._res = np.zeros(max_instances, np.float64)
        self._steps = np.zeros(max_instances, np.uint32)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.olb_b200_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def bytes_for(self, n: int, table: bool = False) -> int:
        """Pool bytes of an instance of side n (with a geometry table: + n^3
        rounded up to 256)."""
        extra = -(-n ** 3 // 256) * 256 if table else 0
        return int(self._lib.olb_b200_ensemble_bytes_per_instance(n, n, n)) + extra

    def add(self, req: Request) -> int | None:
        """Admit a request; None when no slot or pool memory is free."""
        d = _abi.InstanceDesc()
        d.kind, d.nx, d.ny, d.nz = req.kind, req.n, req.n, req.n
        d.omega = req.omega
        d.wall_u[0] = req.lid if req.kind in (_abi.ENSEMBLE_CAVITY, _abi.ENSEMBLE_GEOMETRY) else 0.0
        d.force[0] = req.force
        cells = None
        if req.kind == _abi.ENSEMBLE_GEOMETRY:
            cells = np.ascontiguousarray(req.geometry, dtype=np.uint8).reshape(-1)
            if cells.size != req.cells:
                raise ValueError(f"geometry table has {cells.size} cells, the instance {req.cells}")
            d.cells = cells.ctypes.data
        slot = ctypes.c_int32()
        st = self._lib.olb_b200_ensemble_add(self._h, ctypes.byref(d), ctypes.byref(slot))
        if st == _abi.ERR_OOM:
            return None
        _abi.check(self._lib, st)
        return slot.value

    def remove(self, slot: int) -> None:
        _abi.check(self._lib, self._lib.olb_b200_ensemble_remove(self._h, slot))

    def run(self, steps: int, check: bool = True):
        _abi.check(self._lib, self._lib.olb_b200_ensemble_run(
            self._h, steps, int(check), self._res.ctypes.data, self._steps.ctypes.data))
        return self._res, self._steps

    def moments(self, slot: int, n: int):
        rho = np.empty(n ** 3, np.float32)
        u = np.empty(3 * n ** 3, np.float32)
        _abi.check(self._lib, self._lib.olb_b200_ensemble_get_moments(
            self._h, slot, rho.ctypes.data, u.ctypes.data))
        return rho, u.reshape(3, -1)

    def info(self) -> dict:
        free = ctypes.c_int64()
        active = ctypes.c_int32()
        tiles = ctypes.c_int32()
        _abi.check(self._lib, self._lib.olb_b200_ensemble_info(
            self._h, ctypes.byref(free), ctypes.byref(active), ctypes.byref(tiles)))
        return {"pool_free_bytes": free.value, "active": active.value, "tiles": tiles.value}

    def set_occupancy(self, blocks_per_sm: int) -> None:
        _abi.check(self._lib, self._lib.olb_b200_ensemble_set_occupancy(self._h, blocks_per_sm))


def serve_batched(requests: list, pool_bytes: int, max_instances: int = 1024, check_interval: int = 100,
                  keep_velocity: bool = False, device: int = 0, occupancy: int = 4) -> dict:
    """Continuous batching: admit on arrival while slots and pool memory allow."""
    ens = Ensemble(pool_bytes, max_instances, device)
    ens.set_occupancy(occupancy)
    pending = sorted(requests, key=lambda r: r.arrival)
    queue: list = []
    active: dict = {}   # slot -> (request, start time)
    results: list = []
    t0 = time.perf_counter()
    busy = 0.0
    peak_active = 0
    try:
        while pending or queue or active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.pop(0))
            # admission in arrival order; a request that does not fit waits
            while queue:
                slot = ens.add(queue[0])
                if slot is None:
                    break
                active[slot] = (queue.pop(0), time.perf_counter() - t0)
            peak_active = max(peak_active, len(active))
            if not active:
                if pending:
                    time.sleep(max(0.0, pending[0].arrival - (time.perf_counter() - t0)))
                continue
            c0 = time.perf_counter()
            res, steps = ens.run(check_interval, check=True)
            busy += time.perf_counter() - c0
            now = time.perf_counter() - t0
            for slot in list(active):
                req, start = active[slot]
                done_steps = int(steps[slot])
                if res[slot] < req.tol or done_steps >= req.max_steps:
                    u = ens.moments(slot, req.n)[1] if keep_velocity else None
                    results.append(Result(req.rid, done_steps, float(res[slot]), start, now, req.arrival, u))
                    ens.remove(slot)
                    del active[slot]
    finally:
        ens.close()
    out = summarize(results, time.perf_counter() - t0, busy)
    out["peak_active"] = peak_active
    return out


def cavity_lattice(req: Request, device: int = 0) -> Lattice:
    """The request's lattice on the single-lattice API (same geometry and
    dynamics as the ensemble's instance)."""
    n = req.n
    if req.kind == _abi.ENSEMBLE_GEOMETRY:
        ids = np.ascontiguousarray(req.geometry, dtype=np.uint8).reshape(n, n, n)
        # an axis is periodic where fluid reaches its faces (the instance wraps every axis)
        periodic = tuple(bool(np.any(np.take(ids, 0, axis=a) == 0) or np.any(np.take(ids, -1, axis=a) == 0))
                         for a in range(3))
        fluid = (ForcedBGKdynamics(omega=req.omega, force=(req.force, 0.0, 0.0)) if req.force != 0.0
                 else BGKdynamics(omega=req.omega))
        lat = Lattice(19, (n, n, n), periodic, storage="f32", device=device)
        lat.set_dynamics([fluid, BounceBack(), BounceBackVelocity((req.lid, 0.0, 0.0))], ids.reshape(-1))
    elif req.kind == _abi.ENSEMBLE_CAVITY:
        lat = Lattice(19, (n, n, n), (False, False, False), storage="f32", device=device)
        lat.set_dynamics([BGKdynamics(omega=req.omega), BounceBack(), BounceBackVelocity((req.lid, 0.0, 0.0))],
                         cavity((n, n, n)))
    else:
        ids = np.zeros((n, n, n), np.uint8)
        ids[:, 0, :] = ids[:, -1, :] = ids[:, :, 0] = ids[:, :, -1] = 1
        lat = Lattice(19, (n, n, n), (True, False, False), storage="f32", device=device)
        lat.set_dynamics([ForcedBGKdynamics(omega=req.omega, force=(req.force, 0.0, 0.0)), BounceBack()],
                         ids.reshape(-1))
    return lat


def serve_plain(requests: list, check_interval: int = 100, keep_velocity: bool = False, device: int = 0,
                style: str = "chunked") -> dict:
    """The plain loop: one request at a time, in arrival order.

    ``style="per_step"`` drives each lattice the way an OpenLB example's time
    loop does — one collideAndStream call per step with the lattice statistics
    on (the reference's default; each step then waits for its statistics) —
    and checks the residual every ``check_interval`` steps.  ``"chunked"`` uses
    this library's multi-step call (``check_interval`` steps per call, no
    statistics) between checks."""
    if style not in ("chunked", "per_step"):
        raise ValueError(f"unknown plain-loop style {style!r}")
    pending = sorted(requests, key=lambda r: r.arrival)
    results: list = []
    t0 = time.perf_counter()
    busy = 0.0
    for req in pending:
        now = time.perf_counter() - t0
        if req.arrival > now:
            time.sleep(req.arrival - now)
        start = time.perf_counter() - t0
        c0 = time.perf_counter()
        lat = cavity_lattice(req, device)
        try:
            steps, res = 0, math.inf
            while True:
                if style == "chunked":
                    lat.collide_and_stream(check_interval)
                else:
                    for _ in range(check_interval):
                        lat.collide_and_stream(1, stats=True)
                steps += check_interval
                res = lat.velocity_residual()
                if res < req.tol or steps >= req.max_steps:
                    break
            u = lat.get_moments()[1] if keep_velocity else None
        finally:
            lat.close()
        busy += time.perf_counter() - c0
        results.append(Result(req.rid, steps, res, start, time.perf_counter() - t0, req.arrival, u))
    return summarize(results, time.perf_counter() - t0, busy)


def summarize(results: list, wall: float, busy: float) -> dict:
    """solves/s over the wall time of the run (first arrival to last
    completion), latency percentiles over all requests."""
    lat = np.array([r.latency for r in results]) if results else np.zeros(1)
    return {
        "solves": len(results),
        "wall_s": wall,
        "gpu_busy_s": busy,
        "solves_per_s": len(results) / wall if wall > 0 else 0.0,
        "p50_latency_s": float(np.percentile(lat, 50)),
        "p99_latency_s": float(np.percentile(lat, 99)),
        "mean_steps": float(np.mean([r.steps for r in results])) if results else 0.0,
        "results": results,
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--rate", type=float, default=0.0, help="Poisson arrival rate per s (0: all at once)")
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--nmin", type=int, default=24)
    ap.add_argument("--nmax", type=int, default=96)
    ap.add_argument("--max-steps", type=int, default=20000)
    ap.add_argument("--tol", type=float, default=1e-7)
    ap.add_argument("--check", type=int, default=100)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--max-instances", type=int, default=4096)
    ap.add_argument("--occupancy", type=int, default=4)
    ap.add_argument("--plain", action="store_true", help="also run the plain one-at-a-time loops")
    ap.add_argument("--procedural", action="store_true",
                    help="instances name the built-in cavity instead of carrying geometry tables")
    args = ap.parse_args(argv)
    reqs = make_requests(args.requests, args.rate, args.seed, (args.nmin, args.nmax), tol=args.tol,
                         max_steps=args.max_steps, tables=not args.procedural)
    out = {"config": vars(args), "cell_steps_total": None}
    b = serve_batched(reqs, int(args.budget_gb * 2 ** 30), args.max_instances, args.check,
                      occupancy=args.occupancy)
    steps = {r.rid: r.steps for r in b["results"]}
    out["cell_steps_total"] = float(sum(r.cells * steps[r.rid] for r in reqs))
    out["batched"] = {k: v for k, v in b.items() if k != "results"}
    out["batched"]["mlups"] = out["cell_steps_total"] / b["wall_s"] / 1e6
    if args.plain:
        for style in ("per_step", "chunked"):
            p = serve_plain(reqs, args.check, style=style)
            key = "plain" if style == "per_step" else "plain_chunked"
            out[key] = {k: v for k, v in p.items() if k != "results"}
            out[key]["mlups"] = out["cell_steps_total"] / p["wall_s"] / 1e6
            out[f"speedup_vs_{key}"] = out["batched"]["solves_per_s"] / out[key]["solves_per_s"]
    print(json.dumps(out))


if __name__ == "__main__":
    main()
