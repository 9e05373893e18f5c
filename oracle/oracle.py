"""Python bindings of the C oracle and of the compiled reference driver.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` — never by the ``openlb_b200`` package.

* :func:`step` / :func:`moments` / :func:`equilibrium` call the plain-C
  restatement in ``olb_oracle.c`` (logical layout, shifted populations).
* :func:`run_reference` runs OpenLB's own CPU_SISD build
  (``oracle/_ref/olb_ref_*``, made by ``oracle/ref/Makefile``) on a case
  directory and reads back its dumps.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libolb_oracle.so"
REF_DIR = HERE / "_ref"

(NONE, BGK, TRT, SMAGORINSKY, BOUNCE_BACK, BOUNCE_BACK_VELOCITY, FORCED_BGK, FORCED_TRT,
 INTERP_VELOCITY, INTERP_PRESSURE, LOCAL_VELOCITY, VELOCITY_EDGE, VELOCITY_CORNER,
 VELOCITY_INNER_EDGE, VELOCITY_INNER_CORNER, LOCAL_PRESSURE) = range(16)
KIND_NAMES = {
    NONE: "none", BGK: "bgk", TRT: "trt", SMAGORINSKY: "smagorinsky",
    BOUNCE_BACK: "bounce_back", BOUNCE_BACK_VELOCITY: "bounce_back_velocity",
    FORCED_BGK: "forced_bgk", FORCED_TRT: "forced_trt",
    INTERP_VELOCITY: "interpolated_velocity", INTERP_PRESSURE: "interpolated_pressure",
    LOCAL_VELOCITY: "local_velocity", LOCAL_PRESSURE: "local_pressure",
}
INTERPOLATED = (INTERP_VELOCITY, INTERP_PRESSURE)
# cells whose boundary values (RHO, VELOCITY) come from bc_values
VALUED = (INTERP_VELOCITY, INTERP_PRESSURE, LOCAL_VELOCITY, VELOCITY_EDGE, VELOCITY_CORNER,
          VELOCITY_INNER_EDGE, VELOCITY_INNER_CORNER, LOCAL_PRESSURE)
# edge and corner entries: cells of their boundary setter's material
SETTER_CELLS = (VELOCITY_EDGE, VELOCITY_CORNER, VELOCITY_INNER_EDGE, VELOCITY_INNER_CORNER)


class _Dyn(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("mixin", ctypes.c_int32),
        ("omega", ctypes.c_double), ("magic", ctypes.c_double),
        ("smagorinsky", ctypes.c_double), ("force", ctypes.c_double * 3),
        ("wall_u", ctypes.c_double * 3), ("wall_rho", ctypes.c_double),
        ("direction", ctypes.c_int32), ("orientation", ctypes.c_int32),
        ("normal", ctypes.c_int32 * 3), ("reserved", ctypes.c_int32),
    ]


class _Lattice(ctypes.Structure):
    _fields_ = [
        ("q", ctypes.c_int32), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32), ("periodic", ctypes.c_int32 * 3), ("n_dyn", ctypes.c_int32),
        ("dyn_id", ctypes.c_void_p), ("table", ctypes.POINTER(_Dyn)),
        ("bc_values", ctypes.c_void_p),
        ("force_field", ctypes.c_void_p),
    ]


class _Stats(ctypes.Structure):
    _fields_ = [("sum_rho", ctypes.c_double), ("sum_usqr", ctypes.c_double),
                ("max_usqr", ctypes.c_double), ("n_cells", ctypes.c_int64)]


@dataclass
class Dynamics:
    """One entry of the per-cell dynamics table."""
    kind: int
    omega: float = 1.0
    magic: float = 0.25
    smagorinsky: float = 0.1
    force: tuple = (0.0, 0.0, 0.0)
    wall_u: tuple = (0.0, 0.0, 0.0)
    wall_rho: float = 1.0
    mixin: int = BGK          # boundaries: collision of the mixin dynamics
    direction: int = 0        # flat boundaries: outward normal axis
    orientation: int = -1     # flat boundaries: outward normal sign
    normal: tuple = (0, 0, 0)  # edges and corners: the discrete normal
    boundary: int = LOCAL_VELOCITY  # edges and corners: the setter they come from
                                    # (LOCAL_VELOCITY or INTERP_VELOCITY)


@dataclass
class Case:
    """A lattice case: size, periodicity, per-cell dynamics id + table."""
    q: int
    size: tuple
    periodic: tuple
    table: list
    dyn_id: np.ndarray | None = None  # uint8[nx*ny*nz]
    extra: dict = field(default_factory=dict)
    bc_values: np.ndarray | None = None  # float64[4][nx*ny*nz]: RHO, VELOCITY x, y, z
    force_field: np.ndarray | None = None  # float64[3][nx*ny*nz]: FORCE per cell (forced dynamics)

    @property
    def n(self) -> int:
        nx, ny, nz = self.size
        return nx * ny * nz


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        _lib = ctypes.CDLL(str(LIB_PATH))
        for name in ("oracle_step_f32", "oracle_step_f64"):
            getattr(_lib, name).restype = ctypes.c_int
        _lib.oracle_descriptor.restype = ctypes.c_int
    return _lib


def _lattice(case: Case, keep: list):
    table = (_Dyn * len(case.table))()
    for k, d in enumerate(case.table):
        table[k].kind = d.kind
        table[k].omega = d.omega
        table[k].magic = d.magic
        table[k].smagorinsky = d.smagorinsky
        for e in range(3):
            table[k].force[e] = d.force[e]
            table[k].wall_u[e] = d.wall_u[e]
        table[k].wall_rho = d.wall_rho
        table[k].mixin = d.mixin
        table[k].direction = d.direction
        table[k].orientation = d.orientation
        for e in range(3):
            table[k].normal[e] = int(d.normal[e])
    lat = _Lattice()
    lat.q = case.q
    lat.nx, lat.ny, lat.nz = case.size
    for e in range(3):
        lat.periodic[e] = int(bool(case.periodic[e]))
    lat.n_dyn = len(case.table)
    if case.dyn_id is not None:
        ids = np.ascontiguousarray(case.dyn_id, dtype=np.uint8)
        assert ids.size == case.n
        keep.append(ids)
        lat.dyn_id = ids.ctypes.data
    else:
        lat.dyn_id = None
    lat.table = ctypes.cast(table, ctypes.POINTER(_Dyn))
    keep.append(table)
    if case.bc_values is not None:
        v = np.ascontiguousarray(case.bc_values, dtype=np.float64)
        assert v.size == 4 * case.n
        keep.append(v)
        lat.bc_values = v.ctypes.data
    else:
        lat.bc_values = None
    if case.force_field is not None:
        ff = np.ascontiguousarray(case.force_field, dtype=np.float64)
        assert ff.size == 3 * case.n
        keep.append(ff)
        lat.force_field = ff.ctypes.data
    else:
        lat.force_field = None
    return lat


def _sfx(dtype) -> str:
    dt = np.dtype(dtype)
    if dt == np.float32:
        return "f32"
    if dt == np.float64:
        return "f64"
    raise TypeError(dtype)


def step(case: Case, pops: np.ndarray, steps: int, ghost: float = float("nan"),
         with_stats: bool = False):
    """Run `steps` collide+stream steps in place; returns stats of the last step."""
    keep: list = []
    lat = _lattice(case, keep)
    assert pops.flags.c_contiguous and pops.size == case.q * case.n
    st = _Stats()
    fn = getattr(lib(), f"oracle_step_{_sfx(pops.dtype)}")
    if pops.dtype == np.float32:
        g = ctypes.c_float(ghost)
    else:
        g = ctypes.c_double(ghost)
    rc = fn(ctypes.byref(lat), ctypes.c_void_p(pops.ctypes.data), ctypes.c_int(steps), g,
            ctypes.byref(st) if with_stats else None)
    if rc != 0:
        raise RuntimeError(f"oracle step failed rc={rc}")
    if with_stats:
        return {"sum_rho": st.sum_rho, "sum_usqr": st.sum_usqr,
                "max_usqr": st.max_usqr, "n_cells": st.n_cells}
    return None


def post_process(case: Case, pops: np.ndarray):
    """The PostStream post-processors alone, in place (what the reference's
    lattice initialize() applies to the initial state)."""
    keep: list = []
    lat = _lattice(case, keep)
    fn = getattr(lib(), f"oracle_post_process_{_sfx(pops.dtype)}")
    rc = fn(ctypes.byref(lat), ctypes.c_void_p(pops.ctypes.data))
    if rc != 0:
        raise RuntimeError("oracle post_process failed")


def moments(case: Case, pops: np.ndarray):
    keep: list = []
    lat = _lattice(case, keep)
    rho = np.empty(case.n, pops.dtype)
    u = np.empty(3 * case.n, pops.dtype)
    fn = getattr(lib(), f"oracle_moments_{_sfx(pops.dtype)}")
    rc = fn(ctypes.byref(lat), ctypes.c_void_p(pops.ctypes.data),
            ctypes.c_void_p(rho.ctypes.data), ctypes.c_void_p(u.ctypes.data))
    if rc != 0:
        raise RuntimeError("oracle moments failed")
    return rho, u.reshape(3, case.n)


def equilibrium(q: int, rho: np.ndarray, u: np.ndarray) -> np.ndarray:
    rho = np.ascontiguousarray(rho)
    u = np.ascontiguousarray(u, dtype=rho.dtype).reshape(3, -1)
    n = rho.size
    pops = np.empty(q * n, rho.dtype)
    fn = getattr(lib(), f"oracle_equilibrium_{_sfx(rho.dtype)}")
    rc = fn(ctypes.c_int(q), ctypes.c_int64(n), ctypes.c_void_p(rho.ctypes.data),
            ctypes.c_void_p(u.ctypes.data), ctypes.c_void_p(pops.ctypes.data))
    if rc != 0:
        raise RuntimeError("oracle equilibrium failed")
    return pops


def descriptor(q: int):
    c = np.zeros(3 * q, np.int32)
    opp = np.zeros(q, np.int32)
    w = np.zeros(q, np.float64)
    rc = lib().oracle_descriptor(ctypes.c_int(q), ctypes.c_void_p(c.ctypes.data),
                                 ctypes.c_void_p(opp.ctypes.data), ctypes.c_void_p(w.ctypes.data))
    if rc != 0:
        raise ValueError(q)
    return c.reshape(q, 3), opp, w


# --------------------------------------------------------------------------
# the compiled reference (OpenLB CPU_SISD / CPU_SIMD through its public API)

def reference_binary(q: int, dtype, variant: str = "sisd") -> Path:
    bits = "f32" if np.dtype(dtype) == np.float32 else "f64"
    if variant == "simd":
        flags = open("/proc/cpuinfo").read()
        isa = "avx512" if " avx512f" in flags else "avx2"
        return REF_DIR / f"olb_ref_simd_q{q}_{bits}_{isa}"
    if variant == "nocse":
        return REF_DIR / f"olb_ref_sisd_q{q}_{bits}_nocse"
    return REF_DIR / f"olb_ref_sisd_q{q}_{bits}"


def write_case(dirpath: Path, case: Case, steps: int, init: np.ndarray | None = None,
               rhou: np.ndarray | None = None, stats: bool = False, bench=None,
               normals: bool = False, load_checkpoint: bytes | None = None,
               save_checkpoint: bool = False):
    """Write a case directory for olb_ref_driver (materials = dyn_id + 1).
    ``load_checkpoint``: file text OpenLB resumes from after initialize();
    ``save_checkpoint``: OpenLB saves the lattice after the steps (ckpt_out)."""
    dirpath = Path(dirpath)
    dirpath.mkdir(parents=True, exist_ok=True)
    ids = case.dyn_id if case.dyn_id is not None else np.zeros(case.n, np.uint8)
    (ids.astype(np.int32) + 1).tofile(dirpath / "materials.i32")
    lines = [f"size {case.size[0]} {case.size[1]} {case.size[2]}",
             "periodic {} {} {}".format(*[int(bool(p)) for p in case.periodic])]
    omegas = {d.omega for d in case.table
              if d.kind in (BGK, TRT, SMAGORINSKY, FORCED_BGK, FORCED_TRT) + VALUED}
    if len(omegas) > 1:
        raise ValueError("the reference driver takes one lattice-wide OMEGA")
    for k, d in enumerate(case.table):
        # edge and corner entries are cells of their boundary setter's material
        name = KIND_NAMES[d.boundary] if d.kind in SETTER_CELLS else KIND_NAMES[d.kind]
        lines.append(f"dyn {k + 1} {name}")
        if d.kind == BOUNCE_BACK_VELOCITY:
            lines.append("velocity {} {!r} {!r} {!r}".format(k + 1, *d.wall_u))
        if d.kind in (FORCED_BGK, FORCED_TRT):
            lines.append("force {} {!r} {!r} {!r}".format(k + 1, *d.force))
    first = case.table[0]
    fluid = [d for d in case.table if d.kind not in (NONE, BOUNCE_BACK, BOUNCE_BACK_VELOCITY)]
    ref = fluid[0] if fluid else first
    lines.append(f"omega {ref.omega!r}")
    lines.append(f"magic {ref.magic!r}")
    lines.append(f"smagorinsky {ref.smagorinsky!r}")
    mixins = {d.mixin for d in case.table if d.kind in VALUED}
    if mixins:
        if len(mixins) > 1:
            raise ValueError("the reference driver takes one mixin dynamics for all boundaries")
        lines.append(f"bcmixin {KIND_NAMES[mixins.pop()]}")
        vals = case.bc_values if case.bc_values is not None else np.concatenate(
            [np.ones(case.n), np.zeros(3 * case.n)])
        dt = init.dtype if init is not None else rhou.dtype
        np.ascontiguousarray(vals, dtype=dt).tofile(dirpath / "bcvalues.bin")
        lines.append("bcvalues 1")
    if case.force_field is not None:
        dt = init.dtype if init is not None else rhou.dtype
        np.ascontiguousarray(case.force_field, dtype=dt).tofile(dirpath / "forcefield.bin")
        lines.append("forcefield 1")
    if normals:
        lines.append(f"normals {int(normals)}")
    if init is not None:
        np.ascontiguousarray(init).tofile(dirpath / "init.bin")
        lines.append("init pops")
    else:
        np.ascontiguousarray(rhou).tofile(dirpath / "rhou.bin")
        lines.append("init eq")
    lines.append(f"steps {steps}")
    if stats:
        lines.append("stats 1")
    if bench is not None:
        lines.append(f"bench {bench[0]} {bench[1]}")
    if load_checkpoint is not None:
        (dirpath / "ckpt_in_rank0_size1.dat").write_bytes(load_checkpoint)
        lines.append("load ckpt_in")
    if save_checkpoint:
        lines.append("save ckpt_out")
    (dirpath / "case.txt").write_text("\n".join(lines) + "\n")


def reference_normals(materials: np.ndarray, periodic, boundary_materials, q: int = 19) -> np.ndarray:
    """computeBoundaryTypeAndNormal of OpenLB itself (fluid material 1,
    outside material 0) for every cell of `boundary_materials`: int32[4][n]
    (type, n_x, n_y, n_z), type -1 elsewhere."""
    m = np.ascontiguousarray(materials, dtype=np.int32)
    size = m.shape
    n = m.size
    binary = reference_binary(q, np.float64)
    with tempfile.TemporaryDirectory() as d:
        dp = Path(d)
        m.tofile(dp / "materials.i32")
        lines = [f"size {size[0]} {size[1]} {size[2]}",
                 "periodic {} {} {}".format(*[int(bool(v)) for v in periodic])]
        for mat in sorted(int(v) for v in np.unique(m) if v != 0):
            kind = "interpolated_velocity" if mat in boundary_materials else ("bgk" if mat == 1 else "bounce_back")
            lines.append(f"dyn {mat} {kind}")
        rhou = np.zeros((4, n))
        rhou[0] = 1.0
        rhou.tofile(dp / "rhou.bin")
        lines += ["omega 1.0", "init eq", "steps 0", "normals 2"]
        (dp / "case.txt").write_text("\n".join(lines) + "\n")
        r = subprocess.run([str(binary), d], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference failed: {r.stdout[-2000:]} {r.stderr[-2000:]}")
        return np.fromfile(dp / "out_normals.i32", dtype=np.int32).reshape(4, n)


def run_reference(case: Case, steps: int, dtype, init: np.ndarray | None = None,
                  rhou: np.ndarray | None = None, variant: str = "sisd", stats: bool = False,
                  threads: int | None = None, normals: bool = False,
                  load_checkpoint: bytes | None = None, save_checkpoint: bool = False):
    """Run OpenLB itself; returns dict(pops, rho, u[, stats][, checkpoint])."""
    binary = reference_binary(case.q, dtype, variant)
    if not binary.exists():
        raise RuntimeError(f"reference build missing: {binary} (make -C oracle/ref)")
    with tempfile.TemporaryDirectory() as d:
        write_case(Path(d), case, steps, init=init, rhou=rhou, stats=stats, normals=normals,
                   load_checkpoint=load_checkpoint, save_checkpoint=save_checkpoint)
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        r = subprocess.run([str(binary), d], capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"reference failed: {r.stdout[-2000:]} {r.stderr[-2000:]}")
        n = case.n
        out = {
            "pops": np.fromfile(Path(d) / "out_pops.bin", dtype=dtype),
            "rho": np.fromfile(Path(d) / "out_rho.bin", dtype=dtype),
            "u": np.fromfile(Path(d) / "out_u.bin", dtype=dtype).reshape(3, n),
        }
        if stats:
            out["stats"] = np.loadtxt(Path(d) / "out_stats.txt", ndmin=2)
        if normals:
            out["normals"] = np.fromfile(Path(d) / "out_normals.i32", dtype=np.int32).reshape(4, n)
        if save_checkpoint:
            out["checkpoint"] = (Path(d) / "ckpt_out_rank0_size1.dat").read_bytes()
        return out
