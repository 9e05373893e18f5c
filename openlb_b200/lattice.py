"""Host-side mirror of OpenLB's lattice API for the B200 collide-and-stream.

Two layers:

* :class:`Lattice` — one lattice handle of the C ABI (``include/olb_b200.h``):
  create, dynamics table, populations in/out, collide-and-stream, moments.
* :class:`SuperGeometry` / :class:`SuperLattice` — the user-facing calls of an
  OpenLB example with the reference's names and meaning
  (``examples/laminar/cavity3dBenchmark/cavity3d.cpp:154-243``):
  ``defineDynamics``, ``setParameter<OMEGA>``, ``defineU``, ``defineField<FORCE>``,
  ``iniEquilibrium``, ``initialize``, ``collideAndStream``, ``getStatistics`` and
  the Density3D / Velocity3D functors.

Errors surface as :class:`openlb_b200._abi.OlbError` (a ``RuntimeError``), as
OpenLB surfaces CUDA errors through ``std::runtime_error``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _abi
from .descriptors import D3Q19, D3Q27, descriptor

# ---------------------------------------------------------------------------
# dynamics descriptions (the reference's dynamics aliases)


@dataclass(frozen=True)
class Dynamics:
    """A dynamics alias and its per-dynamics parameters/fields."""
    kind: int
    omega: float | None = None
    magic: float = 0.25
    smagorinsky: float = 0.1
    force: tuple = (0.0, 0.0, 0.0)
    wall_u: tuple = (0.0, 0.0, 0.0)
    wall_rho: float = 1.0
    mixin: int = 0          # boundaries: the mixin's collision kind
    direction: int = 0      # flat boundaries: outward normal axis
    orientation: int = 0    # flat boundaries: outward normal sign
    normal: tuple = (0, 0, 0)  # edges and corners: the discrete normal

    def params(self, omega_default: float | None = None) -> _abi.DynParams:
        p = _abi.DynParams()
        p.kind = self.kind
        p.mixin = int(self.mixin)
        p.direction = int(self.direction)
        p.orientation = int(self.orientation)
        for e in range(3):
            p.normal[e] = int(self.normal[e])
        omega = self.omega if self.omega is not None else omega_default
        p.omega = float(omega) if omega is not None else 1.0
        p.magic = float(self.magic)
        p.smagorinsky = float(self.smagorinsky)
        for e in range(3):
            p.force[e] = float(self.force[e])
            p.wall_u[e] = float(self.wall_u[e])
        p.wall_rho = float(self.wall_rho)
        return p


def NoDynamics() -> Dynamics:
    return Dynamics(_abi.DYN_NONE)


def BGKdynamics(omega: float | None = None) -> Dynamics:
    return Dynamics(_abi.DYN_BGK, omega=omega)


def TRTdynamics(omega: float | None = None, magic: float = 0.25) -> Dynamics:
    return Dynamics(_abi.DYN_TRT, omega=omega, magic=magic)


def ForcedTRTdynamics(omega: float | None = None, magic: float = 0.25, force=(0.0, 0.0, 0.0)) -> Dynamics:
    return Dynamics(_abi.DYN_FORCED_TRT, omega=omega, magic=magic, force=tuple(force))


def ForcedBGKdynamics(omega: float | None = None, force=(0.0, 0.0, 0.0)) -> Dynamics:
    return Dynamics(_abi.DYN_FORCED_BGK, omega=omega, force=tuple(force))


def SmagorinskyBGKdynamics(omega: float | None = None, smagorinsky: float = 0.1) -> Dynamics:
    return Dynamics(_abi.DYN_SMAGORINSKY, omega=omega, smagorinsky=smagorinsky)


def BounceBack(rho: float = 1.0) -> Dynamics:
    return Dynamics(_abi.DYN_BOUNCE_BACK, wall_rho=rho)


def BounceBackVelocity(u=(0.0, 0.0, 0.0), rho: float = 1.0) -> Dynamics:
    return Dynamics(_abi.DYN_BOUNCE_BACK_VELOCITY, wall_u=tuple(u), wall_rho=rho)


def InterpolatedVelocityBoundary(mixin: Dynamics, direction: int, orientation: int) -> Dynamics:
    """A flat interpolated-velocity boundary entry: ``mixin`` collision with
    BasicDirichletVelocityBoundaryTuple<direction,orientation> momenta and
    PlaneFdBoundaryProcessor3D (src/boundary/interpolatedVelocity3D.h:44-81)."""
    return Dynamics(_abi.DYN_INTERPOLATED_VELOCITY, omega=mixin.omega, magic=mixin.magic,
                    smagorinsky=mixin.smagorinsky, mixin=mixin.kind, direction=direction, orientation=orientation)


def InterpolatedPressureBoundary(mixin: Dynamics, direction: int, orientation: int) -> Dynamics:
    """A flat interpolated-pressure boundary entry (BasicDirichletPressureBoundaryTuple,
    src/boundary/interpolatedPressure3D.h:47-90)."""
    return Dynamics(_abi.DYN_INTERPOLATED_PRESSURE, omega=mixin.omega, magic=mixin.magic,
                    smagorinsky=mixin.smagorinsky, mixin=mixin.kind, direction=direction, orientation=orientation)


def LocalVelocityBoundary(mixin: Dynamics, direction: int, orientation: int) -> Dynamics:
    """boundary::LocalVelocity on a flat face (src/boundary/localVelocity3D.h:47-80):
    CombinedRLBdynamics of the mixin with regularised velocity-boundary momenta."""
    return Dynamics(_abi.DYN_LOCAL_VELOCITY, omega=mixin.omega, magic=mixin.magic,
                    smagorinsky=mixin.smagorinsky, mixin=mixin.kind, direction=direction,
                    orientation=orientation)


def LocalPressureBoundary(mixin: Dynamics, direction: int, orientation: int) -> Dynamics:
    """boundary::LocalPressure on a flat face (src/boundary/localPressure3D.h:47-57):
    CombinedRLBdynamics of the mixin with RegularizedPressureBoundaryTuple momenta
    (src/dynamics/momenta/aliases.h:136-141)."""
    return Dynamics(_abi.DYN_LOCAL_PRESSURE, omega=mixin.omega, magic=mixin.magic,
                    smagorinsky=mixin.smagorinsky, mixin=mixin.kind, direction=direction,
                    orientation=orientation)


def VelocityEdgeBoundary(mixin: Dynamics, normal) -> Dynamics:
    """External edge of a local or interpolated velocity boundary: the mixin with
    FixedVelocityBoundaryTuple momenta plus OuterVelocityEdgeProcessor3D."""
    return Dynamics(_abi.DYN_VELOCITY_EDGE, omega=mixin.omega, magic=mixin.magic,
                    smagorinsky=mixin.smagorinsky, mixin=mixin.kind, normal=tuple(int(v) for v in normal))


def VelocityCornerBoundary(mixin: Dynamics, normal) -> Dynamics:
    """External corner of a local or interpolated velocity boundary: the mixin with
    FixedVelocityBoundaryTuple momenta plus OuterVelocityCornerProcessor3D."""
    return Dynamics(_abi.DYN_VELOCITY_CORNER, omega=mixin.omega, magic=mixin.magic,
                    smagorinsky=mixin.smagorinsky, mixin=mixin.kind, normal=tuple(int(v) for v in normal))


def VelocityInnerEdgeBoundary(mixin: Dynamics, normal) -> Dynamics:
    """Internal edge of a local or interpolated velocity boundary:
    CombinedRLBdynamics of the mixin with InnerEdgeVelocityTuple3D momenta."""
    return Dynamics(_abi.DYN_VELOCITY_INNER_EDGE, omega=mixin.omega, magic=mixin.magic,
                    smagorinsky=mixin.smagorinsky, mixin=mixin.kind, normal=tuple(int(v) for v in normal))


def VelocityInnerCornerBoundary(mixin: Dynamics, normal) -> Dynamics:
    """Internal corner of a local or interpolated velocity boundary:
    CombinedRLBdynamics of the mixin with InnerCornerVelocityTuple3D momenta."""
    return Dynamics(_abi.DYN_VELOCITY_INNER_CORNER, omega=mixin.omega, magic=mixin.magic,
                    smagorinsky=mixin.smagorinsky, mixin=mixin.kind, normal=tuple(int(v) for v in normal))


# the flat-face entry of each boundary setter the facade maps
_FLAT_BOUNDARY = {
    _abi.DYN_INTERPOLATED_VELOCITY: InterpolatedVelocityBoundary,
    _abi.DYN_INTERPOLATED_PRESSURE: InterpolatedPressureBoundary,
    _abi.DYN_LOCAL_VELOCITY: LocalVelocityBoundary,
    _abi.DYN_LOCAL_PRESSURE: LocalPressureBoundary,
}

FLUID_KINDS = {_abi.DYN_BGK, _abi.DYN_TRT, _abi.DYN_SMAGORINSKY, _abi.DYN_FORCED_BGK, _abi.DYN_FORCED_TRT}

def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 (Steele, Lea, Flood, OOPSLA 2014) on uint64 arrays."""
    x = np.asarray(x, dtype=np.uint64) + np.uint64(0x9E3779B97F4A7C15)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def inlet_noise(base_u: np.ndarray, cells: np.ndarray, step: int, n_cells: int, amplitude: float,
                seed: int) -> np.ndarray:
    """The inlet velocities olb_b200_set_boundary_noise gives cells ``cells``
    (base velocities base_u, shape (k, 3)) before step ``step``."""
    base_u = np.asarray(base_u, dtype=np.float64).reshape(-1, 3)
    cells = np.asarray(cells, dtype=np.uint64).reshape(-1, 1)
    d = np.arange(3, dtype=np.uint64).reshape(1, 3)
    with np.errstate(over="ignore"):
        key = np.uint64(seed) + (np.uint64(step) * np.uint64(n_cells) + cells) * np.uint64(3) + d
        r = (splitmix64(key) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    mag = np.sqrt(np.sum(base_u * base_u, axis=1, keepdims=True))
    return base_u + amplitude * mag * (2.0 * r - 1.0)


# ---------------------------------------------------------------------------
# block-level handle


class Lattice:
    """One lattice on one GPU, driven through the C ABI."""

    def __init__(self, q: int, size, periodic=(False, False, False), storage: str = "f32",
                 device: int = 0, variant: str = "fast"):
        self._lib = _abi.load(variant)
        self.q = int(q)
        self.size = tuple(int(s) for s in size)
        self.periodic = tuple(bool(p) for p in periodic)
        self.storage = storage
        self.dtype = np.float64 if storage == "f64" else np.float32
        d = _abi.Desc()
        d.q = self.q
        d.nx, d.ny, d.nz = self.size
        for e in range(3):
            d.periodic[e] = int(self.periodic[e])
        if storage not in _abi.STORAGE:
            raise ValueError(f"unknown storage {storage!r}")
        d.storage = _abi.STORAGE[storage]
        d.device = int(device)
        h = ctypes.c_void_p()
        self._check(self._lib.olb_b200_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h

    @property
    def n(self) -> int:
        nx, ny, nz = self.size
        return nx * ny * nz

    def _check(self, status: int) -> None:
        _abi.check(self._lib, status)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.olb_b200_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - GC timing
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- configuration ------------------------------------------------------
    def set_dynamics(self, table, ids: np.ndarray | None = None, omega: float | None = None) -> None:
        params = (_abi.DynParams * len(table))()
        for k, dyn in enumerate(table):
            params[k] = dyn.params(omega)
        ptr = None
        if ids is not None:
            ids = np.ascontiguousarray(ids, dtype=np.uint8).reshape(-1)
            if ids.size != self.n:
                raise ValueError(f"ids has {ids.size} entries, lattice has {self.n} cells")
            ptr = ids.ctypes.data
        self._check(self._lib.olb_b200_set_dynamics(self._h, ptr, params, len(table)))

    def set_boundary_values(self, cells: np.ndarray, values: np.ndarray) -> None:
        """RHO and VELOCITY of interpolated boundary cells: values[j] =
        (rho, ux, uy, uz) of logical cell index cells[j]."""
        cells = np.ascontiguousarray(cells, dtype=np.int64).reshape(-1)
        values = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if values.size != 4 * cells.size:
            raise ValueError(f"{cells.size} cells need {4 * cells.size} values, got {values.size}")
        self._check(self._lib.olb_b200_set_boundary_values(self._h, cells.ctypes.data, cells.size,
                                                           values.ctypes.data))

    def set_force_field(self, force: np.ndarray | None) -> None:
        """A FORCE value per cell for the Guo-forced dynamics (``force`` of
        shape (3, cells) or (3, nx, ny, nz), the cells in population order), in
        place of their entries' constant force; None removes it
        (olb_b200_set_force_field)."""
        if force is None:
            self._check(self._lib.olb_b200_set_force_field(self._h, None))
            return
        f = np.ascontiguousarray(np.asarray(force).reshape(3, self.n), dtype=self.dtype)
        self._check(self._lib.olb_b200_set_force_field(self._h, f.ctypes.data))

    def set_boundary_noise(self, amplitude: float, seed: int = 0) -> None:
        """Per-step inlet fluctuations of relative size ``amplitude`` (see
        olb_b200_set_boundary_noise; :func:`inlet_noise` computes the same
        values on the host)."""
        self._check(self._lib.olb_b200_set_boundary_noise(self._h, float(amplitude), int(seed) & (2 ** 64 - 1)))

    def initialize(self) -> None:
        """SuperLattice::initialize: the PostStream post-processors once on the
        current state (done by the first collide_and_stream otherwise)."""
        self._check(self._lib.olb_b200_initialize(self._h))

    def set_launch_shape(self, block_z: int, block_y: int) -> None:
        self._check(self._lib.olb_b200_set_launch_shape(self._h, block_z, block_y))

    def set_step_variant(self, variant: int) -> None:
        """Select a step-kernel variant (-1: the library's default)."""
        self._check(self._lib.olb_b200_set_step_variant(self._h, int(variant)))

    def autotune(self, trial_steps: int = 0) -> dict:
        """Time every (variant, launch shape) on this lattice and keep the
        fastest; the lattice state is restored afterwards."""
        t = _abi.Tuning()
        self._check(self._lib.olb_b200_autotune(self._h, int(trial_steps), ctypes.byref(t)))
        return t.as_dict()

    def tuning(self) -> dict:
        t = _abi.Tuning()
        self._check(self._lib.olb_b200_get_tuning(self._h, ctypes.byref(t)))
        return t.as_dict()

    # -- state --------------------------------------------------------------
    def set_populations(self, pops: np.ndarray) -> None:
        pops = np.ascontiguousarray(pops, dtype=self.dtype).reshape(-1)
        if pops.size != self.q * self.n:
            raise ValueError(f"populations need {self.q * self.n} values, got {pops.size}")
        self._check(self._lib.olb_b200_set_populations(self._h, pops.ctypes.data))

    def ini_equilibrium(self, rho: np.ndarray, u: np.ndarray) -> None:
        """Every cell's populations from its density (cells) and velocity
        (3, cells): the second-order equilibrium, computed on the device
        (olb_b200_ini_equilibrium)."""
        rho = np.ascontiguousarray(rho, dtype=self.dtype).reshape(-1)
        u = np.ascontiguousarray(u, dtype=self.dtype).reshape(-1)
        if rho.size != self.n or u.size != 3 * self.n:
            raise ValueError(f"need {self.n} densities and {3 * self.n} velocity values")
        self._check(self._lib.olb_b200_ini_equilibrium(self._h, rho.ctypes.data, u.ctypes.data))

    def _out(self, arr, count):
        if arr is None:
            return np.empty(count, self.dtype)
        if arr.dtype != self.dtype or arr.size != count or not arr.flags.c_contiguous:
            raise ValueError(f"output buffer must be a contiguous {np.dtype(self.dtype).name}[{count}]")
        return arr

    def get_populations(self, out: np.ndarray | None = None) -> np.ndarray:
        out = self._out(out, self.q * self.n)
        self._check(self._lib.olb_b200_get_populations(self._h, out.ctypes.data))
        return out

    def get_moments(self, out=None):
        rho = self._out(None if out is None else out[0], self.n)
        u = self._out(None if out is None else out[1], 3 * self.n)
        self._check(self._lib.olb_b200_get_moments(self._h, rho.ctypes.data, u.ctypes.data))
        return rho, u.reshape(3, self.n)

    # -- stepping -----------------------------------------------------------
    def collide_and_stream(self, steps: int = 1, stats: bool = False):
        if stats:
            st = _abi.Stats()
            self._check(self._lib.olb_b200_collide_and_stream(self._h, int(steps), ctypes.byref(st)))
            return st.as_dict()
        self._check(self._lib.olb_b200_collide_and_stream(self._h, int(steps), None))
        return None

    def synchronize(self) -> None:
        self._check(self._lib.olb_b200_synchronize(self._h))

    def set_max_steps_in_flight(self, calls: int) -> None:
        """At most `calls` collide_and_stream calls pending on the device (0: unbounded)."""
        self._check(self._lib.olb_b200_set_max_steps_in_flight(self._h, int(calls)))

    def velocity_residual(self) -> float:
        """||u - u_prev|| / ||u|| over fluid cells since the previous call."""
        r = ctypes.c_double()
        self._check(self._lib.olb_b200_velocity_residual(self._h, ctypes.byref(r)))
        return float(r.value)

    def time_steps(self, steps: int) -> float:
        ms = ctypes.c_float()
        self._check(self._lib.olb_b200_time_steps(self._h, int(steps), ctypes.byref(ms)))
        return float(ms.value)

    def info(self) -> dict:
        sd = ctypes.c_int64()
        nb = ctypes.c_int64()
        bz = ctypes.c_int32()
        by = ctypes.c_int32()
        self._check(self._lib.olb_b200_get_info(self._h, ctypes.byref(sd), ctypes.byref(nb),
                                                ctypes.byref(bz), ctypes.byref(by)))
        return {"steps_done": sd.value, "device_bytes": nb.value, "block_z": bz.value, "block_y": by.value}

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self._lib.olb_b200_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0


# ---------------------------------------------------------------------------
# OpenLB-style facade


class SuperGeometry:
    """Material numbers of a single-cuboid domain (z fastest, as OpenLB).

    Mirrors ``SuperGeometry`` / ``BlockGeometry`` material access
    (``src/geometry/blockGeometry.h:104-121``) and
    ``CuboidDecomposition::setPeriodicity``.
    """

    def __init__(self, size, periodic=(False, False, False), material: int = 1):
        self.size = tuple(int(s) for s in size)
        self.periodic = tuple(bool(p) for p in periodic)
        self.materials = np.full(self.size, int(material), dtype=np.int32)

    def get(self, x, y, z) -> int:
        return int(self.materials[x, y, z])

    def set(self, x, y, z, material: int) -> None:
        self.materials[x, y, z] = material

    def rename(self, old: int, new: int, mask: np.ndarray | None = None) -> None:
        sel = self.materials == old
        if mask is not None:
            sel &= mask
        self.materials[sel] = new

    def getNvoxel(self) -> int:
        """Voxels with material != 0 (superGeometryStatistics3D.hh:318-328)."""
        return int(np.count_nonzero(self.materials))


def dynamics_table(materials: np.ndarray, dyn_of_material: dict, params: dict, force: dict,
                   wall_u: dict, wall_rho: dict):
    """Material numbers -> (dynamics table, per-cell uint8 ids).

    One table entry per material present, in ascending material order; a
    material without defineDynamics gets NoDynamics (the reference's default,
    core/blockLattice.hh:393-416).  Lattice-wide parameters (OMEGA, MAGIC,
    SMAGORINSKY) fill entries that do not set their own; FORCE / VELOCITY /
    RHO fields are per material, as defineField / defineU / defineRho set them.
    """
    flat = np.asarray(materials).reshape(-1)
    mats = np.unique(flat)
    if len(mats) > 256:
        raise ValueError("at most 256 distinct materials")
    table, ids, index = [], np.zeros(flat.size, np.uint8), {}
    omega = params.get("OMEGA")
    for m in (int(v) for v in mats):
        dyn = dyn_of_material.get(m, NoDynamics())
        kw = {}
        if dyn.kind in (_abi.DYN_FORCED_BGK, _abi.DYN_FORCED_TRT) and m in force:
            kw["force"] = force[m]
        if dyn.kind == _abi.DYN_BOUNCE_BACK_VELOCITY and m in wall_u:
            kw["wall_u"] = wall_u[m]
        if m in wall_rho:
            kw["wall_rho"] = wall_rho[m]
        if "MAGIC" in params:
            kw["magic"] = params["MAGIC"]
        if "SMAGORINSKY" in params:
            kw["smagorinsky"] = params["SMAGORINSKY"]
        if dyn.omega is None and omega is not None:
            kw["omega"] = omega
        if kw:
            dyn = Dynamics(**{**dyn.__dict__, **kw})
        if dyn.kind in FLUID_KINDS and dyn.omega is None:
            raise ValueError(f"material {m}: OMEGA not set")
        index[m] = len(table)
        table.append(dyn)
    for m, k in index.items():
        ids[flat == m] = k
    return table, ids


class SuperLattice:
    """The reference's ``SuperLattice<T,DESCRIPTOR>`` calls on the B200 platform."""

    def __init__(self, geometry: SuperGeometry, lattice: str | int = "D3Q19", storage: str = "f32",
                 device: int = 0, variant: str = "fast"):
        self.geometry = geometry
        self.descriptor = descriptor(lattice)
        self.block = Lattice(self.descriptor.q, geometry.size, geometry.periodic, storage, device, variant)
        self._dyn_of_material: dict[int, Dynamics] = {}
        self._params = {"OMEGA": None}
        self._force: dict[int, tuple] = {}
        self._force_field = None                  # (3, n): FORCE per cell, once a field was defined
        self._wall_u: dict[int, tuple] = {}
        self._wall_rho: dict[int, float] = {}
        self._pending_pops = np.zeros((self.descriptor.q, self.block.n), self.block.dtype)
        self._initialized = False
        self._statistics = None
        self._bc: dict[int, tuple] = {}          # material -> (kind, mixin Dynamics or None)
        self._bc_values = None                    # (4, n): RHO, VELOCITY of boundary cells

    # boundary::set<InterpolatedVelocity / InterpolatedPressure / LocalVelocity /
    # LocalPressure>(sLattice, superGeometry, material)
    def setBoundary(self, geometry: SuperGeometry, material: int, kind: int, mixin: Dynamics | None = None) -> None:
        if kind not in _FLAT_BOUNDARY:
            raise ValueError(f"unknown boundary kind {kind}")
        self._bc[int(material)] = (kind, mixin)

    def _values(self):
        if self._bc_values is None:
            self._bc_values = np.zeros((4, self.block.n))
            self._bc_values[0] = 1.0
        return self._bc_values

    def _bc_cells(self, material: int) -> np.ndarray:
        return np.flatnonzero(self.geometry.materials.reshape(-1) == int(material))

    def _push_values(self, material: int) -> None:
        if self._initialized and int(material) in self._bc:
            cells = self._bc_cells(material)
            self.block.set_boundary_values(cells, self._values()[:, cells].T)

    # defineDynamics<DYNAMICS>(superGeometry, material)  superLattice.hh:286-291
    def defineDynamics(self, geometry: SuperGeometry, material: int, dynamics: Dynamics) -> None:
        self._dyn_of_material[int(material)] = dynamics

    # setParameter<FIELD>(value)  blockLattice.h:562-572
    def setParameter(self, name: str, value: float) -> None:
        self._params[name] = float(value)

    # defineField<FORCE>(superGeometry, material, value): a constant 3-vector,
    # or a (3, nx, ny, nz) field whose values the material's cells take
    def defineForce(self, geometry: SuperGeometry, material: int, force) -> None:
        m = int(material)
        fa = np.asarray(force, dtype=np.float64)
        if fa.size == 3 and self._force_field is None:
            self._force[m] = tuple(float(f) for f in fa.reshape(3))
            return
        if self._force_field is None:
            # from now on every forced cell reads the field: seed it with the
            # constants defined so far
            self._force_field = np.zeros((3, self.block.n))
            flat = self.geometry.materials.reshape(-1)
            for mm, g in self._force.items():
                self._force_field[:, flat == mm] = np.asarray(g, np.float64)[:, None]
        cells = self._bc_cells(m)
        self._force_field[:, cells] = fa.reshape(3, 1) if fa.size == 3 else fa.reshape(3, -1)[:, cells]
        if self._initialized:
            self.block.set_force_field(self._force_field)

    # defineU(superGeometry, material, u): the VELOCITY field of moving walls,
    # or per cell on interpolated boundaries (u: a 3-vector or a (3, nx, ny, nz) field)
    def defineU(self, geometry: SuperGeometry, material: int, u) -> None:
        m = int(material)
        if m in self._bc:
            cells = self._bc_cells(m)
            ua = np.asarray(u, dtype=np.float64)
            ua = ua.reshape(3, 1) if ua.size == 3 else ua.reshape(3, -1)[:, cells]
            self._values()[1:, cells] = ua
            self._push_values(m)
            return
        self._wall_u[m] = tuple(float(v) for v in u)

    # defineRho(superGeometry, material, rho): FixedDensity RHO (walls, pressure boundaries)
    def defineRho(self, geometry: SuperGeometry, material: int, rho) -> None:
        m = int(material)
        if m in self._bc:
            cells = self._bc_cells(m)
            ra = np.asarray(rho, dtype=np.float64)
            self._values()[0, cells] = ra if ra.size == 1 else ra.reshape(-1)[cells]
            self._push_values(m)
            return
        self._wall_rho[m] = float(rho)

    # iniEquilibrium(superGeometry, material, rhoF, uF)  superLattice.hh:542-577
    def iniEquilibrium(self, geometry: SuperGeometry, material: int, rho, u) -> None:
        sel = (geometry.materials.reshape(-1) == int(material))
        n = self.block.n
        rho_a = np.broadcast_to(np.asarray(rho, dtype=self.block.dtype), (n,))
        u_a = np.asarray(u, dtype=self.block.dtype)
        if u_a.shape == (3,):
            u_a = np.broadcast_to(u_a[:, None], (3, n))
        u_a = u_a.reshape(3, n)
        feq = self.descriptor.equilibrium(rho_a[sel], u_a[:, sel], self.block.dtype)
        self._pending_pops[:, sel] = feq
        if self._initialized:
            self.block.set_populations(self._pending_pops.reshape(-1))

    def _table(self):
        table, ids = dynamics_table(self.geometry.materials, self._dyn_of_material, self._params,
                                    self._force, self._wall_u, self._wall_rho)
        # flat boundaries: one entry per material and discrete normal
        from . import boundary
        for m, (kind, mixin) in sorted(self._bc.items()):
            mix = mixin if mixin is not None else BGKdynamics()
            kw = {}
            if mix.omega is None:
                kw["omega"] = self._params.get("OMEGA")
            if "MAGIC" in self._params:
                kw["magic"] = self._params["MAGIC"]
            if "SMAGORINSKY" in self._params:
                kw["smagorinsky"] = self._params["SMAGORINSKY"]
            if kw:
                mix = Dynamics(**{**mix.__dict__, **kw})
            make = _FLAT_BOUNDARY[kind]
            for (axis, sign), cells in boundary.normal_groups(self.geometry.materials, self.geometry.periodic,
                                                              m).items():
                if len(table) >= 256:
                    raise ValueError("more than 256 dynamics entries")
                ids[cells] = len(table)
                table.append(make(mix, axis, sign))
        return table, ids

    # initialize()  superLattice.hh:190-204, blockLattice.hh:56-67
    def initialize(self) -> None:
        table, ids = self._table()
        self.block.set_dynamics(table, ids)
        if self._force_field is not None:
            self.block.set_force_field(self._force_field)
        self._initialized = True
        for m in self._bc:
            self._push_values(m)
        self.block.set_populations(self._pending_pops.reshape(-1))
        self.block.initialize()

    # collideAndStream()  superLattice.hh:601-663
    def collideAndStream(self, steps: int = 1, statistics: bool = False):
        if not self._initialized:
            self.initialize()
        self._statistics = self.block.collide_and_stream(steps, stats=statistics)
        return self._statistics

    def getStatistics(self):
        return self._statistics

    # SuperLatticeDensity3D / SuperLatticeVelocity3D  latticeVelocity3D.hh:44-71
    def getDensity(self) -> np.ndarray:
        rho, _ = self.block.get_moments()
        return rho.reshape(self.geometry.size)

    def getVelocity(self) -> np.ndarray:
        _, u = self.block.get_moments()
        return u.reshape((3,) + self.geometry.size)

    # SuperLatticePhysPressure3D (functors/lattice/latticePhysPressure3D.hh): lattice
    # pressure (rho - 1.0) / invCs2, a double expression rounded to T, then
    # UnitConverter::getPhysPressure in T (core/unitConverter.h:417-420); only rho
    # crosses PCIe
    def getPhysPressure(self, conversionPressure: float, charPhysPressure: float = 0.0) -> np.ndarray:
        rho = self.getDensity()
        dt = rho.dtype.type
        lattice_p = ((rho.astype(np.float64) - 1.0) / 3.0).astype(rho.dtype)
        return dt(conversionPressure) * lattice_p + dt(charPhysPressure)

    # SuperLatticePhysVelocity3D (functors/lattice/latticePhysVelocity3D.hh:74-85):
    # UnitConverter::getPhysVelocity = conversionVelocity * u (core/unitConverter.h:293-296)
    def getPhysVelocity(self, conversionVelocity: float) -> np.ndarray:
        u = self.getVelocity()
        return u.dtype.type(conversionVelocity) * u

    def getPopulations(self) -> np.ndarray:
        return self.block.get_populations().reshape(self.descriptor.q, -1)

    def setPopulations(self, pops: np.ndarray) -> None:
        self._pending_pops[...] = np.asarray(pops).reshape(self.descriptor.q, -1)
        if self._initialized:
            self.block.set_populations(self._pending_pops.reshape(-1))

    # -- checkpoints in OpenLB's format (openlb_b200/checkpoint.py) ----------
    def _checkpoint_fields(self, descriptor_fields):
        """The fields OpenLB's block would serialize for this set-up
        (checkpoint.setup_fields over this lattice's dynamics table and the
        boundary values defineU / defineRho gave interpolated boundaries; with
        inlet fluctuations on, those are the base values)."""
        from . import checkpoint as CK
        table, ids = self._table()
        fields, values = CK.setup_fields(self.descriptor.q, ids, table, descriptor_fields,
                                         bc_values=self._values() if self._bc else None)
        if self._force_field is not None and "FORCE" in values:
            values["FORCE"] = self._force_field.astype(values["FORCE"].dtype).reshape(values["FORCE"].shape)
        return fields, values

    # Serializable::save(fileName) (core/serializer.hh:145-149), without the
    # log-directory prefix: writes <fileName>_rank0_size1.dat
    def save(self, fileName: str, descriptor_fields=("FORCE",), overlap: int = 3) -> str:
        """Saves the lattice as OpenLB's ``SuperLattice::save`` does for a
        one-block lattice whose descriptor carries ``descriptor_fields``
        (``D3Q19<FORCE>`` by default) and whose geometry has ``overlap``
        padding layers; returns the file's path."""
        from . import checkpoint as CK
        if not self._initialized:
            self.initialize()
        fields, values = self._checkpoint_fields(descriptor_fields)
        values["POPULATION"] = self.block.get_populations().reshape(self.descriptor.q, -1)
        path = CK.file_name(fileName)
        CK.save(path, values, self.descriptor.q, self.geometry.size, self.geometry.periodic,
                self.block.dtype, overlap, fields)
        return path

    # Serializable::load(fileName) (core/serializer.hh:151-156)
    def load(self, fileName: str, descriptor_fields=("FORCE",)) -> bool:
        """Resumes from ``<fileName>_rank0_size1.dat`` written by OpenLB or by
        :meth:`save`; False when the file does not exist.  The set-up must be
        the one that wrote the file: the file's other fields are checked
        against it (ValueError if they differ)."""
        from pathlib import Path

        from . import checkpoint as CK
        path = Path(CK.file_name(fileName))
        if not path.exists():
            return False
        if not self._initialized:
            self.initialize()
        fields, expect = self._checkpoint_fields(descriptor_fields)
        arrays, _ = CK.load(path, self.descriptor.q, self.geometry.size, self.block.dtype, fields)
        for name, want in expect.items():
            got = arrays[name]
            if not np.array_equal(got, want.astype(got.dtype)):
                raise ValueError(f"checkpoint field {name} differs from this lattice's set-up")
        self._pending_pops[...] = arrays["POPULATION"]
        self.block.set_populations(self._pending_pops.reshape(-1))
        return True

    def close(self) -> None:
        self.block.close()


__all__ = [
    "Dynamics", "NoDynamics", "BGKdynamics", "TRTdynamics", "ForcedTRTdynamics", "ForcedBGKdynamics",
    "SmagorinskyBGKdynamics", "BounceBack", "BounceBackVelocity", "InterpolatedVelocityBoundary",
    "InterpolatedPressureBoundary", "Lattice", "SuperGeometry",
    "SuperLattice", "D3Q19", "D3Q27",
]
