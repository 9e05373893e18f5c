"""ctypes binding of the C ABI in ``include/olb_b200.h``.

The shared library is built in-tree (``openlb_b200/libolb_b200.so``).  There is
no fallback: if the library is missing or cannot be loaded, every entry point
raises :class:`LibraryNotBuilt`.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent

LIBRARIES = {
    "fast": PKG_DIR / "libolb_b200.so",
    # same kernels built with -fmad=false; used to show operation-for-operation parity
    "exact": PKG_DIR / "libolb_b200_exact.so",
}

# status codes (olb_b200_status)
OK, ERR_CUDA, ERR_OOM, ERR_ARG, ERR_DIVERGED, ERR_TIMEOUT, ERR_UNSUPPORTED = range(7)
STATUS_NAMES = {
    OK: "OK", ERR_CUDA: "ERR_CUDA", ERR_OOM: "ERR_OOM", ERR_ARG: "ERR_ARG",
    ERR_DIVERGED: "ERR_DIVERGED", ERR_TIMEOUT: "ERR_TIMEOUT", ERR_UNSUPPORTED: "ERR_UNSUPPORTED",
}

# storage (olb_b200_storage)
STORAGE = {"f32": 0, "f64": 1, "f16": 2, "bf16": 3}

# dynamics kinds (olb_b200_dyn_kind)
DYN_NONE, DYN_BGK, DYN_TRT, DYN_SMAGORINSKY, DYN_BOUNCE_BACK, DYN_BOUNCE_BACK_VELOCITY, \
    DYN_FORCED_BGK, DYN_FORCED_TRT, DYN_INTERPOLATED_VELOCITY, DYN_INTERPOLATED_PRESSURE, \
    DYN_LOCAL_VELOCITY, DYN_VELOCITY_EDGE, DYN_VELOCITY_CORNER, DYN_VELOCITY_INNER_EDGE, \
    DYN_VELOCITY_INNER_CORNER, DYN_LOCAL_PRESSURE = range(16)
DYN_INTERPOLATED = (DYN_INTERPOLATED_VELOCITY, DYN_INTERPOLATED_PRESSURE)
# boundary kinds whose cells carry values (RHO, VELOCITY) set by set_boundary_values
DYN_VALUED = (DYN_INTERPOLATED_VELOCITY, DYN_INTERPOLATED_PRESSURE, DYN_LOCAL_VELOCITY,
              DYN_VELOCITY_EDGE, DYN_VELOCITY_CORNER, DYN_VELOCITY_INNER_EDGE, DYN_VELOCITY_INNER_CORNER,
              DYN_LOCAL_PRESSURE)
ABI_VERSION = 3

EXPORTED = [
    "olb_b200_create", "olb_b200_destroy", "olb_b200_set_dynamics", "olb_b200_set_populations",
    "olb_b200_get_populations", "olb_b200_collide_and_stream", "olb_b200_get_moments",
    "olb_b200_synchronize", "olb_b200_time_steps", "olb_b200_get_stream", "olb_b200_get_info",
    "olb_b200_set_launch_shape", "olb_b200_last_error", "olb_b200_abi_version",
    "olb_b200_build_info", "olb_b200_collide_and_stream_noalloc", "olb_b200_autotune",
    "olb_b200_get_tuning", "olb_b200_set_step_variant", "olb_b200_velocity_residual",
    "olb_b200_ensemble_create", "olb_b200_ensemble_destroy", "olb_b200_ensemble_add",
    "olb_b200_ensemble_remove", "olb_b200_ensemble_run", "olb_b200_ensemble_get_moments",
    "olb_b200_ensemble_info", "olb_b200_ensemble_set_occupancy", "olb_b200_ensemble_bytes_per_instance",
    "olb_b200_set_boundary_values", "olb_b200_initialize", "olb_b200_set_boundary_noise",
    "olb_b200_set_max_steps_in_flight", "olb_b200_set_force_field", "olb_b200_ini_equilibrium",
]

ENSEMBLE_CAVITY, ENSEMBLE_CHANNEL, ENSEMBLE_GEOMETRY = 1, 2, 3


class LibraryNotBuilt(RuntimeError):
    pass


class OlbError(RuntimeError):
    """A non-OK status from the library; ``status`` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Diverged(OlbError):
    pass


class Desc(ctypes.Structure):
    _fields_ = [("q", ctypes.c_int32), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
                ("nz", ctypes.c_int32), ("periodic", ctypes.c_int32 * 3),
                ("storage", ctypes.c_int32), ("device", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 3)]


class DynParams(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("mixin", ctypes.c_int32),
                ("omega", ctypes.c_double), ("magic", ctypes.c_double),
                ("smagorinsky", ctypes.c_double), ("force", ctypes.c_double * 3),
                ("wall_u", ctypes.c_double * 3), ("wall_rho", ctypes.c_double),
                ("direction", ctypes.c_int32), ("orientation", ctypes.c_int32),
                ("normal", ctypes.c_int32 * 3), ("reserved", ctypes.c_int32)]


class Stats(ctypes.Structure):
    _fields_ = [("sum_rho", ctypes.c_double), ("sum_usqr", ctypes.c_double),
                ("max_usqr", ctypes.c_double), ("n_cells", ctypes.c_int64),
                ("average_rho", ctypes.c_double), ("average_energy", ctypes.c_double),
                ("max_u", ctypes.c_double), ("n_nonfinite", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Tuning(ctypes.Structure):
    _fields_ = [("variant", ctypes.c_int32), ("cells_per_thread", ctypes.c_int32),
                ("min_blocks_per_sm", ctypes.c_int32), ("block_z", ctypes.c_int32),
                ("block_y", ctypes.c_int32), ("tuned", ctypes.c_int32), ("candidates", ctypes.c_int32),
                ("ms_per_step", ctypes.c_float)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class EnsembleDesc(ctypes.Structure):
    _fields_ = [("q", ctypes.c_int32), ("storage", ctypes.c_int32), ("device", ctypes.c_int32),
                ("max_instances", ctypes.c_int32), ("pool_bytes", ctypes.c_uint64)]


class InstanceDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
                ("nz", ctypes.c_int32), ("omega", ctypes.c_double), ("wall_u", ctypes.c_double * 3),
                ("force", ctypes.c_double * 3), ("cells", ctypes.c_void_p)]


_loaded: dict = {}


def library_path(variant: str = "fast") -> Path:
    override = os.environ.get("OLB_B200_LIBRARY")
    if override and variant == "fast":
        return Path(override)
    return LIBRARIES[variant]


def load(variant: str = "fast") -> ctypes.CDLL:
    """Load (once) and return the library; raises LibraryNotBuilt."""
    if variant in _loaded:
        return _loaded[variant]
    path = library_path(variant)
    if not path.exists():
        raise LibraryNotBuilt(f"{path} is not built (run __graft_entry__.build() or "
                              f"make -C openlb_b200/csrc)")
    try:
        lib = ctypes.CDLL(str(path))
    except OSError as e:  # pragma: no cover - depends on the host
        raise LibraryNotBuilt(f"cannot load {path}: {e}") from e
    P = ctypes.c_void_p
    st = ctypes.c_int
    lib.olb_b200_create.argtypes = [ctypes.POINTER(Desc), ctypes.POINTER(P)]
    lib.olb_b200_create.restype = st
    lib.olb_b200_destroy.argtypes = [P]
    lib.olb_b200_destroy.restype = None
    lib.olb_b200_set_dynamics.argtypes = [P, P, ctypes.POINTER(DynParams), ctypes.c_int32]
    lib.olb_b200_set_dynamics.restype = st
    lib.olb_b200_set_populations.argtypes = [P, P]
    lib.olb_b200_set_populations.restype = st
    lib.olb_b200_ini_equilibrium.argtypes = [P, P, P]
    lib.olb_b200_ini_equilibrium.restype = st
    lib.olb_b200_get_populations.argtypes = [P, P]
    lib.olb_b200_get_populations.restype = st
    lib.olb_b200_collide_and_stream.argtypes = [P, ctypes.c_int32, ctypes.POINTER(Stats)]
    lib.olb_b200_collide_and_stream.restype = st
    lib.olb_b200_get_moments.argtypes = [P, P, P]
    lib.olb_b200_get_moments.restype = st
    lib.olb_b200_synchronize.argtypes = [P]
    lib.olb_b200_synchronize.restype = st
    lib.olb_b200_set_max_steps_in_flight.argtypes = [P, ctypes.c_int32]
    lib.olb_b200_set_max_steps_in_flight.restype = st
    lib.olb_b200_set_force_field.argtypes = [P, ctypes.c_void_p]
    lib.olb_b200_set_force_field.restype = st
    lib.olb_b200_time_steps.argtypes = [P, ctypes.c_int32, ctypes.POINTER(ctypes.c_float)]
    lib.olb_b200_time_steps.restype = st
    lib.olb_b200_get_stream.argtypes = [P, ctypes.POINTER(P)]
    lib.olb_b200_get_stream.restype = st
    lib.olb_b200_get_info.argtypes = [P, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    lib.olb_b200_get_info.restype = st
    lib.olb_b200_set_launch_shape.argtypes = [P, ctypes.c_int32, ctypes.c_int32]
    lib.olb_b200_set_launch_shape.restype = st
    lib.olb_b200_collide_and_stream_noalloc.argtypes = [ctypes.POINTER(Desc), P, ctypes.c_int64,
                                                        ctypes.POINTER(DynParams), ctypes.c_int32,
                                                        ctypes.POINTER(Stats), P]
    lib.olb_b200_collide_and_stream_noalloc.restype = st
    lib.olb_b200_autotune.argtypes = [P, ctypes.c_int32, ctypes.POINTER(Tuning)]
    lib.olb_b200_autotune.restype = st
    lib.olb_b200_get_tuning.argtypes = [P, ctypes.POINTER(Tuning)]
    lib.olb_b200_get_tuning.restype = st
    lib.olb_b200_set_step_variant.argtypes = [P, ctypes.c_int32]
    lib.olb_b200_set_step_variant.restype = st
    lib.olb_b200_velocity_residual.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
    lib.olb_b200_velocity_residual.restype = st
    lib.olb_b200_ensemble_create.argtypes = [ctypes.POINTER(EnsembleDesc), ctypes.POINTER(P)]
    lib.olb_b200_ensemble_create.restype = st
    lib.olb_b200_ensemble_destroy.argtypes = [P]
    lib.olb_b200_ensemble_destroy.restype = None
    lib.olb_b200_ensemble_add.argtypes = [P, ctypes.POINTER(InstanceDesc), ctypes.POINTER(ctypes.c_int32)]
    lib.olb_b200_ensemble_add.restype = st
    lib.olb_b200_ensemble_remove.argtypes = [P, ctypes.c_int32]
    lib.olb_b200_ensemble_remove.restype = st
    lib.olb_b200_ensemble_run.argtypes = [P, ctypes.c_int32, ctypes.c_int32, P, P]
    lib.olb_b200_ensemble_run.restype = st
    lib.olb_b200_ensemble_get_moments.argtypes = [P, ctypes.c_int32, P, P]
    lib.olb_b200_ensemble_get_moments.restype = st
    lib.olb_b200_ensemble_info.argtypes = [P, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_int32)]
    lib.olb_b200_ensemble_info.restype = st
    lib.olb_b200_ensemble_set_occupancy.argtypes = [P, ctypes.c_int32]
    lib.olb_b200_ensemble_set_occupancy.restype = st
    lib.olb_b200_ensemble_bytes_per_instance.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    lib.olb_b200_ensemble_bytes_per_instance.restype = ctypes.c_uint64
    lib.olb_b200_set_boundary_values.argtypes = [P, P, ctypes.c_int64, P]
    lib.olb_b200_set_boundary_values.restype = st
    lib.olb_b200_set_boundary_noise.argtypes = [P, ctypes.c_double, ctypes.c_uint64]
    lib.olb_b200_set_boundary_noise.restype = st
    lib.olb_b200_initialize.argtypes = [P]
    lib.olb_b200_initialize.restype = st
    lib.olb_b200_last_error.argtypes = []
    lib.olb_b200_last_error.restype = ctypes.c_char_p
    lib.olb_b200_abi_version.argtypes = []
    lib.olb_b200_abi_version.restype = ctypes.c_int32
    lib.olb_b200_build_info.argtypes = []
    lib.olb_b200_build_info.restype = ctypes.c_char_p
    _loaded[variant] = lib
    return lib


def check(lib: ctypes.CDLL, status: int) -> None:
    """Raise on a non-OK status, like OpenLB's device::check() (device.hh:48-62)."""
    if status == OK:
        return
    msg = lib.olb_b200_last_error().decode(errors="replace")
    if status == ERR_DIVERGED:
        raise Diverged(status, msg)
    raise OlbError(status, msg)
