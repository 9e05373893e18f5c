"""Checkpoints in OpenLB's own file format, so that a run can move between
OpenLB and this library in either direction.

OpenLB saves a ``SuperLattice`` through its ``Serializable`` interface
(core/serializer.hh:64-111, io/serializerIO.hh:40-64):

* the file ``<name>_rank<r>_size<n>.dat`` (io/fileName.hh:51-63) holds two
  base64 streams back to back (io/base64.hh:45-124, standard alphabet, each
  padded with ``=`` on its own): the payload size as one little-endian
  ``std::size_t``, then the payload;
* the payload walks the lattice's blocks in order; each block
  (core/blockLattice.hh:597-617) walks its serialized field arrays in the
  order of a ``std::map`` keyed by ``typeid(Array<FIELD>).name()``
  (core/data.h:431,520-525, core/data.hh:52-62), i.e. sorted by the mangled
  type name; a field array is one column per component
  (core/columnVector.h:155-177);
* a column is ``count`` (``std::size_t``) followed by ``count`` values of T
  (cpu/sisd/column.hh:39-63); a cyclic column, which POPULATION uses, is
  ``shift`` (``std::ptrdiff_t``), ``count`` and the raw buffer
  (cpu/sisd/column.hh:67-90), whose logical element i sits at raw index
  ``(i + shift) mod count`` (cpu/sisd/column.h:162-190);
* a block covers its core cells plus ``overlap`` padding layers on every side,
  z fastest (core/blockStructure.h:65-75,150).

Which fields a block serializes depends on the descriptor (every descriptor
field, core/blockLattice.hh:400-411) and on the fields the set-up allocated
(core/blockLattice.hh:438-452).  ``lattice_fields`` builds that list for the
lattices this library runs; ``FIELD_KEYS`` holds each field's type name.

On load the POPULATION columns of the core cells become the lattice's state;
the other fields are returned so the caller can check them against its own
set-up.  On save the populations are written with shift 0, the overlap cells
of periodic directions hold their periodic images and the others the rest
state (0 in OpenLB's shifted storage).  OpenLB overwrites the periodic overlap
after the next collision (core/superLattice.hh:630-632) and the core cells
never read a non-periodic overlap cell that is not a wall, so either side
continues from the file exactly as it would have from its own state.
"""
from __future__ import annotations

import base64
import struct
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _abi

# typeid(olb::Array<FIELD>).name() under the Itanium C++ ABI (g++ and clang on
# Linux) for the fields these lattices serialize:
#   POPULATION, FORCE, VELOCITY  olb::descriptors (descriptor/fields.h:315-339);
#                                VELOCITY is what defineU writes for moving walls
#   RHO                          olb::momenta::FixedDensity::RHO
#                                (dynamics/momenta/elements.h:238): the density of
#                                bounce-back walls and interpolated pressure cells
#   BC_VELOCITY                  olb::momenta::FixedVelocityMomentumGeneric::VELOCITY
#                                (elements.h:529): interpolated velocity cells
#   PRESSURE_VELOCITY_<d><+|->   olb::momenta::FixedPressureMomentum<d,o>::VELOCITY:
#                                interpolated pressure cells of outward normal (d, o)
FIELD_KEYS = {
    "POPULATION": "N3olb5ArrayINS_11descriptors10POPULATIONEEE",
    "FORCE": "N3olb5ArrayINS_11descriptors5FORCEEEE",
    "VELOCITY": "N3olb5ArrayINS_11descriptors8VELOCITYEEE",
    "RHO": "N3olb5ArrayINS_7momenta12FixedDensity3RHOEEE",
    "BC_VELOCITY": "N3olb5ArrayINS_7momenta28FixedVelocityMomentumGeneric8VELOCITYEEE",
}
_COMPONENTS = {"FORCE": 3, "VELOCITY": 3, "RHO": 1, "BC_VELOCITY": 3}


def pressure_velocity_field(direction: int, orientation: int) -> str:
    return f"PRESSURE_VELOCITY_{int(direction)}{'+' if orientation > 0 else '-'}"


def field_key(name: str) -> str:
    if name in FIELD_KEYS:
        return FIELD_KEYS[name]
    if name.startswith("PRESSURE_VELOCITY_") and len(name) == 20 and name[18] in "012" and name[19] in "+-":
        o = "1" if name[19] == "+" else "n1"      # template argument -1 mangles as Lin1E
        return f"N3olb5ArrayINS_7momenta21FixedPressureMomentumILi{name[18]}ELi{o}EE8VELOCITYEEE"
    raise ValueError(f"unknown field {name!r}")


@dataclass(frozen=True)
class FieldSpec:
    name: str
    components: int
    cyclic: bool = False

    @property
    def key(self) -> str:
        return field_key(self.name)


def lattice_fields(q: int, descriptor_fields=(), extra_fields=()) -> list[FieldSpec]:
    """Serialized fields of a block in file order: POPULATION (q cyclic columns),
    the descriptor's own fields (e.g. ``("FORCE",)`` for ``D3Q19<FORCE>``) and
    the fields the set-up allocated, sorted by their type names."""
    names = {"POPULATION", *descriptor_fields, *extra_fields}
    specs = []
    for n in names:
        field_key(n)
        comps = q if n == "POPULATION" else _COMPONENTS.get(n, 3)
        specs.append(FieldSpec(n, comps, cyclic=(n == "POPULATION")))
    return sorted(specs, key=lambda s: s.key)


_FORCED = (_abi.DYN_FORCED_BGK, _abi.DYN_FORCED_TRT)
_WALLS = (_abi.DYN_BOUNCE_BACK, _abi.DYN_BOUNCE_BACK_VELOCITY)
_MOVING_WALL = _abi.DYN_BOUNCE_BACK_VELOCITY


def setup_fields(q: int, ids: np.ndarray, table, descriptor_fields=("FORCE",), bc_values=None):
    """The fields OpenLB's block serializes for a set-up given as a per-cell
    dynamics id and its table (entries with ``kind``, ``force``, ``wall_u``,
    ``wall_rho``, ``direction``, ``orientation``), with their values on the core
    cells: FORCE where defineField<FORCE> set the force of a forced dynamics,
    descriptors::VELOCITY where defineU set a moving wall, the FixedDensity RHO
    of bounce-back walls (their wall density) and of interpolated pressure
    cells, and the momenta VELOCITY fields of interpolated velocity and
    pressure cells (``bc_values``: float[4][cells], the rho, u boundary values).
    Returns (field specs in file order, {name: array[components, cells]})."""
    ids = np.asarray(ids).reshape(-1)
    n = ids.size
    kinds = [int(d.kind) for d in table]
    if any(k in _abi.DYN_INTERPOLATED for k in kinds) and bc_values is None:
        raise ValueError("interpolated boundaries need their boundary values")
    values = {}

    def field(name, comps):
        if name not in values:
            values[name] = np.zeros((comps, n))
        return values[name]

    if "FORCE" in descriptor_fields:
        field("FORCE", 3)
    for k, d in enumerate(table):
        sel = ids == k
        if kinds[k] in _FORCED and "FORCE" in descriptor_fields:
            values["FORCE"][:, sel] = np.asarray(d.force, np.float64)[:, None]
        if kinds[k] == _MOVING_WALL:
            field("VELOCITY", 3)[:, sel] = np.asarray(d.wall_u, np.float64)[:, None]
        if kinds[k] in _WALLS:
            field("RHO", 1)[0, sel] = d.wall_rho
        if kinds[k] == _abi.DYN_INTERPOLATED_VELOCITY:
            field("BC_VELOCITY", 3)[:, sel] = np.asarray(bc_values)[1:4, sel]
        if kinds[k] == _abi.DYN_INTERPOLATED_PRESSURE:
            field("RHO", 1)[0, sel] = np.asarray(bc_values)[0, sel]
            field(pressure_velocity_field(d.direction, d.orientation), 3)[:, sel] = np.asarray(bc_values)[1:4, sel]
    extra = tuple(k for k in values if k not in descriptor_fields)
    return lattice_fields(q, tuple(descriptor_fields), extra), values


def padded_shape(size, overlap: int) -> tuple[int, int, int]:
    return tuple(int(s) + 2 * int(overlap) for s in size)


def overlap_of(size, count: int, max_overlap: int = 16) -> int:
    """The padding width whose padded block holds ``count`` cells."""
    for o in range(max_overlap + 1):
        if int(np.prod(padded_shape(size, o))) == count:
            return o
    raise ValueError(f"a block of {count} cells does not pad {tuple(size)} by 0..{max_overlap} layers")


# -- file level -------------------------------------------------------------
def encode(payload: bytes) -> bytes:
    """Serializer's file text for a payload (io/serializerIO.hh:40-64)."""
    return base64.b64encode(struct.pack("<Q", len(payload))) + base64.b64encode(payload)


def decode(text: bytes) -> bytes:
    """The payload of Serializer's file text; checks the recorded size."""
    text = bytes(text).strip()
    if len(text) < 12:
        raise ValueError("checkpoint too short")
    (size,) = struct.unpack("<Q", base64.b64decode(text[:12], validate=True))
    body = base64.b64decode(text[12:], validate=True)
    if len(body) != size:
        raise ValueError(f"checkpoint payload has {len(body)} bytes, its header says {size}")
    return body


def file_name(name: str, rank: int = 0, size: int = 1) -> str:
    """createParallelFileName + ".dat" (io/fileName.hh:51-63; core/serializer.hh:130-136)."""
    return f"{name}_rank{rank}_size{size}.dat"


# -- payload level ----------------------------------------------------------
def parse_block(payload: bytes, fields: list[FieldSpec], dtype, offset: int = 0):
    """Reads one block; returns ({field: array[components, count]} in the logical
    cell order, the offset after the block)."""
    dtype = np.dtype(dtype)
    out = {}
    pos = offset
    for spec in fields:
        cols = []
        for _ in range(spec.components):
            shift = 0
            if spec.cyclic:
                (shift,) = struct.unpack_from("<q", payload, pos)
                pos += 8
            (count,) = struct.unpack_from("<Q", payload, pos)
            pos += 8
            nbytes = count * dtype.itemsize
            if pos + nbytes > len(payload):
                raise ValueError(f"checkpoint ends inside field {spec.name}")
            raw = np.frombuffer(payload, dtype=dtype, count=count, offset=pos)
            pos += nbytes
            if spec.cyclic and count:
                if not -int(count) < shift < int(count):
                    raise ValueError(f"{spec.name}: shift {shift} out of range for {count} cells")
                raw = np.roll(raw, -shift)
            cols.append(np.array(raw))
        counts = {c.size for c in cols}
        if len(counts) != 1:
            raise ValueError(f"{spec.name}: columns of different lengths")
        out[spec.name] = np.stack(cols)
    return out, pos


def write_block(fields: list[FieldSpec], arrays: dict, dtype) -> bytes:
    """One block with every cyclic column at shift 0."""
    dtype = np.dtype(dtype)
    parts = []
    for spec in fields:
        a = np.ascontiguousarray(arrays[spec.name], dtype=dtype)
        if a.ndim != 2 or a.shape[0] != spec.components:
            raise ValueError(f"{spec.name}: expected {spec.components} columns, got shape {a.shape}")
        for col in a:
            if spec.cyclic:
                parts.append(struct.pack("<q", 0))
            parts.append(struct.pack("<Q", col.size))
            parts.append(col.tobytes())
    return b"".join(parts)


def core_view(padded: np.ndarray, size, overlap: int) -> np.ndarray:
    """[components, padded cells] -> [components, core cells] (z fastest)."""
    o = int(overlap)
    px, py, pz = padded_shape(size, o)
    nx, ny, nz = (int(s) for s in size)
    a = padded.reshape(-1, px, py, pz)[:, o:o + nx, o:o + ny, o:o + nz]
    return np.ascontiguousarray(a).reshape(a.shape[0], -1)


def pad_cells(core: np.ndarray, size, overlap: int, periodic, fill=0.0) -> np.ndarray:
    """[components, core cells] -> [components, padded cells]; periodic axes
    wrap, the others hold ``fill``."""
    o = int(overlap)
    nx, ny, nz = (int(s) for s in size)
    a = core.reshape(-1, nx, ny, nz)
    for axis, per in enumerate(periodic):
        width = [(0, 0)] * 4
        width[axis + 1] = (o, o)
        a = np.pad(a, width, mode="wrap") if per else np.pad(a, width, mode="constant", constant_values=fill)
    return np.ascontiguousarray(a).reshape(a.shape[0], -1)


def load_bytes(text: bytes, q: int, size, dtype, fields: list[FieldSpec] | None = None):
    """Reads a one-block checkpoint's file text; returns (fields on the core
    cells, overlap).  ``fields`` defaults to POPULATION alone; the file must
    hold exactly the listed fields."""
    fields = fields if fields is not None else lattice_fields(q)
    payload = decode(text)
    arrays, end = parse_block(payload, fields, dtype)
    if end != len(payload):
        raise ValueError(f"checkpoint holds {len(payload) - end} bytes after the listed fields "
                         f"{[f.name for f in fields]}: the set-up that wrote it allocated other fields")
    count = arrays["POPULATION"].shape[1]
    overlap = overlap_of(size, count)
    return {k: core_view(v, size, overlap) for k, v in arrays.items()}, overlap


def encode_fields(core_fields: dict, q: int, size, periodic, dtype, overlap: int,
                  fields: list[FieldSpec] | None = None) -> bytes:
    """The file text of a one-block checkpoint from fields on the core cells."""
    fields = fields if fields is not None else lattice_fields(q)
    padded = {}
    for spec in fields:
        a = np.asarray(core_fields[spec.name], dtype=np.dtype(dtype)).reshape(spec.components, -1)
        padded[spec.name] = pad_cells(a, size, overlap, periodic)
    return encode(write_block(fields, padded, dtype))


def load(path, q: int, size, dtype, fields: list[FieldSpec] | None = None):
    """``load_bytes`` of a file."""
    return load_bytes(Path(path).read_bytes(), q, size, dtype, fields)


def save(path, core_fields: dict, q: int, size, periodic, dtype, overlap: int,
         fields: list[FieldSpec] | None = None) -> None:
    """Writes ``encode_fields`` to a file."""
    Path(path).write_bytes(encode_fields(core_fields, q, size, periodic, dtype, overlap, fields))


__all__ = ["FIELD_KEYS", "FieldSpec", "field_key", "pressure_velocity_field", "lattice_fields", "setup_fields", "encode", "decode", "file_name",
           "parse_block", "write_block", "core_view", "pad_cells", "load_bytes", "encode_fields", "load", "save",
           "overlap_of"]
