"""Boundary setters on the B200 platform: interpolated and local velocity /
pressure boundaries.

Mirrors ``boundary::set<boundary::InterpolatedVelocity>(sLattice, superGeometry,
material)`` and ``...<InterpolatedPressure>``, ``<LocalVelocity>``,
``<LocalPressure>`` (``src/boundary/setBoundary.h:79-157``): every cell of the
material gets a discrete normal from the fluid cells (material 1) and the
outside cells (material 0) around it (``computeBoundaryTypeAndNormal``,
``src/geometry/discreteNormals.hh:175-1191``), and from that its dynamics — the
mixin collision with the boundary's momenta and the ``PlaneFdBoundaryProcessor3D``
post-processor (``src/boundary/interpolatedVelocity3D.h:44-81``,
``src/boundary/interpolatedPressure3D.h:47-90``), or ``CombinedRLBdynamics``
with regularised momenta and no post-processor
(``src/boundary/localVelocity3D.h:47-80``, ``src/boundary/localPressure3D.h:47-57``).

This build provides the flat-face type.  A boundary cell is flat when the four
cells around it within one axis plane are neither fluid nor outside and a
neighbour along that axis is fluid; the reference tests the axes x, y, z in
that order and, per axis, the fluid neighbour at +1 before the one at -1, and
the first match is the result (no later edge or corner test can replace it:
those need a second fluid face neighbour, or only fill an empty normal).  Cells
of other types (edges and corners of an inlet that is not bounded by walls)
raise :class:`UnsupportedBoundary`.
"""
from __future__ import annotations

import numpy as np

from . import _abi

FLAT = 0

InterpolatedVelocity = _abi.DYN_INTERPOLATED_VELOCITY
InterpolatedPressure = _abi.DYN_INTERPOLATED_PRESSURE
LocalVelocity = _abi.DYN_LOCAL_VELOCITY
LocalPressure = _abi.DYN_LOCAL_PRESSURE


class UnsupportedBoundary(ValueError):
    """A boundary cell whose discrete normal is not of the flat type."""


def padded_materials(materials: np.ndarray, periodic=None) -> np.ndarray:
    """Materials with one layer around the domain as the classification sees
    it: material 0 (outside) on every face, periodic or not — the reference's
    own dumps (tests/golden/normals_open_face.npz) show that a face cell of a
    periodic axis does not see the periodic image as its neighbour here."""
    return np.pad(np.asarray(materials), 1, mode="constant", constant_values=0)


def discrete_normals(materials: np.ndarray, periodic, cells: np.ndarray, fluid: int = 1,
                     outside: int = 0):
    """Discrete normal of each cell in ``cells`` (an (k, 3) array of x, y, z).

    Returns ``(flat, normal)``: a boolean per cell (flat type found) and the
    outward normal (k, 3) of the flat ones (zeros elsewhere)."""
    pad = padded_materials(materials, periodic)
    is_fluid = pad == fluid
    is_bnd = (pad != fluid) & (pad != outside)
    cells = np.asarray(cells, dtype=np.int64).reshape(-1, 3)
    p = cells + 1
    k = len(cells)
    flat = np.zeros(k, bool)
    normal = np.zeros((k, 3), np.int32)

    def at(mask, off):
        return mask[p[:, 0] + off[0], p[:, 1] + off[1], p[:, 2] + off[2]]

    self_bnd = at(is_bnd, (0, 0, 0))
    for axis in range(3):
        t1, t2 = [a for a in range(3) if a != axis]
        tang = self_bnd.copy()
        for t in (t1, t2):
            for s in (1, -1):
                off = [0, 0, 0]
                off[t] = s
                tang &= at(is_bnd, off)
        for s in (1, -1):          # fluid at +1 first: outward normal -1
            off = [0, 0, 0]
            off[axis] = s
            hit = tang & ~flat & at(is_fluid, off)
            normal[hit, axis] = -s
            flat |= hit
    return flat, normal


def normal_groups(materials: np.ndarray, periodic, material: int):
    """Cells of ``material`` grouped by outward normal: {(axis, sign): flat cell indices}."""
    m = np.asarray(materials)
    xyz = np.argwhere(m == material)
    if len(xyz) == 0:
        return {}
    flat, normal = discrete_normals(m, periodic, xyz)
    if not flat.all():
        bad = xyz[~flat][0]
        raise UnsupportedBoundary(
            f"material {material}: cell {tuple(int(v) for v in bad)} is not a flat boundary cell "
            f"({int((~flat).sum())} such cells); edge and corner boundary cells are not supported")
    nx, ny, nz = m.shape
    index = (xyz[:, 0] * ny + xyz[:, 1]) * nz + xyz[:, 2]
    groups = {}
    for axis in range(3):
        for sign in (-1, 1):
            sel = normal[:, axis] == sign
            if sel.any():
                groups[(axis, sign)] = index[sel]
    return groups


def set(lattice, geometry, material: int, kind: int = InterpolatedVelocity, mixin=None) -> None:
    """``boundary::set<BC>(sLattice, superGeometry, material)`` on a
    :class:`openlb_b200.lattice.SuperLattice`; ``mixin`` is the MixinDynamics
    template argument (the reference's default: BGKdynamics)."""
    lattice.setBoundary(geometry, material, kind, mixin)


__all__ = ["InterpolatedVelocity", "InterpolatedPressure", "LocalVelocity", "LocalPressure",
           "UnsupportedBoundary", "discrete_normals", "normal_groups", "padded_materials", "set"]
