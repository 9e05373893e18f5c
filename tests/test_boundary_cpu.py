"""Host side of the interpolated boundaries, on CPU: the discrete-normal
classification against OpenLB's own computeBoundaryTypeAndNormal
(src/geometry/discreteNormals.hh:175-1191, dumped by the reference build into
tests/golden/normals_*.npz), and the facade's table construction."""
from pathlib import Path

import numpy as np
import pytest

import openlb_b200 as ob
from openlb_b200 import _abi, boundary
from oracle import oracle as O
from tests import cases as C

GOLDEN = Path(__file__).resolve().parent / "golden"
NORMALS = sorted(p.stem for p in GOLDEN.glob("normals_*.npz"))


@pytest.mark.parametrize("name", NORMALS)
def test_flat_normals_match_reference(name):
    z = np.load(GOLDEN / f"{name}.npz")
    mats = z["materials"]
    ref = z["normals"]
    cells = np.argwhere(mats == 3)
    flat, normal = boundary.discrete_normals(mats, tuple(z["periodic"]), cells)
    nx, ny, nz = mats.shape
    idx = (cells[:, 0] * ny + cells[:, 1]) * nz + cells[:, 2]
    r_type = ref[0, idx]
    r_normal = ref[1:, idx].T
    ref_flat = (r_type == 0) & np.any(r_normal != 0, axis=1)
    assert np.array_equal(flat, ref_flat)
    assert np.array_equal(normal[flat], r_normal[flat])
    assert flat.sum() > 0


def test_fixtures_cover_edges_and_corners():
    types = set()
    for name in NORMALS:
        r = np.load(GOLDEN / f"{name}.npz")["normals"][0]
        types |= set(int(t) for t in np.unique(r[r >= 0]))
    assert {0, 1, 3, 4} <= types


def test_normal_groups_of_channel():
    case = C.interpolated_channel_case(19, (12, 8, 7), side=2)
    mats = case.dyn_id.reshape(case.size).astype(np.int32) + 1
    g_in = boundary.normal_groups(mats, (False, False, False), 3)
    g_out = boundary.normal_groups(mats, (False, False, False), 4)
    assert list(g_in) == [(0, -1)] and list(g_out) == [(0, 1)]
    assert np.array_equal(np.sort(g_in[(0, -1)]), np.flatnonzero(case.dyn_id == 2))


def test_non_flat_cells_are_rejected():
    mats = np.full((9, 8, 7), 1, np.int32)
    mats[:, 0, :] = mats[:, -1, :] = 2
    mats[0, :, :] = 3                       # the inlet's rim touches the outside
    with pytest.raises(boundary.UnsupportedBoundary, match="not a flat boundary cell"):
        boundary.normal_groups(mats, (False, False, False), 3)


def test_padding_is_outside_on_every_face():
    m = np.arange(2 * 3 * 4, dtype=np.int32).reshape(2, 3, 4) + 1
    p = boundary.padded_materials(m, (True, False, True))
    assert p.shape == (4, 5, 6)
    assert np.array_equal(p[1:-1, 1:-1, 1:-1], m)
    for axis in range(3):
        assert np.all(np.take(p, 0, axis=axis) == 0) and np.all(np.take(p, -1, axis=axis) == 0)


def test_dyn_params_layout_matches_header():
    import ctypes
    import re
    header = (Path(__file__).resolve().parents[1] / "include" / "olb_b200.h").read_text()
    body = re.search(r"typedef struct \{\n  int32_t kind;         /\* olb_b200_dyn_kind \*/(.*?)\} olb_b200_dyn_params;",
                     header, re.S).group(1)
    names = re.findall(r"^\s*(?:int32_t|double)\s+(\w+)", body, re.M)
    assert ["kind"] + names == [f for f, _ in _abi.DynParams._fields_]
    # kind, mixin, 10 doubles, direction, orientation, normal[3], reserved
    assert ctypes.sizeof(_abi.DynParams) == 4 + 4 + 8 * 10 + 4 + 4 + 3 * 4 + 4


def test_interpolated_entries_from_dynamics():
    mix = ob.SmagorinskyBGKdynamics(omega=1.7, smagorinsky=0.13)
    d = ob.InterpolatedVelocityBoundary(mix, 0, -1)
    p = d.params()
    assert (p.kind, p.mixin, p.direction, p.orientation) == (_abi.DYN_INTERPOLATED_VELOCITY, _abi.DYN_SMAGORINSKY, 0, -1)
    assert p.omega == 1.7 and p.smagorinsky == 0.13
    assert O.INTERP_VELOCITY == _abi.DYN_INTERPOLATED_VELOCITY
    assert O.INTERP_PRESSURE == _abi.DYN_INTERPOLATED_PRESSURE


def test_inlet_noise_is_splitmix64():
    from openlb_b200.lattice import inlet_noise

    def sm64(x):
        m = 2 ** 64
        x = (x + 0x9E3779B97F4A7C15) % m
        x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) % m
        x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) % m
        return x ^ (x >> 31)

    base = np.array([[0.05, 0.001, -0.002], [0.04, 0.0, 0.0]])
    cells = np.array([17, 123456789])
    got = inlet_noise(base, cells, step=7, n_cells=10 ** 9, amplitude=0.02, seed=2 ** 63 + 5)
    for j in range(2):
        mag = float(np.linalg.norm(base[j]))
        for d in range(3):
            key = (2 ** 63 + 5 + (7 * 10 ** 9 + int(cells[j])) * 3 + d) % 2 ** 64
            r = (sm64(key) >> 11) * 2.0 ** -53
            assert got[j, d] == base[j, d] + 0.02 * mag * (2 * r - 1)
