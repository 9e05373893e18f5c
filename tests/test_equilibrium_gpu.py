"""olb_b200_ini_equilibrium: every cell's populations from its density and
velocity, expanded on the device — OpenLB's iniEquilibrium
(src/core/superLattice.hh:542-577) with equilibrium::secondOrder
(src/dynamics/lbm.h:50-64), the oracle's oracle_equilibrium.

Tolerances: the exact build is bit-identical to the oracle's equilibrium
(FP32, FP64); the fast build (FMA contraction) within 1e-6 of the unshifted
population (FP32) / 1e-14 (FP64); 16-bit storage within one storage rounding
of the FP32 values set through set_populations.
"""
import numpy as np
import pytest

import openlb_b200 as ob
from oracle import oracle as O
from tests import cases as C

pytestmark = pytest.mark.gpu


def fields(n, dtype, seed):
    rng = np.random.default_rng(seed)
    rho = (1 + 0.02 * rng.standard_normal(n)).astype(dtype)
    u = (0.05 * rng.standard_normal((3, n))).astype(dtype)
    return rho, u


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("storage", ["f32", "f64"])
@pytest.mark.parametrize("variant", ["exact", "fast"])
def test_matches_oracle_equilibrium(q, storage, variant):
    dtype = np.float64 if storage == "f64" else np.float32
    size = (9, 7, 6)
    n = int(np.prod(size))
    rho, u = fields(n, dtype, q)
    ref = O.equilibrium(q, rho, u)
    with ob.Lattice(q, size, (True, True, True), storage=storage, variant=variant) as lat:
        lat.set_dynamics([ob.BGKdynamics(omega=1.2)])
        lat.collide_and_stream(3)          # odd parity: the call resets the layout
        lat.ini_equilibrium(rho, u)
        got = lat.get_populations()
    if variant == "exact":
        assert np.array_equal(got, ref)
    else:
        tol = 1e-14 if storage == "f64" else 1e-6
        rel, _ = C.pop_tolerance_violation(q, got, ref, tol)
        assert rel <= tol, rel


@pytest.mark.parametrize("storage", ["f16", "bf16"])
@pytest.mark.parametrize("nx", [8, 7])
def test_16bit_storage_matches_uploaded_equilibrium(storage, nx):
    """Paired layout (nx even) and one cell per element (nx odd)."""
    size = (nx, 6, 5)
    n = int(np.prod(size))
    rho, u = fields(n, np.float32, nx)
    with ob.Lattice(19, size, (True, True, True), storage=storage, variant="exact") as lat:
        lat.set_dynamics([ob.BGKdynamics(omega=1.2)])
        lat.set_populations(O.equilibrium(19, rho, u))
        uploaded = lat.get_populations()
        lat.ini_equilibrium(rho, u)
        got = lat.get_populations()
    assert np.array_equal(got, uploaded)


def test_then_steps_like_uploaded_state():
    size = (16, 12, 10)
    n = int(np.prod(size))
    rho, u = fields(n, np.float32, 3)
    out = []
    for how in ("ini", "set"):
        with ob.Lattice(19, size, (True, True, True), storage="f32", variant="exact") as lat:
            lat.set_dynamics([ob.BGKdynamics(omega=1.3)])
            if how == "ini":
                lat.ini_equilibrium(rho, u)
            else:
                lat.set_populations(O.equilibrium(19, rho, u))
            lat.collide_and_stream(5)
            out.append(lat.get_populations())
    assert np.array_equal(out[0], out[1])


def test_rejects_wrong_sizes():
    with ob.Lattice(19, (4, 4, 4), (True, True, True)) as lat:
        with pytest.raises(ValueError):
            lat.ini_equilibrium(np.ones(63, np.float32), np.zeros((3, 64), np.float32))
