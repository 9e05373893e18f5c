"""SuperLatticePhysPressure3D / PhysVelocity3D from the device-side moments
against the same conversions of the oracle's density and velocity
(functors/lattice/latticePhysPressure3D.hh, latticePhysVelocity3D.hh:74-85)."""
import numpy as np
import pytest

import openlb_b200 as ob
from oracle import oracle as O
from tests import cases as C

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage,dtype,tol", [("f32", np.float32, 1e-5), ("f64", np.float64, 1e-12)])
def test_phys_pressure_and_velocity(storage, dtype, tol):
    size = (10, 9, 8)
    case = C.cavity_case(19, size)
    geo = ob.SuperGeometry(size)
    geo.materials[...] = case.dyn_id.reshape(size).astype(np.int32) + 1
    sl = ob.SuperLattice(geo, 19, storage=storage)
    try:
        sl.defineDynamics(geo, 1, ob.BGKdynamics())
        sl.defineDynamics(geo, 2, ob.BounceBack())
        sl.defineDynamics(geo, 3, ob.BounceBackVelocity())
        sl.defineU(geo, 3, case.table[2].wall_u)
        sl.setParameter("OMEGA", case.table[0].omega)
        sl.initialize()
        sl.collideAndStream(30)
        conv_p, char_p, conv_u = 2.5e3, 1.0e5, 0.75
        p = sl.getPhysPressure(conv_p, char_p).reshape(-1)
        u = sl.getPhysVelocity(conv_u).reshape(3, -1)
    finally:
        sl.close()
    f = C.rest_state(19, case.n, dtype)
    O.step(case, f, 30)
    rho, vel = O.moments(case, np.nan_to_num(f))
    fluid = case.dyn_id == 0
    want_p = dtype(conv_p) * ((rho.astype(np.float64) - 1.0) / 3.0).astype(dtype) + dtype(char_p)
    np.testing.assert_allclose(p[fluid], want_p[fluid], rtol=tol, atol=0)
    np.testing.assert_allclose(u[:, fluid], dtype(conv_u) * vel[:, fluid], rtol=0, atol=tol)
