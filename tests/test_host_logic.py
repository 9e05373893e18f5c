"""Host-side logic on CPU: descriptors, equilibrium, geometry -> dynamics
table, workloads, and properties of the oracle itself."""
import numpy as np
import pytest

import openlb_b200 as ob
from openlb_b200 import _abi, workloads
from openlb_b200.lattice import dynamics_table
from oracle import oracle as O
from tests import cases as C


@pytest.mark.parametrize("desc", [ob.D3Q19, ob.D3Q27])
def test_descriptor_tables_match_oracle(desc):
    c, opp, w = O.descriptor(desc.q)
    assert np.array_equal(desc.c, c)
    assert np.array_equal(desc.opposite, opp)
    assert np.array_equal(desc.w(np.float64), w)
    # lattice symmetries: sum w = 1, sum w c = 0, sum w c c = cs^2 I
    assert abs(w.sum() - 1) < 1e-15
    assert np.allclose((w[:, None] * c).sum(0), 0)
    assert np.allclose(np.einsum("i,ia,ib->ab", w, c, c), np.eye(3) / 3)
    assert np.array_equal(c[opp], -c)


@pytest.mark.parametrize("desc", [ob.D3Q19, ob.D3Q27])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_host_equilibrium_is_bit_identical_to_oracle(desc, dtype):
    rng = np.random.default_rng(1)
    rho = (1 + 0.02 * rng.standard_normal(300)).astype(dtype)
    u = (0.05 * rng.standard_normal((3, 300))).astype(dtype)
    assert np.array_equal(desc.equilibrium(rho, u, dtype).reshape(-1), O.equilibrium(desc.q, rho, u))


def test_dynamics_table_from_materials():
    mats = np.zeros((5, 4, 3), np.int32)
    mats[1:4, 1:3, 1] = 1
    mats[1:4, 3, 1] = 3
    mats[0] = 2
    table, ids = dynamics_table(
        mats, {1: ob.BGKdynamics(), 2: ob.BounceBack(), 3: ob.BounceBackVelocity()},
        {"OMEGA": 1.25}, {}, {3: (0.1, 0.0, 0.0)}, {})
    kinds = [d.kind for d in table]
    assert kinds == [_abi.DYN_NONE, _abi.DYN_BGK, _abi.DYN_BOUNCE_BACK, _abi.DYN_BOUNCE_BACK_VELOCITY]
    assert table[1].omega == 1.25
    assert table[3].wall_u == (0.1, 0.0, 0.0)
    assert np.array_equal(ids.reshape(mats.shape), np.searchsorted([0, 1, 2, 3], mats))


def test_dynamics_table_requires_omega():
    with pytest.raises(ValueError, match="OMEGA"):
        dynamics_table(np.ones(8, np.int32), {1: ob.BGKdynamics()}, {}, {}, {}, {})


def test_dynamics_params_struct():
    p = ob.ForcedTRTdynamics(omega=1.1, magic=3 / 16, force=(1e-6, 0, 0)).params()
    assert p.kind == _abi.DYN_FORCED_TRT and p.omega == 1.1 and p.magic == 3 / 16
    assert tuple(p.force) == (1e-6, 0.0, 0.0) and p.wall_rho == 1.0


def test_cavity_geometry():
    ids = workloads.cavity((6, 5, 4)).reshape(6, 5, 4)
    assert (ids[1:-1, 1:-1, 1:-1] == 0).all()
    assert (ids[1:-1, -1, 1:-1] == 2).all()
    assert (ids[0] == 1).all() and (ids[:, 0] == 1).all() and (ids[:, :, 0] == 1).all()
    assert np.array_equal(ids.reshape(-1), C.cavity_ids(6, 5, 4))


def test_tgv_initial_field():
    u = workloads.tgv_velocity(16, 0.05, noise=0.0)
    assert u.shape == (3, 16 ** 3)
    assert abs(u.mean()) < 1e-9
    # divergence-free analytic field: mean of u_x * sin(x) positive, u_z zero
    assert np.all(u[2] == 0)
    omega, pops = workloads.taylor_green(8, noise=0.0)
    assert abs(omega - 1 / 0.5375) < 1e-12
    rho, uu = O.moments(C.periodic_case(19, (8, 8, 8)), pops.reshape(-1))
    assert np.allclose(rho, 1, atol=1e-6)


def test_oracle_periodic_mass_conservation():
    rng = np.random.default_rng(0)
    case = C.periodic_case(19, (10, 9, 8))
    f = C.random_state(19, case.n, np.float64, rng)
    m0 = f.sum()
    O.step(case, f, 20)
    assert abs(f.sum() - m0) < 1e-11 * case.n


def test_oracle_rest_is_fixed_point():
    case = C.cavity_case(19, (8, 7, 6), lid=(0.0, 0.0, 0.0))
    f = C.rest_state(19, case.n, np.float64)
    O.step(case, f, 5)
    valid = ~np.isnan(f)
    assert np.abs(f[valid]).max() < 1e-15


def test_oracle_tgv_decays_like_the_analytic_mode():
    """Low-amplitude TGV: kinetic energy follows exp(-6 nu k^2 t) up to the
    lattice's O((k dx)^2) dispersion (2.4% at 32^3, 4.9% at 24^3)."""
    n, nu, steps = 32, 0.01, 200
    omega, pops = workloads.taylor_green(n, u0=0.005, nu=nu, noise=0.0, dtype=np.float64)
    case = C.periodic_case(19, (n, n, n), omega=omega)
    _, u0 = O.moments(case, pops.reshape(-1))
    f = pops.reshape(-1).copy()
    O.step(case, f, steps)
    _, u1 = O.moments(case, f)
    ratio = workloads.tgv_energy(u1) / workloads.tgv_energy(u0)
    assert abs(ratio / workloads.tgv_energy_decay(steps, n, nu) - 1) < 0.04
