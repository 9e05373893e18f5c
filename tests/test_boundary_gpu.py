"""GPU parity of the interpolated velocity / pressure boundaries
(PlaneFdBoundaryProcessor3D, src/boundary/boundaryPostProcessors3D.hh:39-92).

Each run starts like the reference's lattice initialize(): the PostStream
post-processors once on the initial state (the first collide_and_stream does
it), then collide / stream / PostStream per step.

Tolerances, relative to the unshifted population f_i:
  * FP32 against the reference's own CPU_SISD dumps (golden fixtures) and
    against the C oracle: 1e-5.
  * FP64: 1e-10 against the fixtures (the reference's D3Q19 boundary
    collisions are CSE-generated) and 1e-12 against the oracle.
  * The exact (-fmad=false) build is bit-identical to the oracle.
  * 16-bit storage: relative velocity L2 against the FP64 oracle <= 1e-3 (f16)
    and 5e-3 (bf16).
"""
from pathlib import Path

import numpy as np
import pytest

import openlb_b200 as ob
from oracle import oracle as O
from tests import cases as C
from tests.test_oracle_golden import load

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
INTERP_FIXTURES = sorted(p.stem for p in GOLDEN.glob("interp_*.npz"))


def run_gpu(case, pops0, steps, storage="f32", variant="fast", initialize_only=False):
    lat = ob.Lattice(case.q, case.size, case.periodic, storage=storage, variant=variant)
    try:
        lat.set_dynamics(C.to_abi_table(case), case.dyn_id)
        cells, values = C.boundary_cells_and_values(case)
        lat.set_boundary_values(cells, values)
        lat.set_populations(pops0)
        if initialize_only or steps == 0:
            lat.initialize()
        else:
            lat.collide_and_stream(steps)
        pops = lat.get_populations()
        rho, u = lat.get_moments()
        return pops, rho, u
    finally:
        lat.close()


def run_oracle(case, pops0, steps):
    f = pops0.copy()
    O.post_process(case, f)
    if steps:
        O.step(case, f, steps)
    return f


@pytest.mark.parametrize("name", INTERP_FIXTURES)
def test_matches_reference_fixture(name):
    z, case = load(name)
    storage = "f64" if z["init"].dtype == np.float64 else "f32"
    got, rho, u = run_gpu(case, z["init"], int(z["steps"]), storage=storage)
    tol = 1e-10 if storage == "f64" else 1e-5
    # slots that depend on the reference's padding (NaN in the oracle) only
    # ever reach wall cells and are not compared
    ref = np.where(np.isnan(run_oracle(case, z["init"], int(z["steps"]))), np.nan, z["pops"])
    rel, _ = C.pop_tolerance_violation(case.q, got, ref, tol)
    assert rel <= tol, (name, rel)
    ids = case.dyn_id
    fluid_or_bc = np.array([case.table[i].kind not in (O.BOUNCE_BACK,) for i in ids])
    np.testing.assert_allclose(u[:, fluid_or_bc], z["u"][:, fluid_or_bc], rtol=0, atol=10 * tol)
    np.testing.assert_allclose(rho[fluid_or_bc], z["rho"][fluid_or_bc], rtol=10 * tol, atol=0)


@pytest.mark.parametrize("q,mixin", [(19, O.BGK), (19, O.TRT), (27, O.SMAGORINSKY), (19, O.SMAGORINSKY)])
@pytest.mark.parametrize("storage", ["f32", "f64"])
def test_matches_oracle_with_cylinder(q, mixin, storage):
    dtype = np.float64 if storage == "f64" else np.float32
    case = C.interpolated_channel_case(q, (26, 14, 11), mixin=mixin, side=4, seed=q)
    f0 = C.rest_state(q, case.n, dtype)
    for steps in (0, 1, 2, 57):
        ref = run_oracle(case, f0, steps)
        got, _, _ = run_gpu(case, f0, steps, storage=storage)
        tol = 1e-12 if storage == "f64" else 1e-5
        rel, _ = C.pop_tolerance_violation(q, got, ref, tol)
        assert rel <= tol, (steps, rel)


@pytest.mark.parametrize("q,mixin", [(19, O.BGK), (27, O.SMAGORINSKY), (19, O.TRT)])
@pytest.mark.parametrize("storage", ["f32", "f64"])
def test_exact_build_is_bit_identical(q, mixin, storage):
    dtype = np.float64 if storage == "f64" else np.float32
    case = C.interpolated_channel_case(q, (20, 12, 10), mixin=mixin, side=2, seed=5)
    f0 = C.rest_state(q, case.n, dtype)
    for steps in (0, 3, 30):
        ref = run_oracle(case, f0, steps)
        got, _, _ = run_gpu(case, f0, steps, storage=storage, variant="exact")
        valid = ~np.isnan(ref)
        assert np.array_equal(got[valid], ref[valid]), steps


def test_initialize_applies_post_processors_once():
    case = C.interpolated_channel_case(19, (14, 9, 8), seed=2)
    f0 = C.rest_state(19, case.n, np.float32)
    ref = run_oracle(case, f0, 0)
    assert not np.allclose(ref, f0)
    got, _, _ = run_gpu(case, f0, 0, initialize_only=True)
    rel, _ = C.pop_tolerance_violation(19, got, ref, 1e-6)
    assert rel <= 1e-6
    # explicit initialize, then steps: the same as steps alone
    lat = ob.Lattice(19, case.size, case.periodic)
    try:
        lat.set_dynamics(C.to_abi_table(case), case.dyn_id)
        cells, values = C.boundary_cells_and_values(case)
        lat.set_boundary_values(cells, values)
        lat.set_populations(f0)
        lat.initialize()
        lat.initialize()          # a second call does nothing
        lat.collide_and_stream(5)
        a = lat.get_populations()
    finally:
        lat.close()
    b, _, _ = run_gpu(case, f0, 5)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("storage,bound", [("f16", 1e-3), ("bf16", 5e-3)])
@pytest.mark.parametrize("nx", [24, 23])
def test_16bit_storage_velocity_error(storage, bound, nx):
    case = C.interpolated_channel_case(19, (nx, 12, 10), side=3, seed=9)
    f0 = C.rest_state(19, case.n, np.float64)
    ref = run_oracle(case, f0, 200)
    _, r_u = O.moments(case, np.nan_to_num(ref))
    _, _, u = run_gpu(case, f0.astype(np.float32), 200, storage=storage)
    fluid = case.dyn_id == 0
    err = np.linalg.norm(u[:, fluid] - r_u[:, fluid]) / np.linalg.norm(r_u[:, fluid])
    assert err <= bound, err


def test_boundary_values_validation():
    case = C.interpolated_channel_case(19, (10, 8, 8))
    lat = ob.Lattice(19, case.size, case.periodic)
    try:
        lat.set_dynamics(C.to_abi_table(case), case.dyn_id)
        fluid_cell = int(np.flatnonzero(case.dyn_id == 0)[0])
        with pytest.raises(ob.OlbError, match="not an interpolated boundary cell"):
            lat.set_boundary_values([fluid_cell], [1.0, 0.0, 0.0, 0.0])
        with pytest.raises(ob.OlbError, match="out of range"):
            lat.set_boundary_values([case.n], [1.0, 0.0, 0.0, 0.0])
    finally:
        lat.close()


def test_mixin_must_match_fluid_collision():
    case = C.interpolated_channel_case(19, (10, 8, 8), mixin=O.BGK)
    table = C.to_abi_table(case)
    table[0] = ob.TRTdynamics(omega=1.2)
    lat = ob.Lattice(19, case.size, case.periodic)
    try:
        with pytest.raises(ob.OlbError, match="mixin"):
            lat.set_dynamics(table, case.dyn_id)
    finally:
        lat.close()


@pytest.mark.parametrize("setters", ["interpolated", "local"])
def test_superlattice_facade_channel(setters):
    """The OpenLB-style calls: materials, defineDynamics, boundary::set with
    discrete normals from the geometry, defineU / defineRho on the boundary
    materials, initialize, collideAndStream — against the oracle; the inlet and
    outlet set with InterpolatedVelocity / InterpolatedPressure or with
    LocalVelocity / LocalPressure."""
    nx, ny, nz = 18, 10, 9
    make = C.interpolated_channel_case if setters == "interpolated" else C.local_channel_case
    case = make(19, (nx, ny, nz), omega=1.4, seed=4)
    inlet, outlet = (ob.boundary.InterpolatedVelocity, ob.boundary.InterpolatedPressure) \
        if setters == "interpolated" else (ob.boundary.LocalVelocity, ob.boundary.LocalPressure)
    geo = ob.SuperGeometry((nx, ny, nz))
    mats = case.dyn_id.reshape(nx, ny, nz).astype(np.int32) + 1   # 1 fluid, 2 wall, 3 inlet, 4 outlet
    geo.materials[...] = mats
    sl = ob.SuperLattice(geo, "D3Q19")
    try:
        sl.defineDynamics(geo, 1, ob.BGKdynamics())
        sl.defineDynamics(geo, 2, ob.BounceBack())
        ob.boundary.set(sl, geo, 3, inlet)
        ob.boundary.set(sl, geo, 4, outlet)
        sl.setParameter("OMEGA", 1.4)
        vals = case.bc_values.reshape(4, nx, ny, nz)
        sl.defineU(geo, 3, vals[1:])
        sl.defineRho(geo, 4, vals[0])
        for m in (1, 2, 3, 4):
            sl.iniEquilibrium(geo, m, 1.0, (0.0, 0.0, 0.0))
        sl.initialize()
        sl.collideAndStream(40)
        got_u = sl.getVelocity().reshape(3, -1)
    finally:
        sl.close()
    ref = run_oracle(case, C.rest_state(19, case.n, np.float32), 40)
    _, r_u = O.moments(case, np.nan_to_num(ref))
    fluid = case.dyn_id == 0
    np.testing.assert_allclose(got_u[:, fluid], r_u[:, fluid], rtol=0, atol=1e-6)


@pytest.mark.parametrize("storage", ["f32", "f64"])
def test_inlet_fluctuations_match_host_emulation(storage):
    """Per-step inlet fluctuations on the device equal defineU with the same
    counter-based values before every step (emulated on the oracle)."""
    from openlb_b200.lattice import inlet_noise
    dtype = np.float64 if storage == "f64" else np.float32
    case = C.interpolated_channel_case(19, (16, 10, 9), seed=6)
    f0 = C.rest_state(19, case.n, dtype)
    amp, seed, steps = 0.02, 12345, 12
    lat = ob.Lattice(19, case.size, case.periodic, storage=storage)
    try:
        lat.set_dynamics(C.to_abi_table(case), case.dyn_id)
        cells, values = C.boundary_cells_and_values(case)
        lat.set_boundary_values(cells, values)
        lat.set_boundary_noise(amp, seed)
        lat.set_populations(f0)
        lat.collide_and_stream(steps)
        got = lat.get_populations()
    finally:
        lat.close()
    inlet = cells[np.array([case.table[i].kind for i in case.dyn_id[cells]]) == O.INTERP_VELOCITY]
    base = case.bc_values.copy()
    f = f0.copy()
    O.post_process(case, f)
    for t in range(steps):
        vals = base.copy()
        vals[1:, inlet] = inlet_noise(base[1:, inlet].T, inlet, t, case.n, amp, seed).T
        step_case = O.Case(q=case.q, size=case.size, periodic=case.periodic, table=case.table,
                           dyn_id=case.dyn_id, bc_values=vals)
        O.step(step_case, f, 1)
    tol = 1e-12 if storage == "f64" else 1e-5
    rel, _ = C.pop_tolerance_violation(19, got, f, tol)
    assert rel <= tol, rel
    # and the fluctuations did something
    plain = run_oracle(case, f0, steps)
    assert np.nanmax(np.abs(plain - f)) > 1e-6
