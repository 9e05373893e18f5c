"""GPU parity of OpenLB's local velocity and pressure boundaries and of the
external and internal edges and corners of velocity boundaries.

* boundary::LocalVelocity on flat faces: CombinedRLBdynamics with the
  regularised velocity-boundary momenta (src/boundary/localVelocity3D.h:47-80,
  src/dynamics/dynamics.h:394-437).
* boundary::LocalPressure on flat faces: CombinedRLBdynamics with the
  regularised pressure-boundary momenta (src/boundary/localPressure3D.h:47-57,
  src/dynamics/momenta/aliases.h:136-141, elements.h:578-616).
* External edges and corners (of local and of interpolated velocity
  boundaries): the mixin with FixedVelocityBoundaryTuple momenta plus
  OuterVelocityEdgeProcessor3D / OuterVelocityCornerProcessor3D in the
  PostStream stage (src/boundary/boundaryPostProcessors3D.hh:164-292).
* Internal edges and corners (a block standing in the cavity):
  CombinedRLBdynamics with InnerEdgeVelocityTuple3D / InnerCornerVelocityTuple3D
  (src/dynamics/momenta/aliases.h:203-217, elements.h:400-438,1711-1757).

Cases: cavity3dBenchmark's default set-up (the whole box surface LocalVelocity,
the lid moving), a channel whose whole inlet face, rim included, is an
interpolated velocity inlet, the cavity with a block standing on its floor
(local and interpolated), and a channel with a LocalVelocity inlet and a
LocalPressure outlet around a square cylinder.  Discrete normals come from
OpenLB's own classification (the channels' faces are flat by construction).

Tolerances, relative to the unshifted population f_i: FP32 1e-5 against the
reference's own dumps and the oracle, FP64 1e-10 (fixtures) / 1e-12 (oracle);
the exact build is bit-identical to the oracle; 16-bit storage: velocity L2
against the FP64 oracle <= 1e-3 (f16) and 5e-3 (bf16).
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from tests import cases as C
from tests.test_boundary_gpu import run_gpu, run_oracle
from tests.test_oracle_golden import load

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
FIXTURES = sorted(p.stem for p in GOLDEN.glob("local_cavity_*.npz")) + \
    sorted(p.stem for p in GOLDEN.glob("open_inlet_*.npz")) + \
    sorted(p.stem for p in GOLDEN.glob("concave_*.npz")) + \
    sorted(p.stem for p in GOLDEN.glob("local_channel_*.npz"))


@pytest.mark.parametrize("name", FIXTURES)
def test_matches_reference_fixture(name):
    z, case = load(name)
    storage = "f64" if z["init"].dtype == np.float64 else "f32"
    steps = int(z["steps"])
    got, rho, u = run_gpu(case, z["init"], steps, storage=storage)
    tol = 1e-10 if storage == "f64" else 1e-5
    ref = np.where(np.isnan(run_oracle(case, z["init"], steps)), np.nan, z["pops"])
    rel, _ = C.pop_tolerance_violation(case.q, got, ref, tol)
    assert rel <= tol, (name, rel)
    keep = np.array([case.table[i].kind != O.BOUNCE_BACK for i in case.dyn_id])
    np.testing.assert_allclose(u[:, keep], z["u"][:, keep], rtol=0, atol=10 * tol)
    np.testing.assert_allclose(rho[keep], z["rho"][keep], rtol=10 * tol, atol=0)


def _cases(q):
    return {"cavity": C.local_velocity_cavity_case(q, (20, 17, 15)),
            "inlet": C.open_inlet_channel_case(q, (22, 12, 11), seed=3),
            "concave": C.concave_cavity_case(q, (16, 13, 14)),
            "concave_interp": C.concave_cavity_case(q, (15, 12, 13), setter=O.INTERP_VELOCITY),
            "local_channel": C.local_channel_case(q, (22, 12, 11), side=2, seed=4)}


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("storage", ["f32", "f64"])
def test_matches_oracle(q, storage):
    dtype = np.float64 if storage == "f64" else np.float32
    for which, case in _cases(q).items():
        f0 = C.rest_state(q, case.n, dtype)
        for steps in (0, 1, 2, 41):
            ref = run_oracle(case, f0, steps)
            got, _, _ = run_gpu(case, f0, steps, storage=storage)
            tol = 1e-12 if storage == "f64" else 1e-5
            rel, _ = C.pop_tolerance_violation(q, got, ref, tol)
            assert rel <= tol, (which, steps, rel)


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("storage", ["f32", "f64"])
def test_exact_build_is_bit_identical(q, storage):
    dtype = np.float64 if storage == "f64" else np.float32
    for which, case in _cases(q).items():
        f0 = C.rest_state(q, case.n, dtype)
        for steps in (0, 3, 30):
            ref = run_oracle(case, f0, steps)
            got, _, _ = run_gpu(case, f0, steps, storage=storage, variant="exact")
            valid = ~np.isnan(ref)
            assert np.array_equal(got[valid], ref[valid]), (which, steps)


@pytest.mark.parametrize("which", ["cavity", "local_channel"])
def test_trt_mixin_matches_oracle(which):
    case = C.local_velocity_cavity_case(19, (16, 14, 12), mixin=O.TRT) if which == "cavity" else \
        C.local_channel_case(19, (20, 11, 10), mixin=O.TRT, side=2, seed=9)
    f0 = C.rest_state(19, case.n, np.float32)
    ref = run_oracle(case, f0, 25)
    got, _, _ = run_gpu(case, f0, 25)
    rel, _ = C.pop_tolerance_violation(19, got, ref, 1e-5)
    assert rel <= 1e-5


@pytest.mark.parametrize("storage,bound", [("f16", 1e-3), ("bf16", 5e-3)])
@pytest.mark.parametrize("nx", [24, 23])
def test_16bit_storage_velocity_error(storage, bound, nx):
    case = C.local_velocity_cavity_case(19, (nx, 16, 14))
    f0 = C.rest_state(19, case.n, np.float64)
    ref = run_oracle(case, f0, 300)
    _, r_u = O.moments(case, np.nan_to_num(ref))
    _, _, u = run_gpu(case, f0.astype(np.float32), 300, storage=storage)
    fluid = case.dyn_id == 0
    err = np.linalg.norm(u[:, fluid] - r_u[:, fluid]) / np.linalg.norm(r_u[:, fluid])
    assert err <= bound, err
