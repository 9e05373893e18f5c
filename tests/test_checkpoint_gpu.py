"""SuperLattice.load / save on the GPU against files OpenLB wrote and read.

For each tests/golden/checkpoint_* fixture the lattice is set up with the
OpenLB-style calls, resumes from OpenLB's own file, and continues; its
populations must match OpenLB's run resumed from the same state (slots fed
only from OpenLB's non-periodic padding excepted: the oracle marks them NaN
and no fluid cell reads them).  Saving the state just loaded must give the
file this library wrote when the fixture was made, the one OpenLB resumed
from bit for bit.
"""
from pathlib import Path

import numpy as np
import pytest

import openlb_b200 as ob
from openlb_b200 import checkpoint as CK
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("checkpoint_*.npz"))
# the fast build against OpenLB: FP32 1e-5; FP64 1e-10 (OpenLB's boundary
# post-processor rewrites cells in place, one after another)
RTOL = {np.dtype(np.float32): 1e-5, np.dtype(np.float64): 1e-10}


def build(z, variant):
    q, size = int(z["q"]), tuple(int(s) for s in z["size"])
    periodic = tuple(bool(p) for p in z["periodic"])
    geo = ob.SuperGeometry(size, periodic)
    geo.materials[...] = z["dyn_id"].reshape(size).astype(np.int32) + 1
    storage = "f64" if z["pops_saved"].dtype == np.float64 else "f32"
    sl = ob.SuperLattice(geo, q, storage=storage, variant=variant)
    omega = None
    for k, r in enumerate(z["table"]):
        m, kind = k + 1, int(r[0])
        if kind == O.BGK:
            sl.defineDynamics(geo, m, ob.BGKdynamics())
        elif kind == O.TRT:
            sl.defineDynamics(geo, m, ob.TRTdynamics(magic=r[2]))
        elif kind == O.FORCED_TRT:
            sl.defineDynamics(geo, m, ob.ForcedTRTdynamics(magic=r[2]))
            sl.defineForce(geo, m, tuple(r[4:7]))
        elif kind == O.BOUNCE_BACK:
            sl.defineDynamics(geo, m, ob.BounceBack())
        elif kind == O.BOUNCE_BACK_VELOCITY:
            sl.defineDynamics(geo, m, ob.BounceBackVelocity())
            sl.defineU(geo, m, tuple(r[7:10]))
        elif kind == O.SMAGORINSKY:
            sl.defineDynamics(geo, m, ob.SmagorinskyBGKdynamics(smagorinsky=r[3]))
        elif kind in (O.INTERP_VELOCITY, O.INTERP_PRESSURE):
            mixin = {O.BGK: ob.BGKdynamics(), O.SMAGORINSKY: ob.SmagorinskyBGKdynamics(smagorinsky=r[3])}[int(r[11])]
            ob.boundary.set(sl, geo, m, ob.boundary.InterpolatedVelocity if kind == O.INTERP_VELOCITY
                            else ob.boundary.InterpolatedPressure, mixin)
            vals = z["bc_values"].reshape((4,) + size)
            if kind == O.INTERP_VELOCITY:
                sl.defineU(geo, m, vals[1:])
            else:
                sl.defineRho(geo, m, vals[0])
                sl.defineU(geo, m, vals[1:])
        else:
            raise AssertionError(f"kind {kind} not in the checkpoint fixtures")
        if kind in (O.BGK, O.TRT, O.FORCED_TRT, O.SMAGORINSKY):
            omega = r[1]
    sl.setParameter("OMEGA", omega)
    return sl, geo


def live_slots(z):
    """Slots that do not depend on OpenLB's non-periodic padding."""
    q = int(z["q"])
    table = [O.Dynamics(int(r[0]), omega=r[1], magic=r[2], smagorinsky=r[3], force=tuple(r[4:7]),
                        wall_u=tuple(r[7:10]), wall_rho=r[10], mixin=int(r[11]), direction=int(r[12]),
                        orientation=int(r[13])) for r in z["table"]]
    case = O.Case(q=q, size=tuple(int(s) for s in z["size"]), periodic=tuple(int(p) for p in z["periodic"]),
                  table=table, dyn_id=z["dyn_id"], bc_values=z["bc_values"] if "bc_values" in z.files else None)
    probe = np.ascontiguousarray(z["pops_saved"]).copy()
    O.step(case, probe, int(z["resume_steps"]))
    return np.isfinite(probe)


@pytest.mark.parametrize("variant", ["fast", "exact"])
@pytest.mark.parametrize("name", CASES)
def test_resume_from_openlbs_checkpoint(name, variant, tmp_path):
    z = np.load(GOLDEN / f"{name}.npz")
    q = int(z["q"])
    (tmp_path / CK.file_name("ref")).write_bytes(z["checkpoint_ref"].tobytes())
    sl, _ = build(z, variant)
    try:
        sl.initialize()
        assert sl.load(str(tmp_path / "ref"))
        np.testing.assert_array_equal(sl.getPopulations().reshape(-1), z["pops_saved"])
        saved = sl.save(str(tmp_path / "ours"))
        assert Path(saved).read_bytes() == z["checkpoint_ours"].tobytes()
        sl.collideAndStream(int(z["resume_steps"]))
        got = sl.getPopulations().reshape(-1)
    finally:
        sl.close()
    ref = z["pops_resumed"]
    live = live_slots(z)
    w = ob.D3Q19.w(np.float64) if q == 19 else ob.D3Q27.w(np.float64)
    rel = (np.abs(got - ref) / np.abs(ref + np.repeat(w, ref.size // q)))[live]
    assert rel.max() <= RTOL[ref.dtype], rel.max()


def test_load_rejects_a_different_setup(tmp_path):
    z = np.load(GOLDEN / "checkpoint_cavity_q19_float64.npz")
    (tmp_path / CK.file_name("ref")).write_bytes(z["checkpoint_ref"].tobytes())
    sl, geo = build(z, "fast")
    try:
        lid = int(np.flatnonzero(z["table"][:, 0] == O.BOUNCE_BACK_VELOCITY)[0]) + 1
        sl.defineU(geo, lid, (0.05, 0.0, 0.0))
        sl.initialize()
        with pytest.raises(ValueError, match="VELOCITY"):
            sl.load(str(tmp_path / "ref"))
        assert not sl.load(str(tmp_path / "missing"))
    finally:
        sl.close()
