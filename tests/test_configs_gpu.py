"""The reference's configurations on the GPU.

* Config 1 at full size — lid-driven cavity 64^3, D3Q19 BGK FP64 (nu = 0.064,
  tau = 0.692, lid u = (0.1, 0, 0)), 10 000 steps — against OpenLB's own CPU
  build run on the host (oracle/_ref).  Tolerance: FP64, both runs reorder a
  few operations (CSE code, FMA), so |u - u_ref| <= 1e-10 and
  |rho - rho_ref| <= 1e-10 after 10 000 steps of a steady laminar flow.
* Configs 2-4 through openlb_b200.configs at reduced size: the runners work
  and their comparison numbers are in the expected range (the full-size runs
  are reports, not tests).
"""
import numpy as np
import pytest

import openlb_b200 as ob
from openlb_b200 import configs
from oracle import oracle as O
from tests import cases as C

pytestmark = pytest.mark.gpu


def test_config1_cavity_64_fp64_10k_steps_against_reference():
    n, steps = 64, 10000
    case = C.cavity_case(19, (n, n, n))
    rhou = np.zeros((4, case.n))
    rhou[0] = 1.0
    f0 = O.equilibrium(19, rhou[0].copy(), rhou[1:].copy())
    ref = O.run_reference(case, steps, np.float64, init=f0)
    lat = ob.Lattice(19, (n, n, n), (False, False, False), storage="f64")
    try:
        lat.set_dynamics(C.to_abi_table(case), case.dyn_id)
        lat.set_populations(f0)
        lat.collide_and_stream(steps)
        rho, u = lat.get_moments()
    finally:
        lat.close()
    assert np.abs(ref["u"]).max() > 0.05
    np.testing.assert_allclose(u, ref["u"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(rho, ref["rho"], rtol=0, atol=1e-10)


def test_config2_runner_small():
    out = configs.c2(steps=200, n=32, chunk=100)
    r = out["runs"]
    assert r["f32"]["u_l2_vs_f64"] < 1e-4
    assert r["f16"]["u_l2_vs_f64"] < 1e-3 and r["bf16"]["u_l2_vs_f64"] < 5e-3
    # the linear-limit decay is the right order at this Reynolds number and size
    assert abs(r["f64"]["energy_ratio_end"] / r["f64"]["energy_ratio_linear_theory"] - 1) < 0.1


def test_config3_runner_small():
    out = configs.c3(max_steps=4000, size=(48, 24, 24), check=500, storages=("f64", "f32", "f16"),
                     r_range=(2.0, 4.0))
    r = out["runs"]
    assert out["solid_fraction"] >= 0.3
    assert r["f64"]["permeability"] > 0
    assert r["f32"]["u_l2_vs_f64"] < 1e-4 and r["f32"]["permeability_rel_err"] < 1e-4
    assert r["f16"]["u_l2_vs_f64"] < 5e-2


def test_config4_runner_small():
    out = configs.c4(steps=300, size=(64, 32, 32), side=4, sample=50, storages=("f64", "f64_other_seed", "bf16"))
    r = out["runs"]
    assert np.isfinite(r["bf16"]["time_avg_u_l2_vs_f64"]) and r["bf16"]["time_avg_u_l2_vs_f64"] < 0.05
    assert 0 < r["f64_other_seed"]["time_avg_u_l2_vs_f64"] < 0.05
    assert 0.01 < r["f64"]["mean_ux_fluid"] < 0.1
