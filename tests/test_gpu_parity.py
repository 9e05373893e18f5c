"""GPU parity: the sm_100a collide-and-stream through the C ABI against the C
oracle (itself pinned bit for bit to OpenLB's CPU_SISD generic path).

Tolerances (written here, per the path's precision contract):
  * FP32 populations: |gpu - oracle| <= 1e-5 * |f_i| per slot, f_i the
    unshifted population (f_i - w_i) + w_i, after the stated step count.
  * FP64 populations: 1e-12 * |f_i|.
  * The -fmad=false build of the same kernels ("exact") is bit-identical to the
    oracle for every collision (same operations in the same order).
  * 16-bit storage: relative velocity L2 <= 1e-3 against the FP64 oracle.
Slots the oracle marks NaN depend on OpenLB's unspecified overlap padding
(they only ever reach wall cells) and are not compared.
"""
import numpy as np
import pytest

import openlb_b200 as ob
from oracle import oracle as O
from tests import cases as C

pytestmark = pytest.mark.gpu

RTOL = {"f32": 1e-5, "f64": 1e-12}


def run_gpu(case, pops0, steps, storage="f32", variant="fast", stats=False):
    lat = ob.Lattice(case.q, case.size, case.periodic, storage=storage, variant=variant)
    try:
        lat.set_dynamics(C.to_abi_table(case), case.dyn_id)
        lat.set_populations(pops0)
        st = lat.collide_and_stream(steps, stats=stats) if steps else None
        pops = lat.get_populations()
        rho, u = lat.get_moments()
        return pops, rho, u, st
    finally:
        lat.close()


def run_oracle(case, pops0, steps, stats=False):
    f = pops0.copy()
    st = O.step(case, f, steps, with_stats=stats) if steps else None
    return f, st


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("steps", [0, 1, 2, 7])
def test_periodic_bgk_f32(q, steps):
    rng = np.random.default_rng(100 + q + steps)
    case = C.periodic_case(q, (12, 10, 9))
    f0 = C.random_state(q, case.n, np.float32, rng)
    ref, _ = run_oracle(case, f0, steps)
    got, rho, u, _ = run_gpu(case, f0, steps)
    rel, _ = C.pop_tolerance_violation(q, got, ref, RTOL["f32"])
    assert rel <= RTOL["f32"], rel
    r_rho, r_u = O.moments(case, ref)
    np.testing.assert_allclose(rho, r_rho, rtol=1e-6, atol=0)
    np.testing.assert_allclose(u, r_u, rtol=0, atol=1e-6)


KINDS = [O.BGK, O.TRT, O.SMAGORINSKY, O.FORCED_BGK, O.FORCED_TRT]


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("kind", KINDS, ids=[O.KIND_NAMES[k] for k in KINDS])
@pytest.mark.parametrize("storage", ["f32", "f64"])
def test_periodic_all_collisions(q, kind, storage):
    dtype = np.float64 if storage == "f64" else np.float32
    rng = np.random.default_rng(7 * q + kind)
    case = C.periodic_case(q, (9, 8, 11), kind=kind)
    f0 = C.random_state(q, case.n, dtype, rng)
    for steps in (3, 4):
        ref, _ = run_oracle(case, f0, steps)
        got, _, _, _ = run_gpu(case, f0, steps, storage=storage)
        rel, _ = C.pop_tolerance_violation(q, got, ref, RTOL[storage])
        assert rel <= RTOL[storage], (steps, rel)


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("kind", KINDS, ids=[O.KIND_NAMES[k] for k in KINDS])
@pytest.mark.parametrize("storage", ["f32", "f64"])
def test_exact_build_is_bit_identical(q, kind, storage):
    dtype = np.float64 if storage == "f64" else np.float32
    rng = np.random.default_rng(11 * q + kind)
    case = C.periodic_case(q, (8, 7, 6), kind=kind)
    f0 = C.random_state(q, case.n, dtype, rng)
    ref, _ = run_oracle(case, f0, 5)
    got, _, _, _ = run_gpu(case, f0, 5, storage=storage, variant="exact")
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("storage", ["f32", "f64"])
@pytest.mark.parametrize("steps", [1, 10, 31])
def test_cavity_walls_and_lid(q, storage, steps):
    dtype = np.float64 if storage == "f64" else np.float32
    case = C.cavity_case(q, (14, 12, 10))
    f0 = C.rest_state(q, case.n, dtype)
    ref, _ = run_oracle(case, f0, steps)
    got, rho, u, _ = run_gpu(case, f0, steps, storage=storage)
    rel, _ = C.pop_tolerance_violation(q, got, ref, RTOL[storage])
    assert rel <= RTOL[storage], rel
    # exact build: bit-identical on every slot the reference defines
    got_x, _, _, _ = run_gpu(case, f0, steps, storage=storage, variant="exact")
    valid = ~np.isnan(ref)
    assert np.array_equal(got_x[valid], ref[valid])
    # moments with per-dynamics semantics (walls report RHO and VELOCITY)
    r_rho, r_u = O.moments(case, np.where(valid, ref, 0).astype(dtype))
    tol = 1e-5 if storage == "f32" else 1e-12
    np.testing.assert_allclose(rho, r_rho, rtol=tol, atol=0)
    np.testing.assert_allclose(u, r_u, rtol=0, atol=tol)


def test_porous_forced_trt():
    rng = np.random.default_rng(5)
    case = C.porous_case(19, (24, 16, 14), rng)
    f0 = C.rest_state(19, case.n, np.float32)
    ref, _ = run_oracle(case, f0, 40)
    got, _, _, _ = run_gpu(case, f0, 40)
    rel, _ = C.pop_tolerance_violation(19, got, ref, RTOL["f32"])
    assert rel <= RTOL["f32"], rel


def test_channel_smagorinsky_d3q27():
    case = C.channel_cylinder_case(27, (24, 14, 8))
    rng = np.random.default_rng(9)
    n = case.n
    rho = np.ones(n, np.float32)
    u = np.zeros((3, n), np.float32)
    u[0] = 0.05 * (1 + 0.02 * rng.uniform(-1, 1, n))
    f0 = O.equilibrium(27, rho, u)
    ref, _ = run_oracle(case, f0, 20)
    got, _, _, _ = run_gpu(case, f0, 20)
    rel, _ = C.pop_tolerance_violation(27, got, ref, RTOL["f32"])
    assert rel <= RTOL["f32"], rel


@pytest.mark.parametrize("storage", ["f32", "f64"])
def test_statistics_match(storage):
    dtype = np.float64 if storage == "f64" else np.float32
    case = C.cavity_case(19, (16, 14, 12))
    f0 = C.rest_state(19, case.n, dtype)
    ref, ost = run_oracle(case, f0, 12, stats=True)
    _, _, _, st = run_gpu(case, f0, 12, storage=storage, stats=True)
    assert st["n_cells"] == ost["n_cells"]
    assert st["n_nonfinite"] == 0
    # per-cell rho agrees to FP32 rounding of the populations; the FP64 sums
    # then agree to that rounding averaged over the cells
    np.testing.assert_allclose(st["sum_rho"], ost["sum_rho"], rtol=1e-7 if storage == "f32" else 1e-12)
    np.testing.assert_allclose(st["sum_usqr"], ost["sum_usqr"], rtol=1e-5)
    np.testing.assert_allclose(st["max_usqr"], ost["max_usqr"], rtol=1e-5)
    assert abs(st["average_rho"] - st["sum_rho"] / st["n_cells"]) < 1e-15
    # LatticeStatistics conventions: energy = 0.5 <|u|^2>, maxU = sqrt(max |u|^2)
    assert abs(st["average_energy"] - 0.5 * st["sum_usqr"] / st["n_cells"]) < 1e-15
    assert abs(st["max_u"] - np.sqrt(st["max_usqr"])) < 1e-15


def test_diverged_is_reported_not_trapped():
    case = C.periodic_case(19, (8, 8, 8))
    f0 = C.rest_state(19, case.n, np.float32)
    f0[5 * case.n + 17] = np.nan
    lat = ob.Lattice(19, case.size, case.periodic)
    try:
        lat.set_dynamics(C.to_abi_table(case))
        lat.set_populations(f0)
        with pytest.raises(ob.Diverged):
            lat.collide_and_stream(2, stats=True)
        # the context stays usable
        lat.set_populations(C.rest_state(19, case.n, np.float32))
        st = lat.collide_and_stream(2, stats=True)
        assert st["n_nonfinite"] == 0
    finally:
        lat.close()


@pytest.mark.parametrize("storage,bound", [("f16", 1e-3), ("bf16", 5e-3)])
def test_16bit_storage_velocity_error(storage, bound):
    """Shifted 16-bit storage, FP32 math: velocity L2 vs the FP64 oracle.

    FP16 meets 1e-3.  BF16 keeps 8 significand bits, so each stored deviation
    carries a relative rounding error up to 2^-9 ~ 2e-3; its bound is 5e-3."""
    q = 19
    size = (32, 32, 32)
    n = np.prod(size)
    x = (np.arange(size[0]) + 0.5) * 2 * np.pi / size[0]
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    u0 = 0.05
    u = np.stack([u0 * np.sin(X) * np.cos(Y) * np.cos(Z), -u0 * np.cos(X) * np.sin(Y) * np.cos(Z),
                  np.zeros_like(X)]).reshape(3, -1)
    case = C.periodic_case(q, size, omega=1 / (0.5 + 3 * 0.0125))
    f0_64 = O.equilibrium(q, np.ones(n), u)
    ref, _ = run_oracle(case, f0_64, 200)
    _, r_u = O.moments(case, ref)
    got, _, gu, _ = run_gpu(case, f0_64.astype(np.float32), 200, storage=storage)
    err = np.linalg.norm(gu - r_u) / np.linalg.norm(r_u)
    assert err <= bound, err


@pytest.mark.parametrize("kind", [O.TRT, O.FORCED_TRT], ids=["trt", "forced_trt"])
@pytest.mark.parametrize("storage,bound", [("f16", 1e-3), ("bf16", 5e-3)])
def test_16bit_trt_velocity_error(kind, storage, bound):
    """TRT and Guo-forced TRT on the scaled 16-bit representation: velocity L2
    after 200 steps vs the FP64 oracle, with the FP16/BF16 bounds above."""
    q = 19
    size = (24, 24, 24)
    n = np.prod(size)
    x = (np.arange(size[0]) + 0.5) * 2 * np.pi / size[0]
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    u0 = 0.05
    u = np.stack([u0 * np.sin(X) * np.cos(Y) * np.cos(Z), -u0 * np.cos(X) * np.sin(Y) * np.cos(Z),
                  np.zeros_like(X)]).reshape(3, -1)
    case = C.periodic_case(q, size, kind=kind, omega=1 / (0.5 + 3 * 0.0125), force=(1e-5, -2e-6, 3e-6))
    f0_64 = O.equilibrium(q, np.ones(n), u)
    ref, _ = run_oracle(case, f0_64, 200)
    _, r_u = O.moments(case, ref)
    got, _, gu, _ = run_gpu(case, f0_64.astype(np.float32), 200, storage=storage)
    err = np.linalg.norm(gu - r_u) / np.linalg.norm(r_u)
    assert err <= bound, err


def test_set_populations_resets_layout():
    """Upload after an odd number of steps: the AA parity is internal."""
    rng = np.random.default_rng(3)
    case = C.periodic_case(19, (10, 9, 8))
    f0 = C.random_state(19, case.n, np.float32, rng)
    lat = ob.Lattice(19, case.size, case.periodic)
    try:
        lat.set_dynamics(C.to_abi_table(case))
        lat.set_populations(f0)
        lat.collide_and_stream(3)
        mid = lat.get_populations()
        lat.set_populations(mid)
        lat.collide_and_stream(2)
        got = lat.get_populations()
    finally:
        lat.close()
    ref, _ = run_oracle(case, f0, 5)
    rel, _ = C.pop_tolerance_violation(19, got, ref, RTOL["f32"])
    assert rel <= RTOL["f32"]


def test_invalid_launch_shape_rejected():
    lat = ob.Lattice(19, (8, 8, 8))
    try:
        for bad in [(16, 2), (48, 1), (512, 1), (32, 0)]:
            with pytest.raises(ob.OlbError):
                lat.set_launch_shape(*bad)
    finally:
        lat.close()


@pytest.mark.parametrize("shape", [(32, 1), (32, 4), (64, 2), (128, 2), (256, 1)])
def test_launch_shapes_agree(shape):
    rng = np.random.default_rng(4)
    case = C.cavity_case(19, (12, 11, 40))
    f0 = C.random_state(19, case.n, np.float32, rng, amp_u=0.0, amp_neq=1e-4)
    lat = ob.Lattice(19, case.size, case.periodic)
    try:
        lat.set_dynamics(C.to_abi_table(case), case.dyn_id)
        lat.set_launch_shape(*shape)
        lat.set_populations(f0)
        lat.collide_and_stream(6)
        got = lat.get_populations()
    finally:
        lat.close()
    ref, _ = run_oracle(case, f0, 6)
    rel, _ = C.pop_tolerance_violation(19, got, ref, RTOL["f32"])
    assert rel <= RTOL["f32"]


@pytest.mark.parametrize("storage", ["f32", "f64", "f16"])
@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("build", ["exact", "fast"])
def test_step_variants_agree(storage, masked, build):
    """Kernel variants differ only in work distribution.  Without FMA
    contraction (exact build) their results are bit-identical; with it, nvcc
    may contract differently per instantiation, so the fast build's variants
    agree to the FP32 parity tolerance."""
    rng = np.random.default_rng(8)
    size = (10, 21, 40)
    case = C.cavity_case(19, size) if masked else C.periodic_case(19, size)
    dtype = np.float64 if storage == "f64" else np.float32
    f0 = C.random_state(19, case.n, dtype, rng, amp_u=0.01, amp_neq=1e-4)
    results = []
    for variant in range(4):
        lat = ob.Lattice(19, case.size, case.periodic, storage=storage, variant=build)
        try:
            lat.set_dynamics(C.to_abi_table(case), case.dyn_id)
            lat.set_step_variant(variant)
            assert lat.tuning()["variant"] == variant
            lat.set_populations(f0)
            lat.collide_and_stream(5)
            results.append(lat.get_populations())
        finally:
            lat.close()
    for r in results[1:]:
        if build == "exact":
            assert np.array_equal(r, results[0])
        elif storage == "f16":
            # a one-ulp FP32 difference can move a value across a half-precision
            # rounding boundary: bound by one unit roundoff of the stored value
            assert np.all(np.abs(r - results[0]) <= 2.0 ** -11 * np.abs(results[0]) + 1e-7)
        else:
            rel, _ = C.pop_tolerance_violation(19, r, results[0], RTOL["f32"])
            assert rel <= RTOL["f32"], rel


def test_autotune_restores_state_and_picks_a_candidate():
    rng = np.random.default_rng(9)
    case = C.periodic_case(19, (24, 20, 64))
    f0 = C.random_state(19, case.n, np.float32, rng)
    lat = ob.Lattice(19, case.size, case.periodic)
    try:
        lat.set_dynamics(C.to_abi_table(case))
        lat.set_populations(f0)
        lat.collide_and_stream(3)
        before = lat.get_populations()
        steps_before = lat.info()["steps_done"]
        t = lat.autotune(4)
        assert t["tuned"] == 1 and t["candidates"] >= 4 and t["ms_per_step"] > 0
        assert lat.info()["steps_done"] == steps_before
        assert np.array_equal(lat.get_populations(), before)
        lat.collide_and_stream(2)
        got = lat.get_populations()
    finally:
        lat.close()
    ref, _ = run_oracle(case, f0, 5)
    rel, _ = C.pop_tolerance_violation(19, got, ref, RTOL["f32"])
    assert rel <= RTOL["f32"]


def _shear_wave_state(size, dtype, u0=0.04):
    """Velocity varying along all three axes, so populations cross every face."""
    nx, ny, nz = size
    X, Y, Z = np.meshgrid(*(2 * np.pi * (np.arange(s) + 0.5) / s for s in size), indexing="ij")
    u = np.stack([u0 * np.sin(Y) * np.cos(Z), u0 * np.sin(X) * np.cos(Z), u0 * np.cos(X) * np.sin(Y)])
    rho = 1 + 0.01 * np.cos(X + Y + Z)
    n = nx * ny * nz
    return O.equilibrium(19, rho.reshape(-1).astype(dtype), u.reshape(3, n).astype(dtype))


@pytest.mark.parametrize("nx", [2, 4, 6, 5, 24])
@pytest.mark.parametrize("storage,bound", [("f16", 1e-3), ("bf16", 5e-3)])
def test_16bit_paired_layout_across_the_x_seam(nx, storage, bound):
    """16-bit storage pairs cells x and x+nx/2 (even nx); odd nx keeps the
    natural layout.  Flow crossing the x seam must match the FP64 oracle."""
    size = (nx, 12, 34)
    case = C.periodic_case(19, size, omega=1.2)
    f64 = _shear_wave_state(size, np.float64)
    ref, _ = run_oracle(case, f64, 20)
    _, r_u = O.moments(case, ref)
    got, _, gu, _ = run_gpu(case, f64.astype(np.float32), 20, storage=storage)
    err = np.linalg.norm(gu - r_u) / np.linalg.norm(r_u)
    assert err <= bound, err
    # the populations themselves, relative to the unshifted value
    rel, _ = C.pop_tolerance_violation(19, got, ref, 1.0)
    assert rel <= (2e-4 if storage == "f16" else 2e-3), rel


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_16bit_cavity_with_walls(storage):
    case = C.cavity_case(19, (16, 14, 12))
    ref64, _ = run_oracle(case, C.rest_state(19, case.n, np.float64), 60)
    valid = ~np.isnan(ref64)
    _, r_u = O.moments(case, np.where(valid, ref64, 0))
    _, _, gu, _ = run_gpu(case, C.rest_state(19, case.n, np.float32), 60, storage=storage)
    fluid = case.dyn_id == 0
    err = np.linalg.norm(gu[:, fluid] - r_u[:, fluid]) / np.linalg.norm(r_u[:, fluid])
    assert err <= (2e-3 if storage == "f16" else 1e-2), err


@pytest.mark.parametrize("storage", ["f16", "bf16"])
@pytest.mark.parametrize("nx", [8, 7])
def test_16bit_round_trip(storage, nx):
    rng = np.random.default_rng(12)
    q, size = 19, (nx, 6, 5)
    n = nx * 30
    f = C.random_state(q, n, np.float32, rng)
    lat = ob.Lattice(q, size, (True, True, True), storage=storage)
    try:
        lat.set_populations(f)
        back = lat.get_populations()
    finally:
        lat.close()
    # round to nearest in the 16-bit format: at most one unit roundoff of the
    # stored (shifted, power-of-two scaled) value — 2^-11 for FP16, 2^-8 for
    # BF16 — plus half the FP16 subnormal spacing for values near zero
    u = 2.0 ** -11 if storage == "f16" else 2.0 ** -8
    assert np.all(np.abs(back - f) <= u * np.abs(f) + 2.0 ** -25)
