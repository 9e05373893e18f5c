"""GPU tests of the ensemble (batched) path and the serving loop.

Tolerance: the batched kernel performs the same per-cell arithmetic as the
single-lattice kernel, so an instance's velocity agrees with the same solve on
a lattice handle, and with itself run alone or in a mix, to 1e-6 (absolute, in
lattice units, lid speeds ~0.1) after the stated steps.  Residuals agree to
1e-6 relative (FP64 sums in different orders).
"""
import numpy as np
import pytest

from openlb_b200 import _abi, serving
from openlb_b200.workloads import cavity

pytestmark = pytest.mark.gpu

UTOL = 1e-6


def lattice_velocity(req, steps):
    lat = serving.cavity_lattice(req)
    try:
        lat.collide_and_stream(steps)
        return lat.get_moments()[1]
    finally:
        lat.close()


@pytest.mark.parametrize("n,steps", [(20, 200), (33, 101)])
def test_instance_matches_single_lattice(n, steps):
    req = serving.Request(0, 0.0, n=n, re=100.0, lid=0.1)
    ens = serving.Ensemble(1 << 28, 8)
    try:
        slot = ens.add(req)
        ens.run(steps, check=False)
        u = ens.moments(slot, n)[1]
    finally:
        ens.close()
    ref = lattice_velocity(req, steps)
    assert np.abs(ref).max() > 1e-3
    assert np.max(np.abs(u - ref)) <= UTOL


def test_channel_instance_matches_single_lattice():
    req = serving.Request(0, 0.0, n=18, re=50.0, lid=0.05, kind=_abi.ENSEMBLE_CHANNEL, force=1e-5)
    ens = serving.Ensemble(1 << 28, 8)
    try:
        slot = ens.add(req)
        ens.run(150, check=False)
        u = ens.moments(slot, req.n)[1]
    finally:
        ens.close()
    ref = lattice_velocity(req, 150)
    assert np.abs(u).max() > 1e-5
    assert np.max(np.abs(u - ref)) <= UTOL


def test_same_result_alone_and_in_the_mix():
    """An instance gives the same field whether it runs alone or while others
    of other sizes join and leave."""
    target = serving.Request(0, 0.0, n=26, re=80.0, lid=0.09)
    ens = serving.Ensemble(1 << 29, 16)
    try:
        s = ens.add(target)
        for _ in range(4):
            ens.run(50, check=True)
        alone = ens.moments(s, target.n)[1]
    finally:
        ens.close()
    # in a mix: two others present from the start, one joins after 100 steps,
    # one leaves after 150
    others = [serving.Request(1, 0.0, n=40, re=300.0, lid=0.05), serving.Request(2, 0.0, n=17, re=12.0, lid=0.07)]
    late = serving.Request(3, 0.0, n=31, re=150.0, lid=0.1)
    ens = serving.Ensemble(1 << 29, 16)
    try:
        slots = [ens.add(r) for r in others]
        s = ens.add(target)
        ens.run(50, check=True)
        ens.run(50, check=True)
        ens.add(late)
        ens.run(50, check=True)
        ens.remove(slots[0])
        ens.run(50, check=True)
        mixed = ens.moments(s, target.n)[1]
    finally:
        ens.close()
    assert np.max(np.abs(mixed - alone)) <= UTOL


def test_residual_matches_single_lattice():
    req = serving.Request(0, 0.0, n=22, re=60.0, lid=0.1)
    ens = serving.Ensemble(1 << 28, 4)
    try:
        slot = ens.add(req)
        r1 = ens.run(100, check=True)[0][slot]
        r2 = ens.run(100, check=True)[0][slot]
    finally:
        ens.close()
    lat = serving.cavity_lattice(req)
    try:
        lat.collide_and_stream(100)
        q1 = lat.velocity_residual()
        lat.collide_and_stream(100)
        q2 = lat.velocity_residual()
    finally:
        lat.close()
    assert abs(r1 - 1.0) < 1e-12 and abs(q1 - 1.0) < 1e-12   # first check: against rest
    # same definition (state after the chunk); FP64 sums in different orders
    assert r2 < 1.0 and abs(r2 - q2) <= 1e-6 * q2


def test_admission_by_pool_budget():
    per = _abi.load().olb_b200_ensemble_bytes_per_instance(30, 30, 30)
    ens = serving.Ensemble(3 * per + (1 << 20), 16)
    try:
        slots = [ens.add(serving.Request(k, 0.0, n=30, re=50.0, lid=0.1)) for k in range(4)]
        assert slots[:3] == [0, 1, 2] and slots[3] is None        # fourth does not fit
        assert ens.info()["active"] == 3
        ens.run(10, check=False)
        ens.remove(slots[1])
        again = ens.add(serving.Request(9, 0.0, n=30, re=50.0, lid=0.1))
        assert again == 1                                          # freed memory reused
        ens.run(10, check=False)
    finally:
        ens.close()


def test_slot_limit():
    ens = serving.Ensemble(1 << 28, 2)
    try:
        assert ens.add(serving.Request(0, 0.0, n=12, re=10.0, lid=0.1)) == 0
        assert ens.add(serving.Request(1, 0.0, n=12, re=10.0, lid=0.1)) == 1
        assert ens.add(serving.Request(2, 0.0, n=12, re=10.0, lid=0.1)) is None
    finally:
        ens.close()


@pytest.mark.parametrize("style", ["chunked", "per_step"])
@pytest.mark.parametrize("tables", [False, True])
def test_batched_and_plain_loops_agree(style, tables):
    reqs = serving.make_requests(8, rate=0.0, seed=11, n_range=(16, 30), tol=1e-4, max_steps=600, tables=tables)
    b = serving.serve_batched(reqs, 1 << 30, 16, check_interval=100, keep_velocity=True)
    p = serving.serve_plain(reqs, check_interval=100, keep_velocity=True, style=style)
    assert b["solves"] == p["solves"] == len(reqs)
    rb = {r.rid: r for r in b["results"]}
    rp = {r.rid: r for r in p["results"]}
    for rid in rb:
        assert rb[rid].steps == rp[rid].steps
        assert abs(rb[rid].residual - rp[rid].residual) <= 1e-6 * rp[rid].residual + 1e-15
        assert np.max(np.abs(rb[rid].u - rp[rid].u)) <= UTOL
    assert b["p99_latency_s"] >= b["p50_latency_s"] > 0


# ---------------------------------------------------------------------------
# instances with their own geometry tables (OLB_B200_ENSEMBLE_GEOMETRY)

def obstacle_geometry(n, seed, channel=False):
    """Cell classes of a cavity (or, channel=True, an x-periodic channel with
    walls at the y and z faces) with random box obstacles inside."""
    rng = np.random.default_rng(seed)
    if channel:
        g = np.zeros((n, n, n), np.uint8)
        g[:, 0, :] = g[:, -1, :] = g[:, :, 0] = g[:, :, -1] = 1
    else:
        g = cavity((n, n, n)).reshape(n, n, n).copy()
    for _ in range(3):
        lo = rng.integers(3, n - 6, 3)
        ext = rng.integers(2, 4, 3)
        g[lo[0]:lo[0] + ext[0], lo[1]:lo[1] + ext[1], lo[2]:lo[2] + ext[2]] = 1
    return g.reshape(-1)


def table_request(rid, n, seed, channel=False, **kw):
    kw.setdefault("re", 60.0)
    # the channel has no moving wall; its lid speed only sets the viscosity (nu = lid n / Re)
    kw.setdefault("lid", 0.05 if channel else 0.08)
    req = serving.Request(rid, 0.0, n=n, kind=_abi.ENSEMBLE_GEOMETRY, **kw)
    req.geometry = obstacle_geometry(n, seed, channel)
    return req


def test_cavity_table_equals_procedural_cavity():
    """The cavity given as a table runs the same arithmetic as the built-in one."""
    proc = serving.Request(0, 0.0, n=21, re=90.0, lid=0.1)
    tab = serving.Request(1, 0.0, n=21, re=90.0, lid=0.1, kind=_abi.ENSEMBLE_GEOMETRY)
    tab.geometry = cavity((21, 21, 21))
    ens = serving.Ensemble(1 << 28, 4)
    try:
        a = ens.add(proc)
        b = ens.add(tab)
        ens.run(123, check=True)
        ua = ens.moments(a, 21)[1]
        ub = ens.moments(b, 21)[1]
    finally:
        ens.close()
    assert np.abs(ua).max() > 1e-3
    assert np.array_equal(ua, ub)


@pytest.mark.parametrize("channel", [False, True])
def test_geometry_instance_matches_single_lattice(channel):
    kw = {"force": 2e-5} if channel else {}
    req = table_request(0, 19, seed=3, channel=channel, **kw)
    ens = serving.Ensemble(1 << 28, 4)
    try:
        slot = ens.add(req)
        ens.run(160, check=False)
        u = ens.moments(slot, req.n)[1]
    finally:
        ens.close()
    ref = lattice_velocity(req, 160)
    assert np.abs(ref).max() > 1e-5
    assert np.max(np.abs(u - ref)) <= UTOL


def test_geometry_instances_alone_and_mixed_with_procedural_ones():
    target = table_request(0, 24, seed=5)
    ens = serving.Ensemble(1 << 29, 8)
    try:
        s = ens.add(target)
        ens.run(120, check=True)
        alone = ens.moments(s, target.n)[1]
    finally:
        ens.close()
    ens = serving.Ensemble(1 << 29, 8)
    try:
        ens.add(serving.Request(1, 0.0, n=30, re=200.0, lid=0.06))
        ens.add(table_request(2, 17, seed=8, channel=True, force=1e-5))
        s = ens.add(target)
        ens.run(60, check=True)
        ens.add(serving.Request(3, 0.0, n=13, re=20.0, lid=0.1))
        ens.run(60, check=True)
        mixed = ens.moments(s, target.n)[1]
    finally:
        ens.close()
    assert np.max(np.abs(mixed - alone)) <= UTOL


def test_geometry_table_is_checked():
    ens = serving.Ensemble(1 << 26, 4)
    try:
        bad = table_request(0, 12, seed=1)
        bad.geometry = bad.geometry.copy()
        bad.geometry[7] = 3
        with pytest.raises(_abi.OlbError, match="class 3"):
            ens.add(bad)
        missing = serving.Request(1, 0.0, n=12, re=10.0, lid=0.1, kind=_abi.ENSEMBLE_GEOMETRY)
        with pytest.raises((ValueError, TypeError, _abi.OlbError)):
            ens.add(missing)
        assert ens.info()["active"] == 0
    finally:
        ens.close()
