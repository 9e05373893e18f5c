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
def test_batched_and_plain_loops_agree(style):
    reqs = serving.make_requests(8, rate=0.0, seed=11, n_range=(16, 30), tol=1e-4, max_steps=600)
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
