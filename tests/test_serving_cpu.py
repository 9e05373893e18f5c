"""Host-side pieces of the serving layer, on CPU."""
import math

import numpy as np
import pytest

from openlb_b200 import _abi, serving


def fast_div(n: int, d: int) -> int:
    """Replica of the ensemble kernel's multiply-shift division
    (Granlund & Montgomery): s = ceil(log2 d), m = floor(2^32 (2^s - d) / d) + 1,
    q = (mulhi(n, m) + n) >> s."""
    s = 0
    while (1 << s) < d:
        s += 1
    m = ((1 << 32) * ((1 << s) - d)) // d + 1
    assert m < (1 << 32)
    return (((n * m) >> 32) + n) >> s


@pytest.mark.parametrize("d", [1, 2, 3, 7, 24, 25, 96, 97, 576, 9216, 65535, 1 << 20])
def test_multiply_shift_division(d):
    rng = np.random.default_rng(d)
    ns = list(rng.integers(0, 2 ** 31 - 1, 5000)) + [0, 1, d - 1, d, d + 1, 2 ** 31 - 1, 96 ** 3 - 1]
    for n in ns:
        n = int(n)
        assert fast_div(n, d) == n // d, (n, d)


def test_request_generator_is_seeded_and_in_range():
    a = serving.make_requests(500, rate=20.0, seed=3)
    b = serving.make_requests(500, rate=20.0, seed=3)
    assert [(r.n, r.re, r.lid, r.arrival) for r in a] == [(r.n, r.re, r.lid, r.arrival) for r in b]
    ns = np.array([r.n for r in a])
    assert ns.min() >= 24 and ns.max() <= 96
    res = np.array([r.re for r in a])
    assert res.min() >= 10 and res.max() <= 400
    # log-uniform: the median of log(Re) sits near the middle of the range
    assert abs(np.median(np.log(res)) - 0.5 * (math.log(10) + math.log(400))) < 0.3
    lids = np.array([r.lid for r in a])
    assert lids.min() >= 0.05 and lids.max() <= 0.1
    arr = np.array([r.arrival for r in a])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    # Poisson process at rate 20/s: mean gap 0.05 s
    assert abs(np.mean(np.diff(arr)) - 0.05) < 0.01


def test_request_physics():
    r = serving.Request(0, 0.0, n=64, re=100.0, lid=0.08)
    assert abs(r.nu - 0.08 * 64 / 100) < 1e-15
    assert abs(r.omega - 1 / (3 * r.nu + 0.5)) < 1e-15
    assert 0 < r.omega < 2


def test_pool_bytes_per_instance():
    lib = _abi.load()
    for n in (24, 25, 96):
        cells = n ** 3
        stride = (cells + 63) // 64 * 64
        assert lib.olb_b200_ensemble_bytes_per_instance(n, n, n) == stride * (19 + 3) * 4
    # the 150 GB budget holds 1900+ cavities of the largest size at once
    assert 150 * 2 ** 30 // lib.olb_b200_ensemble_bytes_per_instance(96, 96, 96) > 1900


def test_table_requests_carry_the_cavity_geometry():
    from openlb_b200.workloads import cavity
    reqs = serving.make_requests(5, rate=10.0, seed=3, n_range=(12, 20), tables=True)
    for r in reqs:
        assert r.kind == _abi.ENSEMBLE_GEOMETRY
        assert np.array_equal(r.geometry, cavity((r.n, r.n, r.n)))
    plain = serving.make_requests(5, rate=10.0, seed=3, n_range=(12, 20))
    assert [(r.n, r.re, r.lid, r.arrival) for r in plain] == [(r.n, r.re, r.lid, r.arrival) for r in reqs]
    assert all(r.kind == _abi.ENSEMBLE_CAVITY and r.geometry is None for r in plain)
