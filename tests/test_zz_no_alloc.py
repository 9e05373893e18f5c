"""olb_b200_collide_and_stream_noalloc against the handle-based entry point.

The no-allocation entry point serves callers that cannot let a plug-in
allocate device memory (an application owning a fixed device-memory pool, or
a service that must not allocate on its request path).  They keep the
populations in their own device buffer; here torch allocates that buffer on
the test's behalf, standing in for such a caller's pool.

The check: two calls in a row of the no-allocation entry point produce the
same populations and statistics as olb_b200_collide_and_stream on a lattice
handle with the same input, within the tolerances the parity tests use:
populations within 1e-5 (FP32), 1e-12 (FP64) or 1e-3 (FP16 storage) of the
unshifted population, summed density within 1e-7 relative, summed |u|^2 and
max |u|^2 within 1e-5.  The handle runs the same step-kernel variant and
launch shape as the no-allocation call.  The call only serves triply periodic
lattices; other descriptions are rejected before any device work.  This file
is collected last so a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

import openlb_b200 as ob
from openlb_b200 import _abi

pytestmark = pytest.mark.gpu

# populations: relative to the unshifted population, per storage type (the
# 16-bit bound is one half-precision rounding of the stored deviation)
RTOL_POPS = {"f32": 1e-5, "f64": 1e-12, "f16": 1e-3}
RTOL_STATS = {"sum_rho": 1e-7, "average_rho": 1e-7, "sum_usqr": 1e-5, "average_energy": 1e-5,
              "max_usqr": 1e-5, "max_u": 1e-5}
TORCH_DTYPE = {"f32": "float32", "f64": "float64", "f16": "float16"}


def _state(q, n, rng, dtype):
    rho = (1 + 0.01 * rng.standard_normal(n)).astype(dtype)
    u = (0.03 * rng.standard_normal((3, n))).astype(dtype)
    desc = ob.descriptor(q)
    return (desc.equilibrium(rho, u, dtype) + (1e-3 * rng.standard_normal((q, n))).astype(dtype))


def _scales(q):
    """Storage scale s_i of the 16-bit representation (f_i - w_i) * s_i: the
    power of two s with s / sqrt(2) < 1 / w_i <= s * sqrt(2)."""
    w = ob.descriptor(q).w(np.float64)
    s = np.ones(q)
    for i in range(q):
        while s[i] * np.sqrt(2.0) < 1.0 / w[i]:
            s[i] *= 2.0
    return s


@pytest.mark.parametrize("q,storage", [(19, "f32"), (27, "f32"), (19, "f64"), (27, "f16")])
def test_noalloc_matches_lattice_entry_point(q, storage):
    import torch

    # odd nx: a 16-bit handle then keeps one cell per element, the layout the
    # no-allocation call takes
    size = (41, 36, 70)
    n = size[0] * size[1] * size[2]
    stride = (n + 63) // 64 * 64
    rng = np.random.default_rng(2024 + q)
    compute = np.float64 if storage == "f64" else np.float32
    f0 = _state(q, n, rng, compute)
    omega = 1.3
    lib = _abi.load()
    w = ob.descriptor(q).w(np.float64)[:, None]
    scale = _scales(q)[:, None]

    # existing entry point on a lattice handle
    lat = ob.Lattice(q, size, (True, True, True), storage=storage)
    lat.set_dynamics([ob.BGKdynamics(omega=omega)])
    lat.set_step_variant(0)       # the variant the no-allocation call uses
    lat.set_launch_shape(0, 0)    # the library's default launch shape
    lat.set_populations(f0.reshape(-1))

    # caller-owned device buffer in the library's layout (natural order at step 0)
    dtype = getattr(torch, TORCH_DTYPE[storage])
    buf = torch.zeros((q, stride), dtype=dtype, device="cuda:0")
    stored = f0 * scale if storage == "f16" else f0
    buf[:, :n] = torch.from_numpy(np.ascontiguousarray(stored)).to("cuda:0", dtype)
    torch.cuda.synchronize()

    desc = _abi.Desc()
    desc.q = q
    desc.nx, desc.ny, desc.nz = size
    desc.periodic[0] = desc.periodic[1] = desc.periodic[2] = 1
    desc.storage = _abi.STORAGE[storage]
    desc.device = 0
    bulk = ob.BGKdynamics(omega=omega).params()

    desc_q = ob.descriptor(q)

    def logical(buffer, done):
        """The caller's buffer in the logical post-stream layout, shifted f - w."""
        f = buffer[:, :n].double().cpu().numpy().reshape((q,) + size)
        if done % 2 == 1:
            out = np.empty_like(f)
            for i in range(q):
                # f_i(x) sits in column opp(i) at x - c_i
                out[i] = np.roll(f[desc_q.opposite[i]], shift=tuple(int(c) for c in desc_q.c[i]), axis=(0, 1, 2))
            f = out
        f = f.reshape(q, -1)
        return f / scale if storage == "f16" else f

    steps_done = 0
    try:
        for call, steps in enumerate((3, 3)):  # two calls in a row; the second starts at odd parity
            ref_stats = lat.collide_and_stream(steps, stats=True)
            ref_pops = lat.get_populations().reshape(q, -1).astype(np.float64)

            st = _abi.Stats()
            rc = lib.olb_b200_collide_and_stream_noalloc(ctypes.byref(desc), ctypes.c_void_p(buf.data_ptr()),
                                                        steps_done, ctypes.byref(bulk), steps,
                                                        ctypes.byref(st), None)
            _abi.check(lib, rc)
            steps_done += steps
            torch.cuda.synchronize()

            # statistics of the last step
            for key in ("sum_rho", "sum_usqr", "max_usqr", "average_rho", "average_energy", "max_u"):
                np.testing.assert_allclose(getattr(st, key), ref_stats[key], rtol=RTOL_STATS[key], err_msg=key)
            assert st.n_cells == ref_stats["n_cells"] == n
            assert st.n_nonfinite == 0

            # populations after each call
            got = logical(buf, steps_done)
            err = float((np.abs(got - ref_pops) / np.abs(ref_pops + w)).max())
            assert err <= RTOL_POPS[storage], (call, err)
    finally:
        lat.close()


def _reject(lib, desc, stats=True):
    bulk = ob.BGKdynamics(omega=1.0).params()
    st = _abi.Stats()
    dummy = ctypes.c_void_p(16)  # never dereferenced: argument checks come first
    return lib.olb_b200_collide_and_stream_noalloc(ctypes.byref(desc), dummy, 0, ctypes.byref(bulk), 1,
                                                  ctypes.byref(st) if stats else None, None)


def _periodic_desc(nx, ny, nz):
    desc = _abi.Desc()
    desc.q, desc.nx, desc.ny, desc.nz = 19, nx, ny, nz
    desc.periodic[0] = desc.periodic[1] = desc.periodic[2] = 1
    desc.storage = _abi.STORAGE["f32"]
    return desc


def test_noalloc_rejects_non_periodic_and_malformed_descriptions():
    lib = _abi.load()
    for axis in range(3):
        desc = _periodic_desc(16, 16, 16)
        desc.periodic[axis] = 0
        assert _reject(lib, desc) == _abi.ERR_ARG
        assert b"periodic" in lib.olb_b200_last_error()
    desc = _periodic_desc(16, 16, 16)
    desc.reserved[1] = 7
    assert _reject(lib, desc) == _abi.ERR_ARG
    desc = _periodic_desc(70000, 2, 2)
    assert _reject(lib, desc, stats=False) == _abi.ERR_ARG
    assert b"65535" in lib.olb_b200_last_error()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = _abi.load()
    # 512 x 256 x 256 needs 2 * 128 * 512 = 131072 reduction blocks
    assert _reject(lib, _periodic_desc(512, 256, 256)) == _abi.ERR_ARG
    assert b"scratch" in lib.olb_b200_last_error()
    # a thin lattice of few cells can need too many blocks as well: 1 * 32 * 4096
    assert _reject(lib, _periodic_desc(4096, 256, 1)) == _abi.ERR_ARG
    assert b"reduction blocks" in lib.olb_b200_last_error()
