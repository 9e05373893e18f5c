"""olb_b200_collide_and_stream_noalloc against the handle-based entry point.

The no-allocation entry point serves callers that cannot let a plug-in
allocate device memory (an application owning a fixed device-memory pool, or
a service that must not allocate on its request path).  They keep the
populations in their own device buffer; here torch allocates that buffer on
the test's behalf, standing in for such a caller's pool.

The check: two calls in a row of the no-allocation entry point produce the
same populations and statistics as olb_b200_collide_and_stream on a lattice
handle with the same input, within the tolerances the parity tests use:
populations within 1e-5 of the unshifted population, summed density within
1e-7 relative, summed |u|^2 and max |u|^2 within 1e-5.  The handle runs the
same step-kernel variant and launch shape as the no-allocation call.  This
file is collected last so a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

import openlb_b200 as ob
from openlb_b200 import _abi

pytestmark = pytest.mark.gpu

RTOL_POPS = 1e-5
RTOL_STATS = {"sum_rho": 1e-7, "average_rho": 1e-7, "sum_usqr": 1e-5, "average_energy": 1e-5,
              "max_usqr": 1e-5, "max_u": 1e-5}


def _state(q, n, rng):
    rho = (1 + 0.01 * rng.standard_normal(n)).astype(np.float32)
    u = (0.03 * rng.standard_normal((3, n))).astype(np.float32)
    desc = ob.descriptor(q)
    return (desc.equilibrium(rho, u, np.float32) + (1e-3 * rng.standard_normal((q, n))).astype(np.float32))


def _rel_pop_error(q, got, ref):
    w = ob.descriptor(q).w(np.float64)[:, None]
    g = got.reshape(q, -1).astype(np.float64)
    r = ref.reshape(q, -1).astype(np.float64)
    return float((np.abs(g - r) / np.abs(r + w)).max())


@pytest.mark.parametrize("q", [19, 27])
def test_noalloc_matches_lattice_entry_point(q):
    import torch

    size = (40, 36, 70)
    n = size[0] * size[1] * size[2]
    stride = (n + 63) // 64 * 64
    rng = np.random.default_rng(2024 + q)
    f0 = _state(q, n, rng)
    omega = 1.3
    lib = _abi.load()

    # existing entry point on a lattice handle
    lat = ob.Lattice(q, size, (True, True, True))
    lat.set_dynamics([ob.BGKdynamics(omega=omega)])
    lat.set_step_variant(0)       # the variant the no-allocation call uses
    lat.set_launch_shape(0, 0)    # the library's default launch shape
    lat.set_populations(f0.reshape(-1))

    # caller-owned device buffer in the library's layout (natural order at step 0)
    buf = torch.zeros((q, stride), dtype=torch.float32, device="cuda:0")
    buf[:, :n] = torch.from_numpy(f0).to("cuda:0")
    torch.cuda.synchronize()

    desc = _abi.Desc()
    desc.q = q
    desc.nx, desc.ny, desc.nz = size
    desc.periodic[0] = desc.periodic[1] = desc.periodic[2] = 1
    desc.storage = _abi.STORAGE["f32"]
    desc.device = 0
    bulk = ob.BGKdynamics(omega=omega).params()

    desc_q = ob.descriptor(q)

    def logical(buffer, done):
        """The caller's buffer in the logical post-stream layout."""
        f = buffer[:, :n].cpu().numpy().reshape((q,) + size)
        if done % 2 == 0:
            return f.reshape(q, -1)
        out = np.empty_like(f)
        for i in range(q):
            # f_i(x) sits in column opp(i) at x - c_i
            out[i] = np.roll(f[desc_q.opposite[i]], shift=tuple(int(c) for c in desc_q.c[i]), axis=(0, 1, 2))
        return out.reshape(q, -1)

    steps_done = 0
    try:
        for call, steps in enumerate((3, 3)):  # two calls in a row; the second starts at odd parity
            ref_stats = lat.collide_and_stream(steps, stats=True)
            ref_pops = lat.get_populations()

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
            assert _rel_pop_error(q, got, ref_pops) <= RTOL_POPS, call
    finally:
        lat.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = _abi.load()
    desc = _abi.Desc()
    desc.q, desc.nx, desc.ny, desc.nz = 19, 512, 256, 256
    desc.storage = _abi.STORAGE["f32"]
    bulk = ob.BGKdynamics(omega=1.0).params()
    st = _abi.Stats()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.olb_b200_collide_and_stream_noalloc(ctypes.byref(desc), dummy, 0, ctypes.byref(bulk), 1,
                                                ctypes.byref(st), None)
    assert rc == _abi.ERR_ARG
    assert b"scratch" in lib.olb_b200_last_error()
