"""Checkpoints in OpenLB's Serializable format (openlb_b200/checkpoint.py).

Pinned against files OpenLB itself wrote and read (tests/golden/checkpoint_*.npz,
made by tests/golden/make_golden.py with the compiled reference driver):
  * reading OpenLB's file gives exactly the populations OpenLB dumped for the
    same state, and its other fields as OpenLB set them up;
  * this library's file for a state is byte-identical to the one OpenLB
    resumed from when the fixture was made, and the oracle continued from
    the state read back agrees with OpenLB's own continuation bit for bit.
"""
import base64
import struct
from pathlib import Path

import numpy as np
import pytest

from openlb_b200 import checkpoint as CK
from openlb_b200.descriptors import descriptor

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("checkpoint_*.npz"))


def fixture_case(z):
    """The fixture's set-up as an oracle case."""
    from oracle import oracle as O
    table = [O.Dynamics(int(r[0]), omega=r[1], magic=r[2], smagorinsky=r[3], force=tuple(r[4:7]),
                        wall_u=tuple(r[7:10]), wall_rho=r[10], mixin=int(r[11]), direction=int(r[12]),
                        orientation=int(r[13])) for r in z["table"]]
    return O.Case(q=int(z["q"]), size=tuple(int(s) for s in z["size"]),
                  periodic=tuple(int(p) for p in z["periodic"]), table=table, dyn_id=z["dyn_id"],
                  bc_values=z["bc_values"] if "bc_values" in z.files else None)


def test_file_text_is_two_padded_base64_streams():
    payload = bytes(range(7))
    text = CK.encode(payload)
    assert text[:12] == base64.b64encode(struct.pack("<Q", 7))
    assert text[:12].endswith(b"=")
    assert text[12:] == base64.b64encode(payload)
    assert CK.decode(text) == payload
    assert CK.file_name("run") == "run_rank0_size1.dat"


def test_decode_rejects_a_size_mismatch():
    text = base64.b64encode(struct.pack("<Q", 9)) + base64.b64encode(b"abc")
    with pytest.raises(ValueError, match="header says 9"):
        CK.decode(text)


def test_field_order_follows_the_mangled_type_names():
    names = [f.name for f in CK.lattice_fields(19, ("FORCE",), ("RHO", "VELOCITY", "BC_VELOCITY",
                                                                "PRESSURE_VELOCITY_0-", "PRESSURE_VELOCITY_0+"))]
    assert names == ["POPULATION", "FORCE", "VELOCITY", "RHO", "PRESSURE_VELOCITY_0+", "PRESSURE_VELOCITY_0-",
                     "BC_VELOCITY"]
    # FixedPressureMomentum<0,-1>: a negative template argument mangles as "n1"
    assert CK.field_key("PRESSURE_VELOCITY_0-") == \
        "N3olb5ArrayINS_7momenta21FixedPressureMomentumILi0ELin1EE8VELOCITYEEE"
    with pytest.raises(ValueError):
        CK.field_key("PRESSURE_VELOCITY_3+")


def test_cyclic_columns_unroll_by_their_shift():
    n = 10
    logical = np.arange(n, dtype=np.float32)
    spec = [CK.FieldSpec("POPULATION", 1, cyclic=True)]
    for shift in (0, 3, -4, 9, -9):
        raw = np.empty(n, np.float32)
        raw[(np.arange(n) + shift) % n] = logical      # cpu/sisd/column.h:162-190
        payload = struct.pack("<q", shift) + struct.pack("<Q", n) + raw.tobytes()
        got, end = CK.parse_block(payload, spec, np.float32)
        assert end == len(payload)
        np.testing.assert_array_equal(got["POPULATION"][0], logical)


def test_padding_round_trip_and_periodic_images():
    size, o = (4, 3, 2), 2
    core = np.arange(2 * 24, dtype=np.float64).reshape(2, 24)
    padded = CK.pad_cells(core, size, o, (True, False, True))
    assert padded.shape == (2, 8 * 7 * 6)
    np.testing.assert_array_equal(CK.core_view(padded, size, o), core)
    p = padded.reshape(2, 8, 7, 6)
    np.testing.assert_array_equal(p[:, 0, o:o + 3, o:o + 2], p[:, 4, o:o + 3, o:o + 2])   # x wraps
    assert not p[:, o:o + 4, 0, :].any()                                                    # y filled
    assert CK.overlap_of(size, 8 * 7 * 6) == 2


def test_save_load_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    q, size = 19, (5, 4, 3)
    pops = rng.standard_normal((q, 60)).astype(np.float32)
    force = rng.standard_normal((3, 60)).astype(np.float32)
    fields = CK.lattice_fields(q, ("FORCE",))
    path = tmp_path / CK.file_name("ck")
    CK.save(path, {"POPULATION": pops, "FORCE": force}, q, size, (1, 1, 0), np.float32, 3, fields)
    got, overlap = CK.load(path, q, size, np.float32, fields)
    assert overlap == 3
    np.testing.assert_array_equal(got["POPULATION"], pops)
    np.testing.assert_array_equal(got["FORCE"], force)
    with pytest.raises(ValueError, match="after the listed fields"):
        CK.load(path, q, size, np.float32, CK.lattice_fields(q))


@pytest.mark.parametrize("name", CASES)
def test_reads_openlbs_checkpoint(name):
    z = np.load(GOLDEN / f"{name}.npz")
    q, size = int(z["q"]), tuple(int(s) for s in z["size"])
    dtype = z["pops_saved"].dtype
    fields = CK.lattice_fields(q, tuple(str(s) for s in z["descriptor_fields"]),
                               tuple(str(s) for s in z["extra_fields"]))
    payload = CK.decode(z["checkpoint_ref"].tobytes())
    got = CK.parse_block(payload, fields, dtype)
    assert got[1] == len(payload)
    arrays, overlap = CK.load_bytes(z["checkpoint_ref"].tobytes(), q, size, dtype, fields)
    assert overlap == int(z["overlap"])
    np.testing.assert_array_equal(arrays["POPULATION"].reshape(-1), z["pops_saved"])


@pytest.mark.parametrize("name", CASES)
def test_openlb_resumes_from_our_checkpoint(name, oracle_mod):
    O = oracle_mod
    z = np.load(GOLDEN / f"{name}.npz")
    q, size = int(z["q"]), tuple(int(s) for s in z["size"])
    periodic = tuple(int(p) for p in z["periodic"])
    dtype = z["pops_saved"].dtype
    fields = CK.lattice_fields(q, tuple(str(s) for s in z["descriptor_fields"]),
                               tuple(str(s) for s in z["extra_fields"]))
    other = {k[len("field_"):]: z[k] for k in z.files if k.startswith("field_")}
    text = CK.encode_fields({"POPULATION": z["pops_saved"].reshape(q, -1), **other}, q, size, periodic,
                            dtype, int(z["overlap"]), fields)
    assert text == z["checkpoint_ours"].tobytes()
    # the oracle continues from the state read back exactly as OpenLB continued from the file
    arrays, _ = CK.load_bytes(text, q, size, dtype, fields)
    case = fixture_case(z)
    pops = np.ascontiguousarray(arrays["POPULATION"].reshape(-1))
    O.step(case, pops, int(z["resume_steps"]))
    ref = z["pops_resumed"]
    w = descriptor(q).w(np.float64)
    fin = np.isfinite(pops)
    rel = np.abs(pops - ref).reshape(q, -1) / np.abs(ref.reshape(q, -1) + w[:, None])
    tol = float(z["tolerance"])
    assert np.max(rel[fin.reshape(q, -1)]) <= tol


@pytest.mark.parametrize("name", CASES)
def test_setup_fields_match_openlbs(name):
    """The FORCE / VELOCITY / RHO values this library derives from a set-up are
    the ones OpenLB serialized for the same set-up."""
    z = np.load(GOLDEN / f"{name}.npz")
    q = int(z["q"])
    case = fixture_case(z)
    fields, values = CK.setup_fields(q, z["dyn_id"], case.table, tuple(str(s) for s in z["descriptor_fields"]),
                                     case.bc_values)
    assert [f.name for f in fields] == [f.name for f in CK.lattice_fields(
        q, tuple(str(s) for s in z["descriptor_fields"]), tuple(str(s) for s in z["extra_fields"]))]
    dtype = z["pops_saved"].dtype
    for k, v in values.items():
        np.testing.assert_array_equal(v.astype(dtype), z[f"field_{k}"])


def test_truncated_or_foreign_files_are_rejected(tmp_path):
    q, size = 19, (4, 3, 2)
    pops = np.zeros((q, 24), np.float32)
    text = CK.encode_fields({"POPULATION": pops}, q, size, (1, 1, 1), np.float32, 1)
    payload = CK.decode(text)
    with pytest.raises(ValueError, match="ends inside field POPULATION"):
        CK.parse_block(payload[:-4], CK.lattice_fields(q), np.float32)
    with pytest.raises(ValueError, match="does not pad"):
        CK.load_bytes(text, q, (5, 3, 2), np.float32)
    # a payload written with FP64 values read as FP32 leaves bytes over
    with pytest.raises(ValueError):
        CK.load_bytes(CK.encode_fields({"POPULATION": pops}, q, size, (1, 1, 1), np.float64, 1), q, size,
                      np.float32)
    bad = struct.pack("<q", 24) + struct.pack("<Q", 24) + bytes(96)
    with pytest.raises(ValueError, match="shift 24 out of range"):
        CK.parse_block(bad, [CK.FieldSpec("POPULATION", 1, cyclic=True)], np.float32)
