"""CPU checks of the C ABI library: it loads, exports every symbol the header
declares, and fails with a status (never a crash) where no GPU is present or
arguments are invalid."""
import ctypes
import re
from pathlib import Path

import pytest

import openlb_b200 as ob
from openlb_b200 import _abi

HEADER = Path(__file__).resolve().parents[1] / "include" / "olb_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:olb_b200_status|void|int32_t|uint64_t|const char\*)\s+(olb_b200_\w+)\(",
                                 text, flags=re.M)))


def test_header_declares_the_abi():
    names = declared_functions()
    assert set(names) == set(_abi.EXPORTED), names


@pytest.mark.parametrize("variant", ["fast", "exact"])
def test_library_exports_every_declared_symbol(variant):
    lib = _abi.load(variant)
    for name in declared_functions():
        assert hasattr(lib, name), name
    version = int(re.search(r"#define OLB_B200_ABI_VERSION (\d+)", HEADER.read_text()).group(1))
    assert lib.olb_b200_abi_version() == version
    info = lib.olb_b200_build_info().decode()
    assert "sm_100a" in info
    assert ("fmad=false" in info) == (variant == "exact")


def test_null_arguments_are_rejected_with_status():
    lib = _abi.load()
    h = ctypes.c_void_p()
    assert lib.olb_b200_create(None, ctypes.byref(h)) == _abi.ERR_ARG
    assert b"null" in lib.olb_b200_last_error()
    assert lib.olb_b200_set_dynamics(None, None, None, 1) == _abi.ERR_ARG
    assert lib.olb_b200_collide_and_stream(None, 1, None) == _abi.ERR_ARG
    assert lib.olb_b200_get_populations(None, None) == _abi.ERR_ARG
    assert lib.olb_b200_synchronize(None) == _abi.ERR_ARG
    lib.olb_b200_destroy(None)  # no-op


@pytest.mark.parametrize("field,value", [("q", 15), ("nx", 0), ("storage", 9), ("reserved", 1)])
def test_invalid_descriptor_rejected_before_touching_the_gpu(field, value):
    lib = _abi.load()
    d = _abi.Desc()
    d.q, d.nx, d.ny, d.nz = 19, 4, 4, 4
    if field == "reserved":
        d.reserved[0] = value
    else:
        setattr(d, field, value)
    h = ctypes.c_void_p()
    assert lib.olb_b200_create(ctypes.byref(d), ctypes.byref(h)) == _abi.ERR_ARG
    assert not h.value


def test_create_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ob.OlbError) as e:
        ob.Lattice(19, (4, 4, 4))
    assert e.value.status == _abi.ERR_CUDA


def test_missing_library_raises(monkeypatch, tmp_path):
    monkeypatch.setenv("OLB_B200_LIBRARY", str(tmp_path / "nope.so"))
    monkeypatch.setattr(_abi, "_loaded", {})
    with pytest.raises(_abi.LibraryNotBuilt):
        _abi.load("fast")
