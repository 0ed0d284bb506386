"""CPU checks of the C ABI: the library loads, exports exactly what
include/inti_b200.h declares, and fails cleanly (status + message, no crash)
when no device is usable.  No compute calls run here."""
import ctypes as C
import re
from pathlib import Path

import pytest

import inti_b200
from inti_b200 import _lib as L

ROOT = Path(__file__).resolve().parents[1]


def header_functions():
    text = (ROOT / "include" / "inti_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(inti_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = L.load()
    declared = header_functions()
    assert len(declared) >= 25
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(L.SIGNATURES), set(declared) ^ set(L.SIGNATURES)


def test_version():
    assert L.load().inti_version() == 1


def test_library_is_built_for_sm_100a():
    so = L.LIB_PATH.read_bytes()
    assert b"sm_100a" in so


def test_null_arguments_are_rejected_without_device():
    lib = L.load()
    assert lib.inti_ctx_create(0, None, None) == L.E_ARG
    assert lib.inti_op_apply(None, None, 0, None, 0, 1, None, None, 0) == L.E_ARG
    assert lib.inti_quad_size(None) == -1
    assert lib.inti_ctx_launch_count(None) == -1


def test_context_creation_reports_missing_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present; covered by the GPU tests")
    lib = L.load()
    h = C.c_void_p()
    st = lib.inti_ctx_create(0, None, C.byref(h))
    assert st != L.OK
    assert lib.inti_last_error(None)
    with pytest.raises(inti_b200.InticError):
        inti_b200.Context(0)


def test_julia_binding_calls_only_declared_exports():
    """Every ccall of inti.jl_b200/julia/IntiB200.jl names a function the
    header declares and the library exports (Julia itself is absent here)."""
    text = (ROOT / "inti.jl_b200" / "julia" / "IntiB200.jl").read_text()
    called = sorted(set(re.findall(r"ccall\(\(:(inti_[a-z0-9_]+)", text)))
    assert len(called) >= 10
    lib = L.load()
    declared = set(header_functions())
    for name in called:
        assert name in declared and hasattr(lib, name), name
