"""The C-ABI library loads and exports every symbol include/npme_gpu.h
declares; parameter validation works without a GPU."""
import ctypes
import os
import re
import subprocess

import pytest

import npme_b200
from npme_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "npme_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void)\s+(npme_gpu_\w+)\s*\(", src, re.M)))


def test_header_declares_what_binding_uses():
    assert declared_functions() == sorted(api.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = api.load_library()
    out = subprocess.run(["nm", "-D", "--defined-only", api.lib_path()],
                         capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT\s+(npme_gpu_\w+)", out))
    for f in declared_functions():
        assert f in exported, f
        assert getattr(lib, f) is not None


def test_default_params_are_reference_defaults():
    lib = api.load_library()
    p = api.Params()
    lib.npme_gpu_default_params(ctypes.byref(p))
    assert p.BnOrder == 8 and p.nDeriv == 8 and p.tol == 1e-6
    assert p.a1 == p.a2 == p.a3 == 4.0 and p.nNeigh == 2 and p.useCompactF == 1


@pytest.mark.parametrize("field,value", [
    ("Rdir", 0.0), ("BnOrder", 7), ("BnOrder", 18), ("N1", 66), ("nDeriv", 1),
    ("nDeriv", 16), ("funcType", 5), ("precision", 9), ("nNeigh", 0)])
def test_invalid_params_rejected_before_touching_the_device(field, value):
    p = api.make_params("laplace", "dm", 8.0, 6, grid=(64, 64, 64))
    setattr(p, field, value)
    with pytest.raises(api.NPMEError) as e:
        npme_b200.Solver(p)
    assert e.value.code == api.EINVAL


def test_orig_split_requires_laplace():
    p = api.make_params("ralpha", "orig", 8.0, 6, grid=(64, 64, 64), alpha=-0.5)
    with pytest.raises(api.NPMEError) as e:
        npme_b200.Solver(p)
    assert e.value.code == api.EINVAL


def test_order_must_fit_grid():
    # BnOrder < N/4 on every axis (src/RecSumSupportFunctions.cpp:61-79)
    p = api.make_params("laplace", "dm", 8.0, 8, grid=(64, 64, 32))
    with pytest.raises(api.NPMEError) as e:
        npme_b200.Solver(p)
    assert e.value.code == api.EINVAL


def test_null_handle_errors_are_recorded():
    # every entry point reports a null handle through npme_gpu_last_error(NULL)
    lib = api.load_library()
    buf = ctypes.create_string_buffer(256)
    bad = api.make_params("laplace", "dm", 8.0, 6, grid=(64, 64, 64))
    bad.Rdir = 0.0
    for f in ("npme_gpu_direct_sum_device", "npme_gpu_direct_sum_device_noalloc",
              "npme_gpu_calcv_device"):
        with pytest.raises(api.NPMEError):  # leaves another message behind
            npme_b200.Solver(bad)
        lib.npme_gpu_last_error(None, buf, 256)
        assert b"null handle" not in buf.value
        rc = getattr(lib, f)(None, None, None, None)
        assert rc == api.EINVAL, f
        lib.npme_gpu_last_error(None, buf, 256)
        assert b"null handle" in buf.value, (f, buf.value)
