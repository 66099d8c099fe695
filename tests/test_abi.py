"""The C ABI without a GPU: the library builds, loads, exports every entry point its header
declares, and rejects bad arguments before it touches a device."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fname in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fname.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fname)).read()
            names += re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(rm_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from rustymath_b200 import build, _lib
    build.build()
    return _lib.load()


def test_header_declares_entry_points():
    names = declared_functions()
    for needed in ["rm_dgemm", "rm_dlu_factor", "rm_dlu_solve", "rm_dsolve"]:
        assert needed in names


def test_every_declared_symbol_is_exported(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_python_binding_covers_the_header():
    from rustymath_b200 import _lib
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_status_strings(lib):
    assert lib.rm_version() >= 100
    assert lib.rm_status_string(0) == b"ok"
    assert b"regular" in lib.rm_status_string(2)


def test_bad_arguments_are_rejected_without_a_device(lib):
    from rustymath_b200 import _lib
    RM_BAD_ARG = _lib.RM_BAD_ARG
    assert lib.rm_dgemm(0, 0, -1, 1, 1, 1.0, None, 1, None, 1, 0.0, None, 1, None) == RM_BAD_ARG
    assert lib.rm_dgemm(2, 0, 1, 1, 1, 1.0, None, 1, None, 1, 0.0, None, 1, None) == RM_BAD_ARG
    assert lib.rm_dgemm_host(0, 0, 4, 4, 4, 1.0, None, 3, None, 4, 0.0, None, 4) == RM_BAD_ARG
    assert lib.rm_dlu_factor(-2, None, None, None, None, None) == RM_BAD_ARG
    assert lib.rm_dlu_solve(3, None, None, None, 1, None, 0, None) == RM_BAD_ARG
    assert lib.rm_dlu_solve(3, None, None, None, 1, None, 7, None) == RM_BAD_ARG
    assert lib.rm_dsolve(-1, None, None, 1, None, None, None, None) == RM_BAD_ARG
    # empty and degenerate sizes are no-ops, as in the reference (linalg.rs:803-805)
    assert lib.rm_dgemm(0, 0, 0, 5, 5, 1.0, None, 5, None, 5, 0.0, None, 5, None) == 0
    assert lib.rm_dlu_solve(0, None, None, None, 3, None, 0, None) == 0


def test_empty_system_is_not_regular(lib):
    from rustymath_b200 import _lib
    rep = _lib.SolveReport()
    assert lib.rm_dsolve(0, None, None, 1, None, None, ctypes.byref(rep), None) == _lib.RM_NOT_REGULAR


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import rustymath_b200 as rb
    with pytest.raises(rb.RmError):
        rb.solve(np.eye(3), np.ones(3))
    c = ctypes.c_int(-1)
    from rustymath_b200 import _lib
    assert _lib.load().rm_device_count(ctypes.byref(c)) == 0 and c.value == 0


def test_test_hooks_check_their_arguments(lib):
    from rustymath_b200 import _lib
    assert lib.rm_test_inject_failure(0, 0, 1) == _lib.RM_BAD_ARG
    assert lib.rm_test_inject_failure(_lib.RM_INJECT_OUT_OF_MEMORY, -1, 1) == _lib.RM_BAD_ARG
    assert lib.rm_test_inject_failure(_lib.RM_INJECT_CUDA_ERROR, 0, -1) == _lib.RM_BAD_ARG
    assert lib.rm_test_inject_failure(_lib.RM_INJECT_CUDA_ERROR, 0, 0) == _lib.RM_OK
    assert lib.rm_test_chain_timeout(10) == _lib.RM_BAD_ARG
    assert lib.rm_test_chain_timeout(3_000_000_000) == _lib.RM_BAD_ARG


def test_status_query_without_a_device(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from rustymath_b200 import _lib
    assert lib.rm_take_status(None) == _lib.RM_NO_DEVICE
    assert lib.rm_test_chain_timeout(1_000_000) == _lib.RM_NO_DEVICE
