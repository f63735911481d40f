"""C-ABI checks that need no GPU: the library loads, exports every symbol include/b200tau.h
declares, the job struct matches the header layout, and host-side errors are codes, not aborts."""

import ctypes
import os
import re

import pytest

from lsms_b200 import tau

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "b200tau.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(b200tau_\w+)\s*\(", text)))


def test_header_and_exports_agree():
    decl = declared_symbols()
    assert set(decl) == set(tau.EXPORTS)
    lib = tau.load_library()
    for s in decl:
        assert getattr(lib, s) is not None


def test_job_struct_layout():
    # 4 ints + 2 complex doubles, no padding
    assert ctypes.sizeof(tau.Job) == 48
    assert tau.Job.energy.offset == 16 and tau.Job.prel.offset == 32


def test_gaunt_numbers_bad_lmax():
    lib = tau.load_library()
    buf = (ctypes.c_double * 16)()
    assert lib.b200tau_gaunt_numbers(9, buf) == tau.ERR_ARG
    assert lib.b200tau_gaunt_numbers(-1, buf) == tau.ERR_ARG


def test_create_rejects_bad_parameters():
    lib = tau.load_library()
    ctx = ctypes.c_void_p()
    assert lib.b200tau_create(ctypes.byref(ctx), 0, 7, 1, 1) == tau.ERR_ARG
    assert lib.b200tau_create(ctypes.byref(ctx), 0, 3, 3, 1) == tau.ERR_ARG
    assert lib.b200tau_create(ctypes.byref(ctx), 0, 3, 2, 1) == tau.ERR_ARG  # canted needs pola 2
    assert not ctx


def test_null_context_calls_are_errors():
    lib = tau.load_library()
    assert lib.b200tau_solve(None, None, 0, 0, None) == tau.ERR_ARG
    assert lib.b200tau_upload_tmat(None, None, 0, 0, 0) == tau.ERR_ARG
    assert lib.b200tau_last_error(None) == b"null context"


def test_no_gpu_means_error_not_fallback():
    from tests.conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(tau.B200TauError):
        tau.TauSolver()
