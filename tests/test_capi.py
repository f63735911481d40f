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


def test_autotune_by_size_groups_jobs_per_bucket(monkeypatch):
    """TauSolver.autotune_paired_steps_by_size (host logic only; the timed library call is
    replaced): jobs go to the bucket of their atom's N rounded up to 64, each bucket is tuned on
    at most `sample` of its jobs in their order, the largest bucket first."""
    s = object.__new__(tau.TauSolver)
    s.atom_n = {0: 2160, 1: 2144, 2: 688, 3: 700}
    seen = []

    def fake(jobs, candidates=None, reps=2):
        seen.append([(j.atom, j.iie) for j in jobs])
        return 768, {c: 1.0 for c in candidates}
    monkeypatch.setattr(s, "autotune_paired_steps", fake, raising=False)
    specs = [(a, i, 0, 0.5 + 0.1j) for i in range(5) for a in (0, 1, 2, 3)]
    table = s.autotune_paired_steps_by_size(tau.make_jobs(specs), sample=3)
    assert list(table) == [2176, 704]
    assert seen[0] == [(0, 0), (1, 0), (0, 1)]   # N 2160 and 2144 share the 2176 bucket
    assert seen[1] == [(2, 0), (3, 0), (2, 1)]   # N 688 and 700 share 704
    assert all(v[0] == 768 for v in table.values())
