"""b200tau_solve_dense_noalloc: the dense tau00 solve for callers that cannot allocate device memory
(their GPU memory belongs to another allocator, or cudaMalloc's implicit synchronisation is not
acceptable on their path).  The entry works on device buffers the caller owns and keeps its scratch
in a fixed file-scope device array, so it allocates nothing.

Checked here through the C ABI: two calls in a row on different matrices give the same tau00 as
the allocating entry b200tau_solve_dense and as the oracle (the reference's own calculateTauMatrix
on the same matrix), both at the FP64 tolerance 1e-12, so nothing left in the shared scratch array
by the first call leaks into the second; the device's free memory is the same before and after
each call (nothing was allocated); sizes above the limit are refused.
This file is collected last so that a stop-at-first-failure run has run everything else first."""

import ctypes

import numpy as np
import pytest

from lsms_b200 import tau as T
from lsms_b200 import workloads as W

pytestmark = pytest.mark.gpu
NOALLOC_MAX_N = 512


def _kkr(prob, ref_build):
    m = ref_build(prob, 0)
    t0 = prob.t_block(int(prob.liz_store_idx[0]), 0)
    return m, t0


def _noalloc(lib, m: np.ndarray, t0: np.ndarray, stream) -> tuple[int, np.ndarray, int]:
    """One call on caller-owned device buffers: (status, tau00, change of the device's free bytes
    across the call)."""
    import torch
    n, b = m.shape[0], t0.shape[0]
    dm = torch.from_numpy(np.asfortranarray(m).ravel(order="F").view(np.float64).copy()).cuda()
    dt = torch.from_numpy(np.asfortranarray(t0).ravel(order="F").view(np.float64).copy()).cuda()
    dout = torch.zeros(2 * b * b, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc = lib.b200tau_solve_dense_noalloc(ctypes.c_void_p(dm.data_ptr()), n, n, ctypes.c_void_p(dt.data_ptr()), b,
                                         ctypes.c_void_p(dout.data_ptr()), ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    out = dout.cpu().numpy().view(np.complex128).reshape(b, b, order="F")
    return rc, out, free1 - free0


def test_noalloc_matches_allocating_entry_twice(ref):
    import torch
    lib = T.load_library()
    lib.b200tau_solve_dense_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    stream = torch.cuda.current_stream().cuda_stream
    s = T.TauSolver(3, 1, 1)
    try:
        cases = [W.config_small(seed=7),
                 W.make_problem("bcc", 5.42, 2, 3, [-0.2 + 0.1j], 8, n_species=2, liz_lmax=[3] * 9 + [2] * 6)]
        # a first call loads the library's kernels and its scratch array onto the device (lazy
        # module loading), which the free-memory check below must not count
        m, t0 = _kkr(cases[1], ref.build_kkr)
        assert _noalloc(lib, m, t0, stream)[0] == T.OK
        for prob in cases:  # two calls in a row, different n
            m, t0 = _kkr(prob, ref.build_kkr)
            rc, got, dfree = _noalloc(lib, m, t0, stream)
            assert rc == T.OK
            assert dfree == 0, dfree  # no device memory was allocated by the call
            want = s.solve_tau00_dense(m, t0)
            assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
            b = t0.shape[0]
            oracle = ref.calculate_tau(prob, 0, 0, ref.ZBLOCKLU_CPP).reshape(b, b).T + t0
            assert np.abs(got - oracle).max() <= 1e-12 * np.abs(oracle).max()
    finally:
        s.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    lib = T.load_library()
    lib.b200tau_solve_dense_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    n = NOALLOC_MAX_N + 16
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    assert lib.b200tau_solve_dense_noalloc(p, n, n, p, 16, p, None) == T.ERR_ARG
    assert lib.b200tau_solve_dense_noalloc(p, 64, 64, p, 48, p, None) == T.ERR_ARG
