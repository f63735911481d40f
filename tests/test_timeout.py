"""The timeout path of a bounded device wait, exercised without faulting or hanging the GPU.

Every device-side wait of the library is bounded; one that runs out records a bit in the
context's error word, the waiting CTA still drains the copies it issued before it exits, and the
call returns ERR_TIMEOUT (the reference has no such path: it aborts,
src/Accelerator/zblock_lu_cuda_c.cu:30-52).  The KKR build's first wait on its table copy has a
bound the host can set; 0 makes it give up at once, which is the test's 'flag that nothing
sets'.  The context must stay usable: with the bound restored the next solve matches the oracle."""

import numpy as np
import pytest

from lsms_b200 import tau as T
from lsms_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-12


def _tau_err(prob, got, want):
    from oracle import port
    b = prob.kkrsz_ns
    t0 = -port.tau00_l(prob, np.zeros((b, b), np.complex128), 0, 0)
    return float(np.abs((got + t0) - (want + t0)).max() / np.abs(want + t0).max())


@pytest.mark.parametrize("prec", [T.PREC_FP64, T.PREC_MIXED])
def test_build_wait_that_runs_out_is_reported_and_the_context_recovers(ref, prec):
    prob = W.config_small()
    s = T.TauSolver(prob.lmax, prob.n_spin_cant, prob.n_spin_pola)
    try:
        s.load_problem(prob)
        jobs = T.make_jobs([(0, 0, 0, prob.energies[0])])
        s.set_build_wait(0)
        with pytest.raises(T.B200TauError) as ei:
            s.solve_jobs(jobs, prec)
        assert ei.value.code == T.ERR_TIMEOUT
        # the device-resident entry reports it at the next sync
        import torch
        out = torch.empty(2 * 16 * 16, dtype=torch.float64, device="cuda")
        s.solve_jobs_device(jobs, out.data_ptr(), prec)
        with pytest.raises(T.B200TauError) as ei:
            s.sync()
        assert ei.value.code == T.ERR_TIMEOUT
        s.set_build_wait(1 << 24)
        got = s.solve_jobs(jobs, prec)[0]
        want = ref.calculate_tau(prob, 0, 0, ref.ZBLOCKLU_CPP)
        assert _tau_err(prob, got, want) <= (TOL_FP64 if prec == T.PREC_FP64 else 1e-10)
    finally:
        s.close()


def test_build_wait_bound_is_validated():
    s = T.TauSolver(3, 1, 1)
    try:
        with pytest.raises(T.B200TauError) as ei:
            s.set_build_wait(-1)
        assert ei.value.code == T.ERR_ARG
    finally:
        s.close()
