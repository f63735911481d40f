"""Panel pivoting (B200TAU_PIVOT_PANEL): every 64-column step picks its rows from the whole
remaining column (a partial-pivoting elimination on the diagonal block's rows and the panel's rows
of largest magnitude), approaching LAPACK's zgetrf over a column (the reference's CPU solver
pivots with zgetrf inside ~N/3-row blocks, zblock_lu_cpp.cpp:58; its zgesv path,
linearSolvers_CPU.cpp:76-96, over the whole column).

Parity: FP64 within 1e-12 of the reference's tau00 where the matrices allow it (N = 240, 2160);
at N = 4320 (non-collinear, condition numbers 1e5..1e7) within the spread of the reference's own
two solvers (zgesv 0x2001 vs zblock_lu 0x2005) on the same matrix, times 2.  MIXED within 1e-10
of FP64, with no job left to the FP64 re-solve."""

import numpy as np
import pytest

from lsms_b200 import tau as T
from lsms_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-12
TOL_MIXED = 1e-10


def relerr(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


def t0_local(prob, iie, ispin=0):
    from oracle import port
    b = prob.kkrsz_ns
    return -port.tau00_l(prob, np.zeros((b, b), np.complex128), iie, ispin)


def tau_err(prob, iie, got, want):
    t0 = t0_local(prob, iie)
    return relerr(got + t0, want + t0)


@pytest.fixture
def panel_solver():
    made = []

    def make(prob_or_params, ns=1, npola=1):
        s = T.TauSolver(3, ns, npola)
        s.set_pivoting(T.PIVOT_PANEL)
        made.append(s)
        return s

    yield make
    for s in made:
        s.close()


def test_panel_fp64_and_mixed_small(panel_solver, ref):
    prob = W.config_small()
    s = panel_solver(prob)
    s.load_problem(prob)
    want = ref.calculate_tau(prob, 0, 0, ref.ZBLOCKLU_CPP)
    jobs = T.make_jobs([(0, 0, 0, prob.energies[0])])
    assert tau_err(prob, 0, s.solve_jobs(jobs, T.PREC_FP64)[0], want) <= TOL_FP64
    assert tau_err(prob, 0, s.solve_jobs(jobs, T.PREC_MIXED)[0], want) <= TOL_MIXED
    assert s.last_fallback_count == 0


def test_panel_fp64_without_refinement_is_the_schur_complement(panel_solver, ref):
    """Pivots never leave the rows of the LIZ sites other than the central one, so the trailing
    block is still 1 - Delta and tau00 from it alone (0 refinement steps) is the reference's."""
    prob = W.make_problem("fcc", 6.82, 4, 3, [0.45 + 0.02j], 51, n_species=2)
    s = panel_solver(prob)
    s.load_problem(prob)
    s.set_refinement(T.PREC_FP64, 0)
    got = s.calculate_tau_matrix(0, 0, prob.energies[0], 0, T.PREC_FP64)
    want = ref.calculate_tau(prob, 0, 0, ref.ZBLOCKLU_CPP)
    assert tau_err(prob, 0, got, want) <= TOL_FP64


def test_panel_n2160_contour_matches_reference(panel_solver, ref):
    """All 31 contour points at N = 2160 with panel pivoting: FP64 and MIXED against the
    reference."""
    prob = W.config_n2160()
    s = panel_solver(prob)
    s.load_problem(prob)
    jobs = T.make_jobs([(0, i, 0, prob.energies[i]) for i in range(31)])
    fp64 = s.solve_jobs(jobs, T.PREC_FP64)
    mixed = s.solve_jobs(jobs, T.PREC_MIXED)
    assert s.last_fallback_count == 0
    for i in range(31):
        want = ref.calculate_tau(prob, i, 0, ref.ZBLOCKLU_CPP)
        assert tau_err(prob, i, fp64[i], want) <= TOL_FP64, (i, tau_err(prob, i, fp64[i], want))
        assert tau_err(prob, i, mixed[i], want) <= TOL_MIXED, (i, tau_err(prob, i, mixed[i], want))


def test_panel_dense_matches_zgesv_on_ill_conditioned_matrix(panel_solver, ref):
    prob = W.make_problem("fcc", 6.82, 5, 3, [0.4 + 0.05j], 35, n_species=2)
    m = ref.build_kkr(prob, 0)
    t0 = prob.t_block(int(prob.liz_store_idx[0]), 0)
    rhs = np.zeros((m.shape[0], 16), np.complex128)
    rhs[:16] = t0
    want = np.linalg.solve(m, rhs)[:16]
    s = panel_solver(prob)
    assert relerr(s.solve_tau00_dense(m, t0), want) <= TOL_FP64
    assert relerr(s.solve_tau00_dense(m, t0, T.PREC_MIXED), want) <= TOL_MIXED
