"""Full tau = M^-1 T for the Kubo current matrix: b200tau_solve_tau_full against the reference's
own solveTauFullzgetrf (src/MultipleScattering/linearSolvers_CPU.cpp:125-144, called by
src/Kubo/CurrentMatrix.cpp:184-190) on the same inputs, through the C ABI.

Tolerance: max|tau - tau_ref| / max|tau_ref| <= 1e-12 over the whole N x N matrix (FP64), with
the elimination's default pivoting and with panel pivoting forced.  One energy per tmatStore group
and one lmax for every site, as Kubo uses it (the reference reads the group's first energy and
places uniform kkrsz_ns blocks)."""

import numpy as np
import pytest

from lsms_b200 import tau as T
from lsms_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-12


def relerr(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


@pytest.mark.parametrize("pivot", [T.PIVOT_AUTO, T.PIVOT_PANEL])
@pytest.mark.parametrize("case", ["bcc15", "fcc43_polarized", "bcc15_noncollinear"])
def test_tau_full_matches_reference(ref, pivot, case):
    if case == "bcc15":
        prob = W.config_small()
        ispins = [0]
    elif case == "fcc43_polarized":
        prob = W.make_problem("fcc", 6.82, 3, 3, [0.35 + 0.04j], 61, n_species=2, n_spin_pola=2)
        ispins = [0, 1]
    else:
        prob = W.make_problem("bcc", 5.42, 2, 3, [0.5 + 0.02j], 62, n_species=None, n_spin_cant=2,
                              n_spin_pola=2)
        ispins = [0]
    s = T.TauSolver(prob.lmax, prob.n_spin_cant, prob.n_spin_pola)
    try:
        s.set_pivoting(pivot)
        s.load_problem(prob)
        n = prob.nrmat_ns
        for ispin in ispins:
            got = s.solve_tau_full(0, 0, ispin, prob.energies[0], n)
            want = ref.tau_full(prob, 0, ispin)
            assert relerr(got, want) <= TOL_FP64, (case, ispin, relerr(got, want))
    finally:
        s.close()


def test_tau_full_diagonal_block_is_tau00(ref):
    """Its central block is tau00 itself: the same number b200tau_solve returns (+ t0)."""
    prob = W.config_small()
    s = T.TauSolver(3, 1, 1)
    try:
        s.load_problem(prob)
        full = s.solve_tau_full(0, 0, 0, prob.energies[0], prob.nrmat_ns)
        tau00_l = s.calculate_tau_matrix(0, 0, prob.energies[0], 0, T.PREC_FP64).reshape(16, 16).T
        t0 = prob.t_block(int(prob.liz_store_idx[0]), 0)
        assert relerr(full[:16, :16], tau00_l + t0) <= TOL_FP64
    finally:
        s.close()
