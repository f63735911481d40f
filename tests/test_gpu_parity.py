"""Parity of the CUDA path (through the C ABI) with the reference's own calculateTauMatrix.

Tolerances (FP64 path): KKR matrix elementwise 1e-13 x max|M|; tau00_l max-abs error
<= 1e-12 x max|tau00_l| against the reference (the bar stated for the plain FP64 path)."""

import os

import numpy as np
import pytest

from lsms_b200 import tau as T
from lsms_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL_FP64 = 1e-12


def _cases():
    from tests.golden.make_golden import cases
    return cases()


def _solver(factory, prob):
    s = factory(prob.lmax, prob.n_spin_cant, prob.n_spin_pola)
    s.load_problem(prob)
    return s


def relerr(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


@pytest.mark.parametrize("name", sorted(__import__("tests.golden.make_golden", fromlist=["cases"]).cases()))
def test_build_matches_reference(solver_factory, ref, name):
    make, runs = _cases()[name]
    prob = make()
    s = _solver(solver_factory, prob)
    for iie, ispin in runs:
        m_dev = s.build_kkr(0, iie, ispin, prob.energies[iie], prob.nrmat_ns)
        m_ref = ref.build_kkr(prob, iie, ispin)
        assert np.abs(m_dev - m_ref).max() <= 1e-13 * np.abs(m_ref).max()


@pytest.mark.parametrize("name", sorted(__import__("tests.golden.make_golden", fromlist=["cases"]).cases()))
def test_tau00_matches_golden(solver_factory, name):
    make, runs = _cases()[name]
    prob = make()
    s = _solver(solver_factory, prob)
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    specs = [(0, iie, ispin, prob.energies[iie]) for iie, ispin in runs]
    out = s.solve_jobs(T.make_jobs(specs), T.PREC_FP64)
    for k, (iie, ispin) in enumerate(runs):
        want = g[f"tau_blocklu_{iie}_{ispin}"]
        assert relerr(out[k], want) <= TOL_FP64, (name, iie, ispin, relerr(out[k], want))


def test_n2160_contour_points_match_reference(solver_factory, ref):
    prob = W.config_n2160()
    s = _solver(solver_factory, prob)
    picks = [0, 15, 30]
    out = s.solve_jobs(T.make_jobs([(0, i, 0, prob.energies[i]) for i in picks]), T.PREC_FP64)
    for k, i in enumerate(picks):
        want = ref.calculate_tau(prob, i, 0, ref.ZBLOCKLU_CPP)
        assert relerr(out[k], want) <= TOL_FP64, (i, relerr(out[k], want))


def test_batched_equals_one_at_a_time(solver_factory):
    prob = W.make_problem("fcc", 6.82, 4, 3, W.semicircle_contour(-0.3, 0.7, 6), 21, n_species=2)
    s = _solver(solver_factory, prob)
    specs = [(0, i, 0, prob.energies[i]) for i in range(6)]
    batch = s.solve_jobs(T.make_jobs(specs), T.PREC_FP64)
    for k, spec in enumerate(specs):
        one = s.solve_jobs(T.make_jobs([spec]), T.PREC_FP64)[0]
        assert np.array_equal(one, batch[k])


def test_uneven_liz_sizes_in_one_batch(solver_factory, ref):
    """Atoms with LIZ sizes 43, 55, 79 solved in one call (largest first), each vs the reference."""
    probs = [W.make_problem("fcc", 6.82, sh, 3, [0.4 + 0.05j], 30 + sh, n_species=2) for sh in (3, 4, 5)]
    s = solver_factory(3, 1, 1)
    s.upload_tmat(probs[0].tmat_store)
    for a, p in enumerate(probs):
        p.tmat_store = probs[0].tmat_store  # shared store (2 species)
        s.set_atom(a, p.liz_pos, p.liz_lmax, np.minimum(p.liz_store_idx, 1), p.ubr, p.ubrd)
        p.liz_store_idx = np.minimum(p.liz_store_idx, 1)
    specs = [(a, 0, 0, probs[a].energies[0]) for a in (1, 0, 2)]
    out = s.solve_jobs(T.make_jobs(specs), T.PREC_FP64)
    for k, a in enumerate((1, 0, 2)):
        want = ref.calculate_tau(probs[a], 0, 0, ref.ZBLOCKLU_CPP)
        assert relerr(out[k], want) <= TOL_FP64


def test_dense_known_answers(solver_factory):
    """inversionTest type 2 (t = 1, G = 0 -> tau00 = t0) and type 1 (Hilbert) vs a dense solve."""
    from tests.test_oracle import hilbert_kkr
    s = solver_factory(3, 1, 1)
    b = 16
    t0 = np.eye(b, dtype=np.complex128) * (0.3 - 0.1j)
    m = np.eye(b * 7, dtype=np.complex128)
    assert np.array_equal(s.solve_tau00_dense(m, t0), t0)
    m, t0 = hilbert_kkr(b, 6)
    rhs = np.zeros((m.shape[0], b), np.complex128)
    rhs[:b] = t0
    want = np.linalg.solve(m, rhs)[:b]
    assert relerr(s.solve_tau00_dense(m, t0), want) <= 1e-9


def test_dense_matches_zgesv_on_kkr_matrix(solver_factory, ref):
    prob = W.config_small()
    m = ref.build_kkr(prob, 0)
    t0 = prob.t_block(0, 0)
    rhs = np.zeros((m.shape[0], 16), np.complex128)
    rhs[:16] = t0
    want = np.linalg.solve(m, rhs)[:16]
    s = solver_factory(3, 1, 1)
    assert relerr(s.solve_tau00_dense(m, t0), want) <= TOL_FP64


def test_errors_are_reported(solver_factory):
    s = solver_factory(3, 1, 1)
    with pytest.raises(T.B200TauError) as ei:
        s.solve_jobs(T.make_jobs([(57, 0, 0, 0.5)]))
    assert ei.value.code == T.ERR_ARG
    with pytest.raises(T.B200TauError) as ei:
        s.solve_tau00_dense(np.zeros((64, 64), np.complex128), np.eye(16, dtype=np.complex128))
    assert ei.value.code == T.ERR_SINGULAR
    fresh = T.TauSolver(3, 1, 1)
    with pytest.raises(T.B200TauError) as ei:
        fresh.solve_jobs(T.make_jobs([(0, 0, 0, 0.5)]))
    assert ei.value.code == T.ERR_STATE
    fresh.close()
