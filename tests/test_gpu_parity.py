"""Parity of the CUDA path (through the C ABI) with the reference's own calculateTauMatrix.

Error metric: max|tau - tau_ref| / max|tau_ref| on tau00 before the "- t0" subtraction (in the
frame tau00_l is returned in).  Tolerances: FP64 path 1e-12, mixed-precision path 1e-10 (after
refinement); KKR matrix elementwise 1e-13 x max|M|."""

import os

import numpy as np
import pytest

from lsms_b200 import tau as T
from lsms_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL_FP64 = 1e-12
TOL_MIXED = 1e-10


def _cases():
    from tests.golden.make_golden import cases
    return cases()


def _solver(factory, prob):
    s = factory(prob.lmax, prob.n_spin_cant, prob.n_spin_pola)
    s.load_problem(prob)
    return s


def relerr(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


def t0_local(prob, iie, ispin):
    """t0 in the frame tau00_l is returned in (flat, column-major)."""
    from oracle import port
    b = prob.kkrsz_ns
    return -port.tau00_l(prob, np.zeros((b, b), np.complex128), iie, ispin)


def tau_err(prob, iie, ispin, got, want):
    """Relative max-abs error on tau00 (tau00_l + t0)."""
    t0 = t0_local(prob, iie, ispin)
    return relerr(got + t0, want + t0)


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
        err = tau_err(prob, iie, ispin, out[k], want)
        assert err <= TOL_FP64, (name, iie, ispin, err)


@pytest.mark.parametrize("name", sorted(__import__("tests.golden.make_golden", fromlist=["cases"]).cases()))
def test_tau00_mixed_matches_golden(solver_factory, name):
    make, runs = _cases()[name]
    prob = make()
    s = _solver(solver_factory, prob)
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    specs = [(0, iie, ispin, prob.energies[iie]) for iie, ispin in runs]
    out = s.solve_jobs(T.make_jobs(specs), T.PREC_MIXED)
    assert s.last_fallback_count == 0, name  # the refinement itself converged
    for k, (iie, ispin) in enumerate(runs):
        err = tau_err(prob, iie, ispin, out[k], g[f"tau_blocklu_{iie}_{ispin}"])
        assert err <= TOL_MIXED, (name, iie, ispin, err)


def test_fp64_without_refinement_is_the_block_lu(solver_factory):
    """0 refinement steps: tau00 straight from the Schur block (zblock_lu's contract)."""
    prob = W.config_small()
    s = _solver(solver_factory, prob)
    g = np.load(os.path.join(GOLDEN, "bcc15_E0.6.npz"))
    s.set_refinement(T.PREC_FP64, 0)
    try:
        out = s.calculate_tau_matrix(0, 0, prob.energies[0], 0, T.PREC_FP64)
    finally:
        s.set_refinement(T.PREC_FP64, 1)
    assert tau_err(prob, 0, 0, out, g["tau_blocklu_0_0"]) <= TOL_FP64


def test_n2160_contour_points_match_reference(solver_factory, ref):
    """Every point of the 31-point contour at N = 2160 (the benchmark's workload), FP64 and MIXED
    against the reference's own calculateTauMatrix."""
    prob = W.config_n2160()
    s = _solver(solver_factory, prob)
    picks = list(range(len(prob.energies)))
    out = s.solve_jobs(T.make_jobs([(0, i, 0, prob.energies[i]) for i in picks]), T.PREC_FP64)
    mixed = s.solve_jobs(T.make_jobs([(0, i, 0, prob.energies[i]) for i in picks]), T.PREC_MIXED)
    assert s.last_fallback_count == 0
    for k, i in enumerate(picks):
        want = ref.calculate_tau(prob, i, 0, ref.ZBLOCKLU_CPP)
        assert tau_err(prob, i, 0, out[k], want) <= TOL_FP64, (i, tau_err(prob, i, 0, out[k], want))
        assert tau_err(prob, i, 0, mixed[k], want) <= TOL_MIXED, (i, tau_err(prob, i, 0, mixed[k], want))


@pytest.mark.parametrize("sweep", [T.SWEEP_FP32, T.SWEEP_FP64])
def test_n2160_full_contour_mixed_vs_fp64(solver_factory, sweep):
    """Every point of the 31-point contour at N=2160 (condition numbers 4e2..5e4): the mixed path
    after its adaptive refinement stays within 1e-10 of the FP64 path (which matches the
    reference to 1e-12 at the sampled points above)."""
    prob = W.config_n2160()
    s = _solver(solver_factory, prob)
    s.set_mixed_sweep(sweep)
    try:
        jobs = T.make_jobs([(0, i, 0, prob.energies[i]) for i in range(len(prob.energies))])
        fp64 = s.solve_jobs(jobs, T.PREC_FP64)
        mixed = s.solve_jobs(jobs, T.PREC_MIXED)
        assert s.last_fallback_count == 0
    finally:
        s.set_mixed_sweep(T.SWEEP_FP32)
    errs = [tau_err(prob, i, 0, mixed[i], fp64[i]) for i in range(len(prob.energies))]
    assert max(errs) <= TOL_MIXED, errs


def test_mixed_resolves_unconverged_jobs_in_fp64(solver_factory):
    """A mixed wave whose refinement stops before the convergence test can pass (one round) hands
    every job to the FP64 re-solve, which the host queues without waiting for the outcome; its
    results are the FP64 path's.  The next wave, with the full refinement, converges and re-solves
    nothing."""
    prob = W.config_n2160()
    s = _solver(solver_factory, prob)
    idx = [0, 7, 15, 30]
    jobs = T.make_jobs([(0, i, 0, prob.energies[i]) for i in idx])
    fp64 = s.solve_jobs(jobs, T.PREC_FP64)
    s.set_refinement(T.PREC_MIXED, 1)
    try:
        forced = s.solve_jobs(jobs, T.PREC_MIXED)
        assert s.last_fallback_count == len(idx)
    finally:
        s.set_refinement(T.PREC_MIXED, 10)
    errs = [tau_err(prob, i, 0, forced[k], fp64[k]) for k, i in enumerate(idx)]
    assert max(errs) <= TOL_FP64, errs
    mixed = s.solve_jobs(jobs, T.PREC_MIXED)
    assert s.last_fallback_count == 0
    errs = [tau_err(prob, i, 0, mixed[k], fp64[k]) for k, i in enumerate(idx)]
    assert max(errs) <= TOL_MIXED, errs


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
    probs = [W.make_problem("fcc", 6.82, sh, 3, [0.4 + 0.1j], 30 + sh, n_species=2) for sh in (3, 4, 5)]
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
        assert tau_err(probs[a], 0, 0, out[k], want) <= TOL_FP64


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
    assert relerr(s.solve_tau00_dense(m, t0, T.PREC_MIXED), want) <= TOL_MIXED


def test_errors_are_reported(solver_factory):
    s = solver_factory(3, 1, 1)
    with pytest.raises(T.B200TauError) as ei:
        s.solve_jobs(T.make_jobs([(57, 0, 0, 0.5)]))
    assert ei.value.code == T.ERR_ARG
    with pytest.raises(T.B200TauError) as ei:
        s.solve_tau00_dense(np.zeros((64, 64), np.complex128), np.eye(16, dtype=np.complex128))
    assert ei.value.code == T.ERR_SINGULAR
    with pytest.raises(T.B200TauError) as ei:
        s.set_refinement(T.PREC_MIXED, 99)
    assert ei.value.code == T.ERR_ARG
    fresh = T.TauSolver(3, 1, 1)
    with pytest.raises(T.B200TauError) as ei:
        fresh.solve_jobs(T.make_jobs([(0, 0, 0, 0.5)]))
    assert ei.value.code == T.ERR_STATE
    fresh.close()


@pytest.mark.parametrize("sweep", [T.SWEEP_FP32, T.SWEEP_FP64])
@pytest.mark.parametrize("engine", [T.ENGINE_TENSOR, T.ENGINE_SIMT])
def test_mixed_engines_match_reference(solver_factory, ref, engine, sweep):
    """Both trailing-update engines of the mixed path (tcgen05 TF32 hi/lo and FP32 CUDA cores),
    with the correction solve in FP32 or FP64 arithmetic, reach the mixed tolerance after
    refinement on an N=688 problem near the real axis."""
    prob = W.make_problem("fcc", 6.82, 3, 3, [0.45 + 0.01j, 0.1 + 0.3j], 41, n_species=2)
    s = _solver(solver_factory, prob)
    s.set_mixed_engine(engine)
    s.set_mixed_sweep(sweep)
    try:
        out = s.solve_jobs(T.make_jobs([(0, i, 0, prob.energies[i]) for i in range(2)]), T.PREC_MIXED)
        assert s.last_fallback_count == 0
    finally:
        s.set_mixed_engine(T.ENGINE_TENSOR)
        s.set_mixed_sweep(T.SWEEP_FP32)
    for i in range(2):
        want = ref.calculate_tau(prob, i, 0, ref.ZBLOCKLU_CPP)
        assert tau_err(prob, i, 0, out[i], want) <= TOL_MIXED, (engine, i, tau_err(prob, i, 0, out[i], want))


def test_mixed_without_refinement_is_fp32_accurate(solver_factory, ref):
    """0 refinement steps exposes the factorisation alone: TF32 hi/lo + FP32 accumulation keeps
    tau00 near FP32 accuracy (well below 1e-3), far above the FP64 path's error."""
    prob = W.make_problem("fcc", 6.82, 3, 3, [0.3 + 0.2j], 42, n_species=2)
    s = _solver(solver_factory, prob)
    s.set_refinement(T.PREC_MIXED, 0)
    try:
        out = s.calculate_tau_matrix(0, 0, prob.energies[0], 0, T.PREC_MIXED)
    finally:
        s.set_refinement(T.PREC_MIXED, 10)
    want = ref.calculate_tau(prob, 0, 0, ref.ZBLOCKLU_CPP)
    err = tau_err(prob, 0, 0, out, want)
    assert 1e-12 < err < 1e-3, err


def test_solver_parity_on_the_reference_matrix(solver_factory, ref):
    """Solver-only parity on an ill-conditioned KKR matrix (fcc 79 sites, N=1264, E=0.4+0.05i,
    cond(M) ~ 7e3): the reference's own M fed to b200tau_solve_dense gives the reference's tau00 to
    1e-12.  (Through the full path the device-built M differs from the reference's at the 1e-15
    level, which this condition number amplifies to ~1e-12 in tau00.)"""
    prob = W.make_problem("fcc", 6.82, 5, 3, [0.4 + 0.05j], 35, n_species=2)
    m = ref.build_kkr(prob, 0)
    t0 = prob.t_block(int(prob.liz_store_idx[0]), 0)
    want = ref.calculate_tau(prob, 0, 0, ref.ZBLOCKLU_CPP).reshape(16, 16).T + t0
    s = solver_factory(3, 1, 1)
    assert relerr(s.solve_tau00_dense(m, t0), want) <= TOL_FP64
    assert relerr(s.solve_tau00_dense(m, t0, T.PREC_MIXED), want) <= TOL_MIXED


def test_batched_alloy_with_vacancies_matches_reference(solver_factory, ref):
    """The batched configuration's inputs (random fcc alloy, 5% vacancies, LIZ sizes 43..135):
    a sample of atoms and energies solved in one call, each against the reference."""
    wl = W.config_batched(n_atoms=12)
    s = solver_factory(3, 1, 1)
    s.upload_tmat(wl.tmat_store)
    for a, at in enumerate(wl.atoms):
        s.set_atom(a, at.liz_pos, at.liz_lmax, at.liz_store_idx, at.ubr, at.ubrd)
    picks = [(a, iie) for a, iie in zip(range(12), [0, 5, 9, 14, 20, 31, 3, 7, 11, 17, 25, 30])]
    specs = [(a, iie, 0, wl.energies[iie]) for a, iie in picks]
    fp64 = s.solve_jobs(T.make_jobs(specs), T.PREC_FP64)
    mixed = s.solve_jobs(T.make_jobs(specs), T.PREC_MIXED)
    assert len({wl.atoms[a].num_liz for a, _ in picks}) >= 3
    for k, (a, iie) in enumerate(picks):
        prob = wl.problem(a)
        want = ref.calculate_tau(prob, iie, 0, ref.ZBLOCKLU_CPP)
        assert tau_err(prob, iie, 0, fp64[k], want) <= TOL_FP64, (a, iie)
        assert tau_err(prob, iie, 0, mixed[k], want) <= TOL_MIXED, (a, iie)


def test_noncollinear_n4320_matches_reference(solver_factory, ref):
    """Non-collinear kkrsz_ns = 32 over the 135-site fcc LIZ (N = 4320), spin-dependent phase
    shifts with a random moment per site (condition numbers 1e5..1e7), five (atom, energy) jobs.
    The reference's own two solvers disagree on these matrices by `spread` = |zgesv (0x2001) -
    zblock_lu (0x2005)| (up to ~4e-11); the FP64 path, with its default pivots inside the diagonal
    blocks and with panel pivoting forced, must agree with zgesv within max(1e-12, spread) and with
    zblock_lu within max(1e-12, 2 spread), on the full path (device-built M) and solver-only on the
    reference's own M; the MIXED path (panel pivoting, the default at this size) within 1e-10 of
    FP64 without re-solving any job in FP64."""
    wl = W.config_noncollinear_batch(n_atoms=2)
    s = solver_factory(3, 2, 2)
    s.upload_tmat(wl.tmat_store)
    for a, at in enumerate(wl.atoms):
        s.set_atom(a, at.liz_pos, at.liz_lmax, at.liz_store_idx, at.ubr, at.ubrd)
    picks = [(0, 2), (1, 9), (0, 0), (1, 5), (0, 15)]
    specs = [(a, iie, 0, wl.energies[iie]) for a, iie in picks]
    fp64 = s.solve_jobs(T.make_jobs(specs), T.PREC_FP64)
    mixed = s.solve_jobs(T.make_jobs(specs), T.PREC_MIXED)
    assert s.last_fallback_count == 0
    s.set_pivoting(T.PIVOT_PANEL)
    try:
        fp64_panel = s.solve_jobs(T.make_jobs(specs), T.PREC_FP64)
    finally:
        s.set_pivoting(T.PIVOT_AUTO)
    for k, (a, iie) in enumerate(picks):
        prob = wl.problem(a)
        assert prob.nrmat_ns == 4320
        blocklu = ref.calculate_tau(prob, iie, 0, ref.ZBLOCKLU_CPP)
        zgesv = ref.calculate_tau(prob, iie, 0, ref.ZGESV)
        spread = tau_err(prob, iie, 0, zgesv, blocklu)
        tol_z, tol_b = max(TOL_FP64, spread), max(TOL_FP64, 2 * spread)
        for got in (fp64[k], fp64_panel[k]):
            assert tau_err(prob, iie, 0, got, zgesv) <= tol_z, (a, iie, tau_err(prob, iie, 0, got, zgesv), spread)
            assert tau_err(prob, iie, 0, got, blocklu) <= tol_b, (a, iie, tau_err(prob, iie, 0, got, blocklu), spread)
        assert tau_err(prob, iie, 0, mixed[k], fp64[k]) <= TOL_MIXED, (a, iie, tau_err(prob, iie, 0, mixed[k], fp64[k]))
        if k < 2:  # solver-only on the reference's own matrix
            m = ref.build_kkr(prob, iie)
            t0 = prob.t_block(int(prob.liz_store_idx[0]), iie)
            dense = s.solve_tau00_dense(m, t0)
            assert relerr(dense, port_tau00_raw(prob, iie, zgesv)) <= tol_z
            assert relerr(dense, port_tau00_raw(prob, iie, blocklu)) <= tol_b


def port_tau00_raw(prob, iie, tau00_l):
    """The reference's raw tau00 (global frame, not minus t0) from its returned tau00_l, by
    undoing the trgtol rotation (u is unitary: mg = ud ml u, blockwise) and adding t0."""
    b = prob.kkrsz_ns
    kk = b // 2
    ml = tau00_l.reshape(4, kk, kk).transpose(0, 2, 1)  # block k, [row, col]
    U = prob.ubr.reshape(2, 2, order="F")
    Ud = prob.ubrd.reshape(2, 2, order="F")
    big_l = np.zeros((b, b), np.complex128)
    for k, (p, q) in enumerate([(0, 0), (1, 0), (0, 1), (1, 1)]):
        big_l[p * kk:(p + 1) * kk, q * kk:(q + 1) * kk] = ml[k]
    Ub = np.kron(U, np.eye(kk))
    Udb = np.kron(Ud, np.eye(kk))
    mg = Udb @ big_l @ Ub
    return mg + prob.t_block(int(prob.liz_store_idx[0]), iie)


def test_wave_graphs_match_separate_launches(solver_factory):
    """A wave replayed from its captured CUDA graph gives the results of the same kernels launched
    one by one (FP64 bit for bit; MIXED within 1e-12, its later sweeps may size clusters
    differently), and a second call replays the graph."""
    prob = W.config_n2160(npts=6)
    s = _solver(solver_factory, prob)
    jobs = T.make_jobs([(0, i, 0, prob.energies[i]) for i in range(6)])
    try:
        s.set_graphs(False)
        f_sep = s.solve_jobs(jobs, T.PREC_FP64)
        m_sep = s.solve_jobs(jobs, T.PREC_MIXED)
        s.set_graphs(True)
        for _ in range(2):
            f_g = s.solve_jobs(jobs, T.PREC_FP64)
            m_g = s.solve_jobs(jobs, T.PREC_MIXED)
            assert np.array_equal(f_g, f_sep)
            assert max(tau_err(prob, i, 0, m_g[i], m_sep[i]) for i in range(6)) <= 1e-12
    finally:
        s.set_graphs(True)


@pytest.mark.parametrize("min_rest", [0, 1, 768])
def test_paired_steps_match_reference(solver_factory, ref, min_rest):
    """MIXED at N = 2160 with paired elimination steps everywhere they fit (min_rest = 1), at the
    default threshold (768) and off: every job converges without the FP64 re-solve and matches the
    reference's calculateTauMatrix; paired and single steps leave the same factors, so their
    results agree to the refinement's tolerance."""
    prob = W.config_n2160(npts=8)
    s = _solver(solver_factory, prob)
    jobs = T.make_jobs([(0, i, 0, prob.energies[i]) for i in range(8)])
    try:
        s.set_paired_steps(0)
        single = s.solve_jobs(jobs, T.PREC_MIXED)
        s.set_paired_steps(min_rest)
        for graphs in (False, True):
            s.set_graphs(graphs)
            mixed = s.solve_jobs(jobs, T.PREC_MIXED)
            assert s.last_fallback_count == 0
            for i in range(8):
                want = ref.calculate_tau(prob, i, 0, ref.ZBLOCKLU_CPP)
                assert tau_err(prob, i, 0, mixed[i], want) <= TOL_MIXED, (i, tau_err(prob, i, 0, mixed[i], want))
                assert tau_err(prob, i, 0, mixed[i], single[i]) <= 1e-11
    finally:
        s.set_paired_steps(768)
        s.set_graphs(True)


def test_autotune_paired_steps(solver_factory, ref):
    """The paired-steps autotuner times each candidate threshold on the caller's jobs, keeps the
    fastest, and the solves that follow at that setting still match the reference; bad candidates
    are refused without touching the setting."""
    prob = W.config_n2160(npts=8)
    s = _solver(solver_factory, prob)
    jobs = T.make_jobs([(0, i, 0, prob.energies[i]) for i in range(8)])
    try:
        with pytest.raises(T.B200TauError):
            s.autotune_paired_steps(jobs, candidates=[768, -1])
        chosen, ms = s.autotune_paired_steps(jobs, candidates=[0, 768, 1400], reps=1)
        assert chosen in ms and all(t > 0 for t in ms.values())
        fastest = min(ms, key=ms.get)
        # the setting in force (768) stays unless beaten by 2%
        assert chosen == (fastest if ms[fastest] <= 0.98 * ms[768] else 768)
        mixed = s.solve_jobs(jobs, T.PREC_MIXED)
        assert s.last_fallback_count == 0
        for i in range(8):
            want = ref.calculate_tau(prob, i, 0, ref.ZBLOCKLU_CPP)
            assert tau_err(prob, i, 0, mixed[i], want) <= TOL_MIXED
    finally:
        s.set_paired_steps(768)


def test_autotuned_threshold_applies_to_its_size_bucket(solver_factory):
    """The tuned threshold is recorded for the jobs' size bucket and used by later waves of that
    size (seen in the number of trailing-update passes the profiler times: paired steps update the
    trailing block once for two steps); b200tau_set_paired_steps clears it."""
    prob = W.config_n2160(npts=4)
    s = _solver(solver_factory, prob)
    jobs = T.make_jobs([(0, i, 0, prob.energies[i]) for i in range(4)])
    try:
        def launches(min_rest=None):
            if min_rest is not None:
                s.set_paired_steps(min_rest)
            s.set_profiling(True)
            s.solve_jobs(jobs, T.PREC_MIXED)
            n = s.profile_read()[1]
            s.set_profiling(False)
            return n
        n_off, n_on = launches(0), launches(768)
        assert n_off != n_on
        chosen, _ = s.autotune_paired_steps(jobs, candidates=[0], reps=1)
        assert chosen == 0
        assert launches() == n_off
        assert launches(768) == n_on
    finally:
        s.set_profiling(False)
        s.set_paired_steps(768)
