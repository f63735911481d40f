"""Adjoint of tau00 and of ln det M with respect to the site t-matrices (b200tau_solve_vjp).

The C-ABI gradients, contracted with dt/d(delta_l) of a phase-shift site, are compared with the
derivative oracle (oracle/adjoint.py): a bicomplex complex step (h = 1e-20) through the
reference's own G and M, and central differences of the reference's own tau00 re-solved at
perturbed phase shifts.  Tolerances: 1e-8 relative to the largest derivative checked for the
complex step (both FP64, condition numbers up to ~1e4), 1e-5 for the finite differences.
"""

import numpy as np
import pytest

from lsms_b200 import tau as T
from lsms_b200 import workloads as W
from oracle import adjoint as A

TOL_CS = 1e-8
TOL_FD = 1e-5


def _problem_small(seed=11):
    return W.make_problem("bcc", 5.42, 2, 3, [0.5 + 0.1j, -0.1 + 0.3j], seed, n_species=None)


def _contract(prob, grads, site, l, iie):
    """sum_ab grad_site,ab dt_site,ab / d delta_l (compact block of the site)."""
    d = A.dt_ddelta(prob, site, l, iie)
    kk = d.shape[0]
    return np.sum(grads[site][:kk, :kk] * d)


# --- oracle self-consistency (CPU) ------------------------------------------------------------

def test_complex_step_agrees_with_reference_finite_differences(ref):
    prob = _problem_small()
    rng = np.random.default_rng(3)
    tb = rng.normal(size=(16, 16)) + 1j * rng.normal(size=(16, 16))
    pairs = [(0, 0), (0, 2), (3, 1), (14, 3)]
    cs = A.complex_step(prob, 0, tb, pairs)
    for (site, l), (dl, dd) in zip(pairs, cs):
        fl, fd = A.finite_difference(prob, 0, tb, site, l)
        assert abs(dl - fl) <= TOL_FD * abs(dl), (site, l, dl, fl)
        assert abs(dd - fd) <= TOL_FD * max(abs(dd), 1e-3), (site, l, dd, fd)


def test_bicomplex_solve_is_exact_arithmetic():
    rng = np.random.default_rng(5)
    a = rng.normal(size=(6, 6)) + 1j * rng.normal(size=(6, 6)) + 4 * np.eye(6)
    b = 1e-20 * (rng.normal(size=(6, 6)) + 1j * rng.normal(size=(6, 6)))
    x = A.bc_solve(A.Bicomplex(a, b), A.Bicomplex(np.eye(6)))
    prod = A.Bicomplex(a, b) @ x
    assert np.abs(prod.a - np.eye(6)).max() < 1e-13
    assert np.abs(prod.b).max() < 1e-33


# --- the CUDA adjoint -------------------------------------------------------------------------

@pytest.mark.gpu
def test_vjp_matches_complex_step_every_site(solver_factory):
    prob = _problem_small()
    s = solver_factory(3, 1, 1)
    s.load_problem(prob)
    rng = np.random.default_rng(7)
    for iie in range(2):
        tb = rng.normal(size=(16, 16)) + 1j * rng.normal(size=(16, 16))
        tau, g, d = s.solve_vjp(T.make_jobs([(0, iie, 0, prob.energies[iie])]), tb[None], [prob.num_liz])
        pairs = [(site, l) for site in range(prob.num_liz) for l in range(4)]
        cs = A.complex_step(prob, iie, tb, pairs)
        got_l = np.array([_contract(prob, g[0], site, l, iie) for site, l in pairs])
        got_d = np.array([_contract(prob, d[0], site, l, iie) for site, l in pairs])
        want_l = np.array([c[0] for c in cs])
        want_d = np.array([c[1] for c in cs])
        assert np.abs(got_l - want_l).max() <= TOL_CS * np.abs(want_l).max()
        assert np.abs(got_d - want_d).max() <= TOL_CS * np.abs(want_d).max()


@pytest.mark.gpu
def test_vjp_tau00_is_the_forward_solve(solver_factory):
    prob = _problem_small()
    s = solver_factory(3, 1, 1)
    s.load_problem(prob)
    jobs = T.make_jobs([(0, i, 0, prob.energies[i]) for i in range(2)])
    tau, _, _ = s.solve_vjp(jobs, np.zeros((2, 16, 16), np.complex128), [prob.num_liz] * 2)
    fwd = s.solve_jobs(jobs, T.PREC_FP64)
    for i in range(2):
        t0 = prob.t_block(int(prob.liz_store_idx[0]), i)
        want = fwd[i].reshape(16, 16).T + t0
        assert np.abs(tau[i] - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.gpu
def test_vjp_batched_uneven_equals_single_calls(solver_factory):
    """Atoms with LIZ sizes 15 and 9 in one call: each job's blocks land at its own offset."""
    p1 = _problem_small(11)
    p2 = W.make_problem("bcc", 5.42, 1, 3, [0.5 + 0.1j, -0.1 + 0.3j], 12, n_species=None)
    s = solver_factory(3, 1, 1)
    store = np.concatenate([p1.tmat_store, p2.tmat_store], axis=0)
    s.upload_tmat(store)
    s.set_atom(0, p1.liz_pos, p1.liz_lmax, p1.liz_store_idx, None, None)
    s.set_atom(1, p2.liz_pos, p2.liz_lmax, p2.liz_store_idx + p1.tmat_store.shape[0], None, None)
    rng = np.random.default_rng(9)
    tb = rng.normal(size=(3, 16, 16)) + 1j * rng.normal(size=(3, 16, 16))
    specs = [(1, 0, 0, p2.energies[0]), (0, 1, 0, p1.energies[1]), (1, 1, 0, p2.energies[1])]
    Ls = [p2.num_liz, p1.num_liz, p2.num_liz]
    tau, g, d = s.solve_vjp(T.make_jobs(specs), tb, Ls)
    for k, spec in enumerate(specs):
        t1, g1, d1 = s.solve_vjp(T.make_jobs([spec]), tb[k:k + 1], [Ls[k]])
        assert np.array_equal(tau[k], t1[0])
        assert np.array_equal(g[k], g1[0])
        assert np.array_equal(d[k], d1[0])


@pytest.mark.gpu
def test_vjp_fcc87_against_complex_step_and_reference(solver_factory):
    """The adjoint configuration's shape: fcc LIZ of 87 sites (N = 1392), two contour energies
    in one call; sampled (site, l) pairs against the complex step, two against the reference's
    tau re-solved at perturbed phase shifts."""
    prob = W.make_problem("fcc", 6.82, 6, 3, W.semicircle_contour(-0.3, 0.7, 16)[[3, 12]], 51, n_species=None)
    assert prob.nrmat_ns == 1392
    s = solver_factory(3, 1, 1)
    s.load_problem(prob)
    rng = np.random.default_rng(13)
    tb = rng.normal(size=(2, 16, 16)) + 1j * rng.normal(size=(2, 16, 16))
    jobs = T.make_jobs([(0, i, 0, prob.energies[i]) for i in range(2)])
    _, g, d = s.solve_vjp(jobs, tb, [prob.num_liz] * 2)
    pairs = [(0, 0), (0, 3), (1, 2), (40, 1), (86, 0)]
    for iie in range(2):
        cs = A.complex_step(prob, iie, tb[iie], pairs)
        for (site, l), (wl, wd) in zip(pairs, cs):
            gl = _contract(prob, g[iie], site, l, iie)
            gd = _contract(prob, d[iie], site, l, iie)
            assert abs(gl - wl) <= TOL_CS * abs(wl), (iie, site, l, gl, wl)
            assert abs(gd - wd) <= TOL_CS * max(abs(wd), 1e-6), (iie, site, l, gd, wd)
    for site, l in [(0, 1), (7, 2)]:
        fl, fd = A.finite_difference(prob, 0, tb[0], site, l)
        assert abs(_contract(prob, g[0], site, l, 0) - fl) <= TOL_FD * abs(fl)
        assert abs(_contract(prob, d[0], site, l, 0) - fd) <= TOL_FD * max(abs(fd), 1e-3)


@pytest.mark.gpu
def test_autograd_function_gradient_of_a_real_loss(solver_factory):
    """torch.autograd through the C ABI: d/d(delta) of Re<w, tau00> for phase shifts held as a
    torch leaf equals the complex-step derivative."""
    import torch
    from tests.autograd_tau import Tau00
    prob = _problem_small(21)
    s = solver_factory(3, 1, 1)
    iie = 0
    kappa = complex(W.prel_of(prob.energies[iie]))
    L = prob.num_liz
    t0 = np.stack([A.site_t(prob, j, iie) for j in range(L)])
    deltas = np.stack([[np.angle(1 - 2j * kappa * t0[j][l * l, l * l]) / 2 for l in range(4)] for j in range(L)])
    delta = torch.tensor(deltas, dtype=torch.float64, requires_grad=True)
    lidx = torch.tensor([int(np.floor(np.sqrt(k))) for k in range(16)])
    tl = -(1.0 / kappa) * torch.sin(delta) * torch.exp(1j * delta)  # (L, 4)
    t = torch.diag_embed(tl[:, lidx])                                  # (L, 16, 16)
    rng = np.random.default_rng(17)
    w = torch.from_numpy(rng.normal(size=(16, 16)) + 1j * rng.normal(size=(16, 16)))
    tau = Tau00.apply(t, s, prob, iie)
    loss = (w.conj() * tau).real.sum()
    loss.backward()
    pairs = [(0, 0), (0, 3), (5, 1), (14, 2)]
    cs = A.complex_step(prob, iie, np.conj(w.numpy()), pairs)
    for (site, l), (dl, _) in zip(pairs, cs):
        assert abs(delta.grad[site, l].item() - dl.real) <= TOL_CS * np.abs([c[0] for c in cs]).max()


@pytest.mark.gpu
def test_vjp_reuses_the_forward_factors():
    """With b200tau_set_keep_factors, the vjp after an FP64 forward solve of the same jobs
    reuses that solve's factors: no KKR build of M, no elimination and no refinement launches (the
    launch count drops by at least the elimination's three launches per 64-column step), and the
    gradients are those of a vjp with its own factorisation, bit for bit.  The kept factors serve
    one vjp; the next vjp factorises again."""
    prob = W.make_problem("fcc", 6.82, 6, 3, [0.45 + 0.05j, 0.2 + 0.2j], 23, n_species=None)
    assert prob.nrmat_ns == 1392
    s = T.TauSolver(3, 1, 1)
    try:
        s.load_problem(prob)
        jobs = T.make_jobs([(0, i, 0, prob.energies[i]) for i in range(2)])
        rng = np.random.default_rng(9)
        tb = rng.normal(size=(2, 16, 16)) + 1j * rng.normal(size=(2, 16, 16))
        Ls = [prob.num_liz] * 2
        ref_out = s.solve_vjp(jobs, tb, Ls)
        full_launches = s.last_launch_count
        s.set_keep_factors(True)
        fwd = s.solve_jobs(jobs, T.PREC_FP64)
        kept_out = s.solve_vjp(jobs, tb, Ls)
        kept_launches = s.last_launch_count
        again = s.solve_vjp(jobs, tb, Ls)  # the kept factors were used: this one factorises
        again_launches = s.last_launch_count
        s.set_keep_factors(False)
        steps = (prob.nrmat_ns - 16 + 63) // 64
        assert kept_launches <= full_launches - 3 * steps, (kept_launches, full_launches)
        assert again_launches == full_launches
        for a, b in zip(ref_out, kept_out):
            if isinstance(a, list):
                for x, y in zip(a, b):
                    assert np.array_equal(x, y)
            else:
                assert np.array_equal(a, b)
        for i in range(2):  # the forward tau00_l is the vjp's tau00 minus t0
            t0 = prob.t_block(int(prob.liz_store_idx[0]), i)
            assert np.abs(fwd[i].reshape(16, 16).T + t0 - kept_out[0][i]).max() <= 1e-13 * np.abs(t0).max()
    finally:
        s.close()
