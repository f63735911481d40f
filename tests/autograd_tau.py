"""torch.autograd.Function around the C-ABI solve and its adjoint (test harness only).

Forward: per-site t-matrices (L, b, b) of one energy -> raw tau00 (b, b) through b200tau_solve.
Backward: b200tau_solve_vjp.  torch's convention for a holomorphic map is
grad_t = J^H grad_tau, the C ABI returns the holomorphic pull-back J^T v, so
grad_t = conj(vjp(conj(grad_tau))).  Sites are assumed to own their store column
(store index == site index), as in problems built with n_species=None.
"""

from __future__ import annotations

import numpy as np
import torch

from lsms_b200 import tau as T


class Tau00(torch.autograd.Function):
    @staticmethod
    def forward(ctx, t_sites, solver, prob, iie):
        t = t_sites.detach().cpu().numpy()
        b = prob.kkrsz_ns
        store = prob.tmat_store.copy()
        for s in range(t.shape[0]):
            store[s, iie, :b * b] = t[s].T.reshape(-1)
        prob.tmat_store = store
        solver.load_problem(prob)
        jobs = T.make_jobs([(0, iie, 0, prob.energies[iie])])
        tau = solver.solve_jobs(jobs, T.PREC_FP64)[0].reshape(b, b).T + t[0]
        ctx.solver, ctx.prob, ctx.iie = solver, prob, iie
        return torch.from_numpy(tau.copy())

    @staticmethod
    def backward(ctx, grad_tau):
        prob, iie = ctx.prob, ctx.iie
        jobs = T.make_jobs([(0, iie, 0, prob.energies[iie])])
        v = np.conj(grad_tau.detach().cpu().numpy())[None]
        _, tbar, _ = ctx.solver.solve_vjp(jobs, v, [prob.num_liz], want_logdet=False)
        return torch.from_numpy(np.conj(tbar[0])), None, None, None
