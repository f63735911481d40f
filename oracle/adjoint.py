"""ORACLE / TEST INFRASTRUCTURE ONLY: derivative references for b200tau_solve_vjp.

The reference has no derivative code (no adjoint, no ln det M), so the derivatives of tau00 and
of ln det M with respect to a site's phase shifts are pinned two independent ways, both on the
reference's own KKR matrix:

* complex step with bicomplex numbers (h = 1e-20): the phase shift delta of one (site, l)
  becomes delta + j h with a second imaginary unit j (j^2 = -1, ij = ji), t(delta) and
  M = 1 - T G are evaluated in bicomplex arithmetic and the j part of tau00 (or of ln det M)
  divided by h is the derivative, free of subtractive cancellation.  G is the reference's
  structure-constant matrix, obtained from its own build (oracle/_ref, buildKKRMatrix_CPU.cpp)
  with every t set to the identity: M(t = 1) = 1 - G.
* central finite differences of the reference's own tau00 (calculateTauMatrix with the block-LU
  solver) re-solved at delta +/- eps, and of ln det of the reference's own M.

Phase-shift t-matrices (t_l = -(1/kappa) sin d_l e^{i d_l}, the workloads' recipe for collinear
sites) give dt_l / d d_l = -(1/kappa) e^{2 i d_l} = -(1/kappa) (1 - 2 i kappa t_l), so the
directional derivatives need only t itself.
"""

from __future__ import annotations

import copy

import numpy as np

from . import reflib


class Bicomplex:
    """a + j b with complex a, b (arrays), j^2 = -1 commuting with i.  Products drop nothing:
    (a + j b)(c + j d) = (a c - b d) + j (a d + b c)."""

    def __init__(self, a, b=None):
        self.a = np.asarray(a, np.complex128)
        self.b = np.zeros_like(self.a) if b is None else np.asarray(b, np.complex128)

    def __add__(self, o):
        o = o if isinstance(o, Bicomplex) else Bicomplex(o)
        return Bicomplex(self.a + o.a, self.b + o.b)

    def __sub__(self, o):
        o = o if isinstance(o, Bicomplex) else Bicomplex(o)
        return Bicomplex(self.a - o.a, self.b - o.b)

    def __neg__(self):
        return Bicomplex(-self.a, -self.b)

    def __mul__(self, o):  # elementwise
        o = o if isinstance(o, Bicomplex) else Bicomplex(o)
        return Bicomplex(self.a * o.a - self.b * o.b, self.a * o.b + self.b * o.a)

    def __matmul__(self, o):
        o = o if isinstance(o, Bicomplex) else Bicomplex(o)
        return Bicomplex(self.a @ o.a - self.b @ o.b, self.a @ o.b + self.b @ o.a)


def bc_solve(A: Bicomplex, B: Bicomplex) -> Bicomplex:
    """X with A X = B: A X = B splits into a(x) - b(y) = B.a, a(y) + b(x) = B.b, i.e. the real
    2 x 2 block system [[a, -b], [b, a]] [x; y] = [B.a; B.b] over the complex numbers."""
    n = A.a.shape[0]
    big = np.block([[A.a, -A.b], [A.b, A.a]])
    rhs = np.concatenate([B.a, B.b], axis=0)
    sol = np.linalg.solve(big, rhs)
    return Bicomplex(sol[:n], sol[n:])


def bc_logdet(A: Bicomplex) -> Bicomplex:
    """ln det (a + j b) = ln det a + j tr(a^-1 b) to first order in b (b = O(h), h = 1e-20:
    the dropped terms are O(h^2), far below double precision)."""
    sign, ld = np.linalg.slogdet(A.a)
    return Bicomplex(np.log(sign) + ld, np.trace(np.linalg.solve(A.a, A.b)))


def _prel(prob, iie):
    from lsms_b200.workloads import prel_of
    return prel_of(prob.energies[iie])


def structure_constants(prob, iie: int, ispin: int = 0) -> np.ndarray:
    """G (N x N, reference site order) from the reference's build with every t = 1."""
    p = copy.deepcopy(prob)
    b = p.kkrsz_ns
    eye = np.eye(b, dtype=np.complex128).T.reshape(-1)
    p.tmat_store = p.tmat_store.copy()
    p.tmat_store[:, :, :] = 0.0
    p.tmat_store[:, :, :b * b] = eye
    if p.n_spin_pola != p.n_spin_cant:
        p.tmat_store[:, :, b * b:2 * b * b] = eye
    return np.eye(prob.nrmat_ns, dtype=np.complex128) - reflib.build_kkr(p, iie, ispin)


def site_layout(prob):
    kks = ((prob.liz_lmax + 1) ** 2).astype(int)
    ns = prob.n_spin_cant
    offs = np.concatenate([[0], np.cumsum(ns * kks)]).astype(int)
    return kks, offs


def site_t(prob, site: int, iie: int, ispin: int = 0) -> np.ndarray:
    """Compact t of a LIZ site as it enters M (calculateTauMatrix.cpp:156-183)."""
    kks, _ = site_layout(prob)
    full = prob.t_block(int(prob.liz_store_idx[site]), iie, ispin)
    kk = prob.kkrsz
    sel = np.concatenate([np.arange(kks[site]), kk + np.arange(kks[site])]) if prob.n_spin_cant == 2 \
        else np.arange(kks[site])
    return full[np.ix_(sel, sel)]


def dt_ddelta(prob, site: int, l: int, iie: int, ispin: int = 0) -> np.ndarray:
    """d t_site / d delta_l for a collinear phase-shift site (compact, diagonal)."""
    kappa = _prel(prob, iie)
    t = site_t(prob, site, iie, ispin)
    d = np.zeros_like(t)
    for m in range(-l, l + 1):
        k = l * (l + 1) + m
        d[k, k] = -(1.0 / kappa) * (1.0 - 2j * kappa * t[k, k])
    return d


def complex_step(prob, iie: int, taubar: np.ndarray, pairs, ispin: int = 0, h: float = 1e-20):
    """For each (site, l): (d<taubar, tau00>/d delta, d ln det M / d delta) by the bicomplex step.
    tau00 is the raw central block [M^-1]_00 t_0 (reference site order: central site first)."""
    assert prob.n_spin_cant == 1, "phase-shift derivatives are set up for collinear sites"
    G = structure_constants(prob, iie, ispin)
    kks, offs = site_layout(prob)
    L = prob.num_liz
    N = int(offs[-1])
    T = np.zeros((N, N), np.complex128)
    for s in range(L):
        T[offs[s]:offs[s + 1], offs[s]:offs[s + 1]] = site_t(prob, s, iie, ispin)
    b = prob.kkrsz_ns
    out = []
    for site, l in pairs:
        dT = np.zeros((N, N), np.complex128)
        dT[offs[site]:offs[site + 1], offs[site]:offs[site + 1]] = h * dt_ddelta(prob, site, l, iie, ispin)
        Tb = Bicomplex(T, dT)
        M = Bicomplex(np.eye(N)) - Tb @ Bicomplex(G)
        rhs = Bicomplex(np.zeros((N, b)))
        rhs.a[:b] = T[:b, :b]
        rhs.b[:b] = dT[:b, :b]
        X = bc_solve(M, rhs)
        dtau = X.b[:b] / h
        dL = np.sum(taubar * dtau)
        dlogdet = bc_logdet(M).b / h
        out.append((dL, dlogdet))
    return out


def finite_difference(prob, iie: int, taubar: np.ndarray, site: int, l: int, ispin: int = 0,
                      eps: float = 1e-6):
    """Central differences in delta_l of the site's store column: the reference's tau00
    (calculateTauMatrix, block-LU solver) and ln det of the reference's M."""
    kappa = _prel(prob, iie)
    b = prob.kkrsz_ns
    store = int(prob.liz_store_idx[site])
    base = prob.tmat_store[store, iie].copy()

    def at(sign):
        p = copy.copy(prob)
        p.tmat_store = prob.tmat_store.copy()
        blk = base.copy()
        for m in range(-l, l + 1):
            k = l * (l + 1) + m
            t = blk[k + k * b]
            delta = np.angle(1.0 - 2j * kappa * t) / 2.0 + sign * eps
            blk[k + k * b] = -(1.0 / kappa) * np.sin(delta) * np.exp(1j * delta)
        p.tmat_store[store, iie] = blk
        tau = reflib.calculate_tau(p, iie, ispin, reflib.ZBLOCKLU_CPP).reshape(b, b).T
        tau = tau + p.t_block(int(p.liz_store_idx[0]), iie, ispin)
        sign_, ld = np.linalg.slogdet(reflib.build_kkr(p, iie, ispin))
        return np.sum(taubar * tau), np.log(sign_) + ld

    (lp, dp), (lm, dm) = at(+1), at(-1)
    dd = dp - dm
    dd = dd - 2j * np.pi * np.round(dd.imag / (2 * np.pi))  # branch of the complex logarithm
    return (lp - lm) / (2 * eps), dd / (2 * eps)
