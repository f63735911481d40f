"""ORACLE / TEST INFRASTRUCTURE ONLY: numpy restatement of the tau00 path.

A second, independently written checker beside ``oracle.reflib`` (the
reference's own C++ compiled as-is).  Each function cites the reference code it
restates:

* ``angular_tables``  - Indices.hpp:136-170, cgaunt_c.f90:3-109 + gaunt.f:1-119,
  ifacts_c.f:3-72, associatedLegendreFunction.hpp:33-69, quadrature.cpp:10-13.
* ``build_kkr``       - buildKKRMatrix_CPU.cpp:23-59 (Hankel, sin/cos powers),
  :96-176 (buildBGijCPU), :61-94 (spin-diagonal embed), :253-427 (M = 1 - t G);
  t gather as calculateTauMatrix.cpp:156-183 (F77 build semantics).
* ``schur_tau00``     - zblock_lu_cpp.cpp:19-86 + block_inverse.cpp:24-47 +
  linearSolvers_CPU.cpp:261-331 (delta = B D^-1 C, tau00 = (1-delta)^-1 t0).
* ``tau00_l``         - tau00Postprocess.cpp:52-101 (tau00 - t, trgtol rotation).
"""

from __future__ import annotations

import math

import numpy as np


def legendre_normalized(x: np.ndarray, lmax: int) -> np.ndarray:
    """P-bar_lm(x) at index l(l+1)/2+m (associatedLegendreFunction.hpp:33-69)."""
    x = np.asarray(x, np.float64)
    nd = (lmax + 1) * (lmax + 2) // 2
    out = np.zeros(x.shape + (nd,), np.float64)
    idx = lambda l, m: l * (l + 1) // 2 + m
    y = np.sqrt(1.0 - x * x)
    out[..., 0] = math.sqrt(1.0 / (4.0 * math.pi))
    for m in range(1, lmax + 1):
        out[..., idx(m, m)] = -math.sqrt((2 * m + 1) / (2 * m)) * y * out[..., idx(m - 1, m - 1)]
        out[..., idx(m, m - 1)] = math.sqrt(2 * m + 1) * x * out[..., idx(m - 1, m - 1)]
    for m in range(0, lmax):
        for l in range(m + 2, lmax + 1):
            a = math.sqrt((4 * l * l - 1) / (l * l - m * m))
            b = math.sqrt(((l - 1) ** 2 - m * m) / (4 * (l - 1) ** 2 - 1))
            out[..., idx(l, m)] = a * (x * out[..., idx(l - 1, m)] - b * out[..., idx(l - 2, m)])
    return out


def angular_tables(lmax: int):
    """lofk/mofk for 2*lmax, Gaunt numbers cgnt[l3/2, j1, j2], illp, ilp1."""
    lofk, mofk = [], []
    for l in range(2 * lmax + 1):
        for m in range(-l, l + 1):
            lofk.append(l)
            mofk.append(m)
    lofk = np.array(lofk)
    mofk = np.array(mofk)
    # cgaunt: 2(2lmax+1) Gauss-Legendre nodes on [-1,1] (ascending), only the
    # first 2lmax+1 used, normalised P_lm up to 2 lmax.
    ng = 2 * (2 * lmax + 1)
    tg, wg = np.polynomial.legendre.leggauss(ng)
    n1 = 2 * lmax + 1
    plmg = legendre_normalized(tg[:n1], 2 * lmax)  # (n1, ndlm)

    def jl(l, m):
        return (1, l * (l + 1) // 2 + m) if m >= 0 else ((-1) ** abs(m), l * (l + 1) // 2 - m)

    kk = (lmax + 1) ** 2
    cgnt = np.zeros((lmax + 1, kk, kk))
    for j2 in range(kk):
        l2, m2 = lofk[j2], mofk[j2]
        for j1 in range(kk):
            l1, m1 = lofk[j1], mofk[j1]
            m3 = m2 - m1
            for l3 in range(l1 + l2, max(abs(m3), abs(l1 - l2)) - 1, -2):
                f1, i1 = jl(l1, m1)
                f2, i2 = jl(l2, -m2)
                f3, i3 = jl(l3, m3)
                v = float(np.sum(wg[:n1] * plmg[:, i1] * plmg[:, i2] * plmg[:, i3]))
                if abs(v) < 1e-14:
                    v = 0.0
                else:
                    v = 4.0 * math.pi * v * f1 * (1 - 2 * (abs(m2) % 2)) * f2 * f3
                cgnt[l3 // 2, j1, j2] = v
    il = np.array([1j ** l for l in range(2 * lmax + 1)])
    illp = np.zeros((kk, kk), np.complex128)
    for a in range(kk):
        for b in range(kk):
            illp[a, b] = il[lofk[a]] / il[lofk[b]]
    ilp1 = il * 1j
    return lofk, mofk, cgnt, illp, ilp1


def gij_blocks(rij: np.ndarray, prel: complex, lmax: int, tables=None) -> np.ndarray:
    """G_ij (kkrsz x kkrsz, rows = site i L, cols = site j L) for displacement
    vectors rij (P, 3), buildKKRMatrix_CPU.cpp:96-176."""
    lofk, mofk, cgnt, illp, ilp1 = tables if tables is not None else angular_tables(lmax)
    rij = np.atleast_2d(rij)
    lend = 2 * lmax
    r = np.sqrt((rij ** 2).sum(1))
    z = prel * r
    hfn = np.zeros((rij.shape[0], lend + 1), np.complex128)
    hfn[:, 0] = -1j
    hfn[:, 1] = -1.0 - 1j / z
    for l in range(1, lend):
        hfn[:, l + 1] = (2.0 * l + 1.0) * hfn[:, l] / z - hfn[:, l - 1]
    fac = np.exp(1j * z) / r
    hfn = -hfn * fac[:, None] * ilp1[None, :lend + 1]
    plm = legendre_normalized(rij[:, 2] / r, lend)
    pmag = np.sqrt(rij[:, 0] ** 2 + rij[:, 1] ** 2)
    ok = pmag > 1e-6
    c1 = np.where(ok, rij[:, 0] / np.where(ok, pmag, 1.0), 0.0)
    s1 = np.where(ok, rij[:, 1] / np.where(ok, pmag, 1.0), 0.0)
    cosm = np.zeros((rij.shape[0], lend + 1))
    sinm = np.zeros((rij.shape[0], lend + 1))
    cosm[:, 0] = 1.0
    if lend >= 1:
        cosm[:, 1], sinm[:, 1] = c1, s1
    for m in range(2, lend + 1):
        cosm[:, m] = cosm[:, m - 1] * c1 - sinm[:, m - 1] * s1
        sinm[:, m] = sinm[:, m - 1] * c1 + cosm[:, m - 1] * s1
    dlm = np.zeros((rij.shape[0], (lend + 1) ** 2), np.complex128)
    for l in range(lend + 1):
        j = l * (l + 1)
        ll = j // 2
        dlm[:, j] = hfn[:, l] * plm[:, ll]
        m1m = 1.0
        for m in range(1, l + 1):
            m1m = -m1m
            f = plm[:, ll + m] * (cosm[:, m] + 1j * sinm[:, m])
            dlm[:, j - m] = hfn[:, l] * m1m * f
            dlm[:, j + m] = hfn[:, l] * np.conj(f)
    kk = (lmax + 1) ** 2
    g = np.zeros((rij.shape[0], kk, kk), np.complex128)
    pi4 = 4.0 * 2.0 * math.asin(1.0)
    for lm1 in range(kk):
        l1, m1 = lofk[lm1], mofk[lm1]
        for lm2 in range(kk):
            l2, m2 = lofk[lm2], mofk[lm2]
            m3 = m2 - m1
            llow = max(abs(m3), abs(l1 - l2))
            acc = np.zeros(rij.shape[0], np.complex128)
            for l3 in range(l1 + l2, llow - 1, -2):
                acc = acc + cgnt[l3 // 2, lm1, lm2] * dlm[:, l3 * (l3 + 1) + m3]
            g[:, lm2, lm1] = acc * (pi4 * illp[lm2, lm1])
    return g


def build_kkr(prob, iie: int, ispin: int = 0) -> np.ndarray:
    """M = 1 - t G over the LIZ in the reference's site order (numpy [row, col])."""
    lmax = prob.lmax
    ns = prob.n_spin_cant
    tables = angular_tables(lmax)
    L = prob.num_liz
    kks = ((prob.liz_lmax + 1) ** 2).astype(int)
    offs = np.concatenate([[0], np.cumsum(ns * kks)])
    n = int(offs[-1])
    m = np.eye(n, dtype=np.complex128)
    pos = prob.liz_pos.T
    ii, jj = np.nonzero(~np.eye(L, dtype=bool))
    g = gij_blocks(pos[ii] - pos[jj], _prel(prob, iie), lmax, tables)
    for p, (i, j) in enumerate(zip(ii, jj)):
        ki, kj = kks[i], kks[j]
        gij = g[p, :ki, :kj]
        if ns == 2:
            bg = np.zeros((2 * ki, 2 * kj), np.complex128)
            bg[:ki, :kj] = gij
            bg[ki:, kj:] = gij
        else:
            bg = gij
        t = _site_t(prob, int(prob.liz_store_idx[i]), iie, ispin, ki)
        m[offs[i]:offs[i + 1], offs[j]:offs[j + 1]] = -(t @ bg)
    return m


def _prel(prob, iie):
    from lsms_b200.workloads import prel_of
    return prel_of(prob.energies[iie])


def _site_t(prob, store: int, iie: int, ispin: int, kk_site: int) -> np.ndarray:
    """t of a LIZ site reduced to its own lmax, F77 gather calculateTauMatrix.cpp:156-183."""
    full = prob.t_block(store, iie, ispin)
    kk = prob.kkrsz
    if prob.n_spin_cant == 2:
        sel = np.concatenate([np.arange(kk_site), kk + np.arange(kk_site)])
    else:
        sel = np.arange(kk_site)
    return full[np.ix_(sel, sel)]


def schur_tau00(m: np.ndarray, t0: np.ndarray) -> np.ndarray:
    """tau00 = (1 - delta)^-1 t0 with delta = B D^-1 C (zero A block), the
    zblock_lu / solveTau00zblocklu_cpp contract."""
    b = t0.shape[0]
    B = m[:b, b:]
    C = m[b:, :b]
    D = m[b:, b:]
    delta = B @ np.linalg.solve(D, C)
    return np.linalg.solve(np.eye(b) - delta, t0)


def trgtol(nr: int, nc: int, u: np.ndarray, ud: np.ndarray, mg: np.ndarray) -> np.ndarray:
    """trgtol.f:3-110: returns ml (nr, nc, 4) with block k the column-major (u mg ud) entry."""
    U = u.reshape(2, 2, order="F")
    Ud = ud.reshape(2, 2, order="F")
    blocks = [[mg[:nr, :nc], mg[:nr, nc:]], [mg[nr:, :nc], mg[nr:, nc:]]]
    out = np.zeros((nr, nc, 4), np.complex128)
    for k, (a, c) in enumerate([(0, 0), (1, 0), (0, 1), (1, 1)]):
        acc = np.zeros((nr, nc), np.complex128)
        for p in range(2):
            for q in range(2):
                acc += U[a, p] * blocks[p][q] * Ud[q, c]
        out[:, :, k] = acc
    return out


def tau00_l(prob, tau00: np.ndarray, iie: int, ispin: int = 0) -> np.ndarray:
    """tau00 - t0, rotated to the local frame for n_spin_cant = 2; returned as
    the flat column-major array the reference writes into tau00_l."""
    t0 = prob.t_block(int(prob.liz_store_idx[0]), iie, ispin)
    d = tau00 - t0
    if prob.n_spin_cant == 2:
        kk = prob.kkrsz
        ml = trgtol(kk, kk, prob.ubr, prob.ubrd, d)
        return np.concatenate([ml[:, :, k].T.reshape(-1) for k in range(4)])
    return d.T.reshape(-1)


def solve(prob, iie: int, ispin: int = 0) -> np.ndarray:
    m = build_kkr(prob, iie, ispin)
    t0 = prob.t_block(int(prob.liz_store_idx[0]), iie, ispin)
    return tau00_l(prob, schur_tau00(m, t0), iie, ispin)
