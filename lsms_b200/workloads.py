"""Seeded synthetic inputs for the tau00 solve.

LSMS produces the inputs of this path elsewhere (LIZ geometry in
src/Main/buildLIZandCommLists.cpp:136-410, single-site t-matrices in
src/SingleSite, the energy contour in src/Main/energyContourIntegration.cpp:85-137).
None of that is on the hot path, so the benchmark and the parity tests build the
same data structures from seeded recipes:

* LIZ: the central site plus whole coordination shells of a bcc or fcc lattice,
  sorted by distance with the central site first (buildLIZandCommLists.cpp:377).
* t-matrices: diagonal in L, ``t_l = -(1/kappa) sin(d_l) exp(i d_l)`` with
  phase shifts ``d_l ~ U(0, 1.2)`` per species, kappa = prel.
* tmatStore: the reference's column-major store, one column per stored site,
  ``blkSizeTmatStore = (2 (lmax+1)^2)^2`` complex numbers per energy
  (buildLIZandCommLists.cpp:552-555).  Non-collinear t-matrices use the
  ``(is*kkrsz + i, js*kkrsz + j)`` layout (calculateTauMatrix.cpp:158-169);
  collinear spin-polarised ones hold spin down at offset ``kkrsz^2``.
* energies: the Gauss-Legendre semicircle of src/Misc/congauss_c.f:90-99.
"""

from __future__ import annotations

import dataclasses
import itertools
import math

import numpy as np

# include/PhysicalConstants.hpp:5-8
ALPHA_INVERSE = 137.035999206
CPHOT = 2.0 * ALPHA_INVERSE
C2INV = 1.0 / (CPHOT * CPHOT)


def prel_of(energy: complex) -> complex:
    """Scattering wave number, calculateTauMatrix.cpp:846."""
    e = complex(energy)
    return complex(np.sqrt(e * (1.0 + e * C2INV)))


def lattice_shells(kind: str, a: float, nshells: int) -> np.ndarray:
    """Positions (3, L) of the central site and its first ``nshells`` shells."""
    if kind == "bcc":
        basis = [(0.0, 0.0, 0.0), (0.5, 0.5, 0.5)]
    elif kind == "fcc":
        basis = [(0.0, 0.0, 0.0), (0.5, 0.5, 0.0), (0.5, 0.0, 0.5), (0.0, 0.5, 0.5)]
    else:
        raise ValueError(f"unknown lattice {kind!r}")
    rng = range(-6, 7)
    pts = []
    for i, j, k in itertools.product(rng, rng, rng):
        for b in basis:
            p = (a * (i + b[0]), a * (j + b[1]), a * (k + b[2]))
            pts.append(p)
    pts = np.array(sorted(set(pts)), dtype=np.float64)
    d2 = np.round((pts ** 2).sum(1) / (a * a), 9)
    shells = np.unique(d2)
    keep = d2 <= shells[nshells]
    pts, d2 = pts[keep], d2[keep]
    order = np.lexsort((pts[:, 2], pts[:, 1], pts[:, 0], d2))
    return np.ascontiguousarray(pts[order].T)


def semicircle_contour(ebot: float, etop: float, npts: int, eibot: float = 0.0025,
                       extra_point: bool = False) -> np.ndarray:
    """Gauss-Legendre semicircle from ebot to etop (congauss_c.f:90-99)."""
    x, _ = np.polynomial.legendre.leggauss(npts)
    erad = 0.5 * (etop - ebot)
    e = 0.5 * (etop + ebot) + erad * np.exp(1j * 0.5 * math.pi * (1.0 - x))
    if extra_point:
        e = np.concatenate([e, [etop + 1j * eibot]])
    return e.astype(np.complex128)


def spin_trafo(evec) -> tuple[np.ndarray, np.ndarray]:
    """u, ud (column-major 2x2 as 4 complex) for moment direction evec,
    src/Misc/spin_trafo.f:1-59."""
    ex, ey, ez = (float(v) for v in evec)
    u = np.zeros(4, np.complex128)
    u[0] = math.sqrt(0.5 * (1.0 + ez))
    if abs(u[0]) < 1e-8:
        u[0], u[1], u[2] = 0.0, 1.0, 1.0
    else:
        u[1] = -0.5 * (ex + 1j * ey) / u[0]
        u[2] = 0.5 * (ex - 1j * ey) / u[0]
    u[3] = u[0]
    ud = np.array([np.conj(u[0]), np.conj(u[2]), np.conj(u[1]), np.conj(u[3])])
    return u, ud


def t_diagonal(delta_l: np.ndarray, lmax: int, prel: complex) -> np.ndarray:
    """kkrsz x kkrsz diagonal t: t_l = -(1/kappa) sin d_l exp(i d_l)."""
    kkrsz = (lmax + 1) ** 2
    t = np.zeros((kkrsz, kkrsz), np.complex128)
    for l in range(lmax + 1):
        tl = -(1.0 / prel) * math.sin(delta_l[l]) * np.exp(1j * delta_l[l])
        for m in range(-l, l + 1):
            k = l * (l + 1) + m
            t[k, k] = tl
    return t


@dataclasses.dataclass
class Problem:
    """One atom's LIZ, the t-matrix store and the energies to solve at.

    Field layouts follow the reference's boundary types: ``liz_pos`` is
    AtomData::LIZPos (3, numLIZ), ``tmat_store`` is LocalTypeInfo::tmatStore
    viewed as (nstore, group_size, blk) C-order == column-major (blk*group, nstore).
    """

    lmax: int
    n_spin_cant: int
    n_spin_pola: int
    liz_pos: np.ndarray          # (3, L) float64
    liz_lmax: np.ndarray         # (L,) int32
    liz_store_idx: np.ndarray    # (L,) int32
    tmat_store: np.ndarray       # (nstore, group_size, blk) complex128
    energies: np.ndarray         # (group_size,) complex128
    ubr: np.ndarray              # (4,) complex128, central site spin frame
    ubrd: np.ndarray

    @property
    def kkrsz(self) -> int:
        return (self.lmax + 1) ** 2

    @property
    def kkrsz_ns(self) -> int:
        return self.n_spin_cant * self.kkrsz

    @property
    def num_liz(self) -> int:
        return int(self.liz_pos.shape[1])

    @property
    def nrmat_ns(self) -> int:
        return self.n_spin_cant * int(((self.liz_lmax + 1) ** 2).sum())

    @property
    def blk(self) -> int:
        return (2 * self.kkrsz) ** 2

    def t_block(self, store: int, iie: int, ispin: int = 0) -> np.ndarray:
        """kkrsz_ns x kkrsz_ns t-matrix of a stored site (column-major block)."""
        b = self.kkrsz_ns
        off = b * b * ispin if self.n_spin_pola != self.n_spin_cant else 0
        flat = self.tmat_store[store, iie, off:off + b * b]
        return flat.reshape(b, b).T.copy()


def make_problem(lattice: str, a: float, nshells: int, lmax: int, energies,
                 seed: int, n_species: int | None = 1, n_spin_cant: int = 1,
                 n_spin_pola: int = 1, liz_lmax=None) -> Problem:
    """Seeded problem.  ``n_species=None`` gives every LIZ site its own store
    column; otherwise sites draw one of ``n_species`` phase-shift sets."""
    rng = np.random.default_rng(seed)
    pos = lattice_shells(lattice, a, nshells)
    L = pos.shape[1]
    energies = np.asarray(energies, np.complex128).reshape(-1)
    if n_species is None:
        nstore = L
        store_idx = np.arange(L, dtype=np.int32)
    else:
        nstore = n_species
        store_idx = rng.integers(0, n_species, size=L).astype(np.int32)
        store_idx[0] = 0
    kkrsz = (lmax + 1) ** 2
    b = n_spin_cant * kkrsz
    blk = (2 * kkrsz) ** 2
    nspin_t = 2 if (n_spin_pola == 2 or n_spin_cant == 2) else 1
    deltas = rng.uniform(0.0, 1.2, size=(nstore, nspin_t, lmax + 1))
    evecs = rng.normal(size=(nstore, 3))
    evecs /= np.linalg.norm(evecs, axis=1, keepdims=True)
    store = np.zeros((nstore, energies.size, blk), np.complex128)
    for s in range(nstore):
        for ie, e in enumerate(energies):
            p = prel_of(e)
            if n_spin_cant == 2:
                tu = t_diagonal(deltas[s, 0], lmax, p)
                td = t_diagonal(deltas[s, 1], lmax, p)
                u, ud = spin_trafo(evecs[s])
                U = u.reshape(2, 2, order="F")
                Ud = ud.reshape(2, 2, order="F")
                # global-frame t = ud * diag(t_up, t_dn) * u, per L element
                tg = np.zeros((b, b), np.complex128)
                loc = [[tu, np.zeros_like(tu)], [np.zeros_like(tu), td]]
                for is_ in range(2):
                    for js in range(2):
                        acc = np.zeros_like(tu)
                        for p_ in range(2):
                            for q in range(2):
                                acc += Ud[is_, p_] * loc[p_][q] * U[q, js]
                        tg[is_ * kkrsz:(is_ + 1) * kkrsz, js * kkrsz:(js + 1) * kkrsz] = acc
                store[s, ie, :b * b] = tg.T.reshape(-1)
            elif n_spin_pola == 2:
                for isp in range(2):
                    t = t_diagonal(deltas[s, isp], lmax, p)
                    store[s, ie, isp * b * b:(isp + 1) * b * b] = t.T.reshape(-1)
            else:
                t = t_diagonal(deltas[s, 0], lmax, p)
                store[s, ie, :b * b] = t.T.reshape(-1)
    if liz_lmax is None:
        liz_lmax = np.full(L, lmax, np.int32)
    liz_lmax = np.asarray(liz_lmax, np.int32)
    u0, ud0 = spin_trafo(evecs[store_idx[0]])
    return Problem(lmax=lmax, n_spin_cant=n_spin_cant, n_spin_pola=n_spin_pola,
                   liz_pos=pos, liz_lmax=liz_lmax, liz_store_idx=store_idx,
                   tmat_store=store, energies=energies, ubr=u0, ubrd=ud0)


# Named workloads (shapes of the reference's published configurations).
def config_small(seed: int = 1) -> Problem:
    """bcc a=5.42 bohr, central site + 2 shells (15 sites), lmax 3, N=240, E=0.6+0.005i."""
    return make_problem("bcc", 5.42, 2, 3, [0.6 + 0.005j], seed, n_species=1)


def config_n2160(seed: int = 2, npts: int = 31) -> Problem:
    """fcc a=6.82 bohr, 7 shells (135 sites), lmax 3, N=2160, binary alloy,
    31-point semicircle contour from -0.3 to 0.7 Ry."""
    return make_problem("fcc", 6.82, 7, 3, semicircle_contour(-0.3, 0.7, npts), seed,
                        n_species=2)


def config_noncollinear(seed: int = 4, npts: int = 16, nshells: int = 7) -> Problem:
    """fcc LIZ, kkrsz_ns = 32 (non-collinear), N = 32 * L."""
    return make_problem("fcc", 6.82, nshells, 3, semicircle_contour(-0.3, 0.7, npts), seed,
                        n_species=None, n_spin_cant=2, n_spin_pola=2)


@dataclasses.dataclass
class AtomLIZ:
    """One local atom: AtomData's LIZPos (3, L), LIZlmax, LIZStoreIdx and spin frame."""
    liz_pos: np.ndarray
    liz_lmax: np.ndarray
    liz_store_idx: np.ndarray
    ubr: np.ndarray
    ubrd: np.ndarray

    @property
    def num_liz(self) -> int:
        return int(self.liz_pos.shape[1])


@dataclasses.dataclass
class Batch:
    """Many local atoms sharing one tmatStore and one energy group (calculateAllTauMatrices)."""
    lmax: int
    n_spin_cant: int
    n_spin_pola: int
    tmat_store: np.ndarray       # (nstore, group_size, blk) complex128
    energies: np.ndarray
    atoms: list

    @property
    def kkrsz_ns(self) -> int:
        return self.n_spin_cant * (self.lmax + 1) ** 2

    def nrmat_ns(self, a: int) -> int:
        return self.n_spin_cant * int(((self.atoms[a].liz_lmax + 1) ** 2).sum())

    def problem(self, a: int) -> "Problem":
        """Atom a as a single-atom Problem (for the oracle)."""
        at = self.atoms[a]
        return Problem(lmax=self.lmax, n_spin_cant=self.n_spin_cant, n_spin_pola=self.n_spin_pola,
                       liz_pos=at.liz_pos, liz_lmax=at.liz_lmax, liz_store_idx=at.liz_store_idx,
                       tmat_store=self.tmat_store, energies=self.energies, ubr=at.ubr, ubrd=at.ubrd)


def _phase_shift_store(rng, nstore: int, energies, lmax: int, n_spin_cant: int,
                       delta_range=(0.0, 1.2)) -> tuple[np.ndarray, np.ndarray]:
    """tmatStore of phase-shift t-matrices (non-collinear: a random moment per store column,
    t = U^+ diag(t_up, t_dn) U per L element).  Returns (store, moment directions)."""
    kkrsz = (lmax + 1) ** 2
    b = n_spin_cant * kkrsz
    blk = (2 * kkrsz) ** 2
    deltas = rng.uniform(delta_range[0], delta_range[1], size=(nstore, 2, lmax + 1))
    evecs = rng.normal(size=(nstore, 3))
    evecs /= np.linalg.norm(evecs, axis=1, keepdims=True)
    store = np.zeros((nstore, len(energies), blk), np.complex128)
    for s in range(nstore):
        for ie, e in enumerate(energies):
            p = prel_of(e)
            if n_spin_cant == 2:
                tu, td = t_diagonal(deltas[s, 0], lmax, p), t_diagonal(deltas[s, 1], lmax, p)
                u, ud = spin_trafo(evecs[s])
                U, Ud = u.reshape(2, 2, order="F"), ud.reshape(2, 2, order="F")
                tg = np.zeros((b, b), np.complex128)
                loc = [[tu, 0 * tu], [0 * tu, td]]
                for is_ in range(2):
                    for js in range(2):
                        acc = sum(Ud[is_, p_] * loc[p_][q] * U[q, js] for p_ in range(2) for q in range(2))
                        tg[is_ * kkrsz:(is_ + 1) * kkrsz, js * kkrsz:(js + 1) * kkrsz] = acc
                store[s, ie, :b * b] = tg.T.reshape(-1)
            else:
                store[s, ie, :b * b] = t_diagonal(deltas[s, 0], lmax, p).T.reshape(-1)
    return store, evecs


def config_batched(seed: int = 3, n_atoms: int = 256) -> Batch:
    """Random fcc alloy (a = 6.82 bohr, two species 50/50) with 5% vacancies: every local atom's
    LIZ size is drawn from {43, 55, 79, 87, 135} (3..7 shells, N = 688..2160), lmax 3, 31-point
    contour plus etop + i eibot (32 energies).  Store columns: 0, 1 species, 2 vacancy (small
    phase shifts)."""
    rng = np.random.default_rng(seed)
    energies = semicircle_contour(-0.3, 0.7, 31, extra_point=True)
    store, _ = _phase_shift_store(rng, 3, energies, 3, 1)
    vac, _ = _phase_shift_store(rng, 1, energies, 3, 1, delta_range=(0.0, 0.05))
    store[2] = vac[0]
    shells = {3: 43, 4: 55, 5: 79, 6: 87, 7: 135}
    geo = {sh: lattice_shells("fcc", 6.82, sh) for sh in shells}
    atoms = []
    u0, ud0 = spin_trafo((0.0, 0.0, 1.0))
    for _ in range(n_atoms):
        sh = int(rng.choice(list(shells)))
        pos = geo[sh]
        L = pos.shape[1]
        st = rng.choice(3, size=L, p=[0.475, 0.475, 0.05]).astype(np.int32)
        st[0] = rng.integers(0, 2)
        atoms.append(AtomLIZ(pos, np.full(L, 3, np.int32), st, u0, ud0))
    return Batch(3, 1, 1, store, energies, atoms)


def config_noncollinear_batch(seed: int = 4, n_atoms: int = 64, npts: int = 16) -> Batch:
    """Non-collinear (kkrsz_ns = 32), fcc LIZ of 135 sites (N = 4320), 64 atoms x 16 contour
    energies.  135 store columns with spin-dependent phase shifts and a random moment each;
    atom a sees column (site + 7 a) mod 135 at each LIZ site."""
    rng = np.random.default_rng(seed)
    energies = semicircle_contour(-0.3, 0.7, npts)
    pos = lattice_shells("fcc", 6.82, 7)
    L = pos.shape[1]
    store, evecs = _phase_shift_store(rng, L, energies, 3, 2)
    atoms = []
    for a in range(n_atoms):
        st = ((np.arange(L) + 7 * a) % L).astype(np.int32)
        u, ud = spin_trafo(evecs[st[0]])
        atoms.append(AtomLIZ(pos, np.full(L, 3, np.int32), st, u, ud))
    return Batch(3, 2, 2, store, energies, atoms)


def config_adjoint_batch(seed: int = 5, n_atoms: int = 64, npts: int = 16) -> Batch:
    """fcc LIZ of 87 sites (N = 1392), lmax 3, 64 atoms x 16 contour energies; every LIZ site
    of every atom has its own store column (phase shifts drawn per column)."""
    rng = np.random.default_rng(seed)
    energies = semicircle_contour(-0.3, 0.7, npts)
    pos = lattice_shells("fcc", 6.82, 6)
    L = pos.shape[1]
    store, _ = _phase_shift_store(rng, L * n_atoms, energies, 3, 1)
    u0, ud0 = spin_trafo((0.0, 0.0, 1.0))
    atoms = [AtomLIZ(pos, np.full(L, 3, np.int32), np.arange(a * L, (a + 1) * L, dtype=np.int32), u0, ud0)
             for a in range(n_atoms)]
    return Batch(3, 1, 1, store, energies, atoms)
