"""ORACLE / TEST INFRASTRUCTURE ONLY: ctypes binding of oracle/_ref/libtauref.so.

The library is the reference's own C++ tau00 path (calculateTauMatrix.cpp,
buildKKRMatrix_CPU.cpp, linearSolvers_CPU.cpp, block_inverse.cpp,
zblock_lu_cpp.cpp, Coeficients/Indices/associatedLegendreFunction/quadrature)
compiled from the reference tree plus oracle/ref_*.{cpp,c} (shims and
restatements of the few Fortran helpers).  Solver ids follow
src/MultipleScattering/linearSolvers.hpp:18-199 (build 0x2000 = C++ build).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libtauref.so")

# Solver ids (linearSolvers.hpp) combined with the C++ build id 0x2000.
ZGESV = 0x2001
ZGETRF = 0x2002
ZBLOCKLU_CPP = 0x2005
BLOCK_INVERSE_CPP = 0x2F01

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle ref)")
        _lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        I = ctypes.c_int
        D = ctypes.c_double
        _lib.tauref_calculate.argtypes = [I, I, I, ctypes.c_uint, I, P, P, P, I, I, P, I, I,
                                          D, D, P, P, P]
        _lib.tauref_build_kkr.argtypes = [I, I, I, I, P, P, P, I, I, P, I, I, D, D, P]
        _lib.tauref_tables.argtypes = [I, P, P, P]
        _lib.tauref_tau_full.argtypes = [I, I, I, I, P, P, P, I, I, P, I, I, D, D, P]
        _lib.tauref_set_num_threads.argtypes = [I]
    return _lib


def set_num_threads(n: int) -> None:
    lib().tauref_set_num_threads(int(n))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def tables(lmax: int):
    """(cgnt[l3/2, j1, j2], illp[lm, lmp], ilp1[l]) after the reference's init."""
    kk = (lmax + 1) ** 2
    cg = np.zeros(((lmax + 1) * kk * kk,), np.float64)
    il = np.zeros((kk * kk,), np.complex128)
    i1 = np.zeros((2 * lmax + 1,), np.complex128)
    lib().tauref_tables(lmax, _ptr(cg), _ptr(il), _ptr(i1))
    return (cg.reshape(kk, kk, lmax + 1).transpose(2, 1, 0).copy(),
            il.reshape(kk, kk).T.copy(), i1)


def _common(prob):
    pos = np.ascontiguousarray(prob.liz_pos.T, np.float64)          # (L, 3)
    lm = np.ascontiguousarray(prob.liz_lmax, np.int32)
    si = np.ascontiguousarray(prob.liz_store_idx, np.int32)
    tm = np.ascontiguousarray(prob.tmat_store, np.complex128)
    return pos, lm, si, tm


def calculate_tau(prob, iie: int, ispin: int = 0, solver: int = ZBLOCKLU_CPP) -> np.ndarray:
    """tau00_l (b x b, or kkrsz x kkrsz x 4 for non-collinear) as the reference returns it."""
    pos, lm, si, tm = _common(prob)
    b = prob.kkrsz_ns
    out = np.zeros((b * b,), np.complex128)
    e = complex(prob.energies[iie])
    ubr = np.ascontiguousarray(prob.ubr, np.complex128)
    ubrd = np.ascontiguousarray(prob.ubrd, np.complex128)
    lib().tauref_calculate(prob.lmax, prob.n_spin_cant, prob.n_spin_pola, solver,
                           prob.num_liz, _ptr(pos), _ptr(lm), _ptr(si),
                           tm.shape[0], tm.shape[1], _ptr(tm), iie, ispin,
                           e.real, e.imag, _ptr(ubr), _ptr(ubrd), _ptr(out))
    return out


def build_kkr(prob, iie: int, ispin: int = 0) -> np.ndarray:
    """The reference's KKR matrix M (N x N, numpy [row, col])."""
    pos, lm, si, tm = _common(prob)
    n = prob.nrmat_ns
    m = np.zeros((n * n,), np.complex128)
    e = complex(prob.energies[iie])
    lib().tauref_build_kkr(prob.lmax, prob.n_spin_cant, prob.n_spin_pola, prob.num_liz,
                           _ptr(pos), _ptr(lm), _ptr(si), tm.shape[0], tm.shape[1], _ptr(tm),
                           iie, ispin, e.real, e.imag, _ptr(m))
    return m.reshape(n, n).T.copy()


def tau_full(prob, iie: int, ispin: int = 0) -> np.ndarray:
    """The reference's solveTauFullzgetrf on its own M: tau = M^-1 T (N x N, numpy [row, col])."""
    pos, lm, si, tm = _common(prob)
    n = prob.nrmat_ns
    out = np.zeros((n * n,), np.complex128)
    e = complex(prob.energies[iie])
    lib().tauref_tau_full(prob.lmax, prob.n_spin_cant, prob.n_spin_pola, prob.num_liz,
                          _ptr(pos), _ptr(lm), _ptr(si), tm.shape[0], tm.shape[1], _ptr(tm),
                          iie, ispin, e.real, e.imag, _ptr(out))
    return out.reshape(n, n).T.copy()
