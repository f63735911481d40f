"""Python host side of b200tau, mirroring the reference's tau00 call surface.

The names follow src/MultipleScattering/calculateTauMatrix.cpp and linearSolvers_CPU.cpp:

* ``TauSolver.calculate_tau_matrix``   <- ``calculateTauMatrix(lsms, local, atom,
  localAtomIndex, ispin, energy, prel, tau00_l, m, iie)`` (calculateTauMatrix.cpp:320-837)
* ``TauSolver.calculate_all_tau_matrices`` <- ``calculateAllTauMatrices`` (:841-945), batched over
  every (atom, energy, spin) of an energy group in one device pass
* ``TauSolver.solve_tau00_dense``      <- ``solveTau00zblocklu_cpp`` / ``solveTau00zgesv``
  (linearSolvers_CPU.cpp:76-96,261-331)
* ``TauSolver.upload_tmat`` / ``set_atom`` <- ``DeviceStorage::copyTmatStoreToDevice`` and
  ``DeviceAtom::copyFromAtom`` (src/Accelerator/DeviceStorage.cu:284-303,341-404)

Everything goes through the C ABI of ``lsms_b200/_lib/libb200tau.so`` (include/b200tau.h).  There
is no CPU fallback: if the library or a GPU is missing, construction raises.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import workloads

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libb200tau.so")

OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_OOM = 3
ERR_SINGULAR = 4
ERR_TIMEOUT = 5
ERR_STATE = 6
PREC_FP64 = 0
PREC_MIXED = 1
ENGINE_TENSOR = 0
ENGINE_SIMT = 1
SWEEP_FP64 = 0
SWEEP_FP32 = 1
PIVOT_AUTO = 0
PIVOT_BLOCK = 1
PIVOT_PANEL = 2

# Symbols declared in include/b200tau.h.
EXPORTS = (
    "b200tau_create", "b200tau_destroy", "b200tau_last_error", "b200tau_stream",
    "b200tau_upload_tmat", "b200tau_set_atom", "b200tau_solve", "b200tau_solve_device",
    "b200tau_sync", "b200tau_solve_dense", "b200tau_build_kkr", "b200tau_last_launch_count",
    "b200tau_gaunt_numbers", "b200tau_set_refinement", "b200tau_set_profiling",
    "b200tau_profile_read", "b200tau_set_mixed_engine", "b200tau_solve_dense_noalloc",
    "b200tau_profile_phases", "b200tau_set_mixed_sweep", "b200tau_solve_vjp",
    "b200tau_last_fallback_count", "b200tau_set_mixed_fallback", "b200tau_set_build_wait",
    "b200tau_set_pivoting", "b200tau_solve_tau_full", "b200tau_set_graphs",
    "b200tau_set_keep_factors", "b200tau_set_paired_steps",
    "b200tau_autotune_paired_steps",
)


class B200TauError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"b200tau error {code}: {msg}")
        self.code = code


class Job(ctypes.Structure):
    """``b200tau_job``: one (atom, energy, spin) solve."""
    _fields_ = [("atom", ctypes.c_int), ("iie", ctypes.c_int), ("ispin", ctypes.c_int),
                ("reserved", ctypes.c_int), ("energy", ctypes.c_double * 2),
                ("prel", ctypes.c_double * 2)]


_lib = None


def load_library():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"b200tau CUDA library not built: {LIB_PATH} (python -m lsms_b200.build)")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, L, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_long, ctypes.c_double
    lib.b200tau_create.argtypes = [ctypes.POINTER(P), I, I, I, I]
    lib.b200tau_destroy.argtypes = [P]
    lib.b200tau_destroy.restype = None
    lib.b200tau_last_error.argtypes = [P]
    lib.b200tau_last_error.restype = ctypes.c_char_p
    lib.b200tau_stream.argtypes = [P]
    lib.b200tau_stream.restype = P
    lib.b200tau_upload_tmat.argtypes = [P, P, L, I, I]
    lib.b200tau_set_atom.argtypes = [P, I, I, P, P, P, P, P]
    lib.b200tau_solve.argtypes = [P, P, I, I, P]
    lib.b200tau_solve_device.argtypes = [P, P, I, I, P]
    lib.b200tau_sync.argtypes = [P]
    lib.b200tau_solve_dense.argtypes = [P, P, I, I, P, I, I, P]
    lib.b200tau_build_kkr.argtypes = [P, P, P, I]
    lib.b200tau_last_launch_count.argtypes = [P]
    lib.b200tau_last_launch_count.restype = L
    lib.b200tau_gaunt_numbers.argtypes = [I, P]
    lib.b200tau_set_refinement.argtypes = [P, I, I]
    lib.b200tau_set_profiling.argtypes = [P, I]
    lib.b200tau_set_mixed_engine.argtypes = [P, I]
    lib.b200tau_profile_read.argtypes = [P, P, P, P]
    lib.b200tau_profile_phases.argtypes = [P, P]
    lib.b200tau_set_mixed_sweep.argtypes = [P, I]
    lib.b200tau_solve_vjp.argtypes = [P, P, I, P, P, P, P]
    lib.b200tau_last_fallback_count.argtypes = [P]
    lib.b200tau_last_fallback_count.restype = L
    lib.b200tau_set_mixed_fallback.argtypes = [P, I]
    lib.b200tau_set_build_wait.argtypes = [P, L]
    lib.b200tau_set_pivoting.argtypes = [P, I]
    lib.b200tau_solve_tau_full.argtypes = [P, P, P, I]
    lib.b200tau_set_graphs.argtypes = [P, I]
    lib.b200tau_set_paired_steps.argtypes = [P, I]
    lib.b200tau_autotune_paired_steps.argtypes = [P, P, I, P, I, I, P, P]
    lib.b200tau_set_keep_factors.argtypes = [P, I]
    _lib = lib
    return lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def gaunt_numbers(lmax: int = 3) -> np.ndarray:
    """The library's Gaunt table as cgnt[l3/2, j1, j2] (host-only call)."""
    kk = (lmax + 1) ** 2
    out = np.zeros(((lmax + 1) * kk * kk,), np.float64)
    rc = load_library().b200tau_gaunt_numbers(lmax, _ptr(out))
    if rc != OK:
        raise B200TauError(rc, "b200tau_gaunt_numbers")
    return out.reshape(kk, kk, lmax + 1).transpose(2, 1, 0).copy()


def make_jobs(specs) -> ctypes.Array:
    """specs: iterable of (atom, iie, ispin, energy) -> b200tau_job array (prel computed as
    calculateTauMatrix.cpp:846)."""
    specs = list(specs)
    arr = (Job * max(len(specs), 1))()
    for k, (atom, iie, ispin, energy) in enumerate(specs):
        e = complex(energy)
        p = workloads.prel_of(e)
        arr[k].atom, arr[k].iie, arr[k].ispin, arr[k].reserved = int(atom), int(iie), int(ispin), 0
        arr[k].energy[0], arr[k].energy[1] = e.real, e.imag
        arr[k].prel[0], arr[k].prel[1] = p.real, p.imag
    return arr


class TauSolver:
    """A b200tau context on one GPU (LSMSSystemParameters: maxlmax, n_spin_cant, n_spin_pola)."""

    def __init__(self, lmax: int = 3, n_spin_cant: int = 1, n_spin_pola: int = 1, device: int = 0):
        self.lib = load_library()
        self.ctx = ctypes.c_void_p()
        rc = self.lib.b200tau_create(ctypes.byref(self.ctx), device, lmax, n_spin_cant, n_spin_pola)
        if rc != OK:
            raise B200TauError(rc, "b200tau_create failed (no CUDA device or bad parameters)")
        self.lmax, self.n_spin_cant, self.n_spin_pola = lmax, n_spin_cant, n_spin_pola
        self.kkrsz = (lmax + 1) ** 2
        self.kkrsz_ns = n_spin_cant * self.kkrsz
        self.atom_n = {}  # atom index -> N of its KKR matrix (from set_atom)

    # -- plumbing -------------------------------------------------------------------------
    def close(self):
        if self.ctx:
            self.lib.b200tau_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != OK:
            raise B200TauError(rc, self.lib.b200tau_last_error(self.ctx).decode())

    @property
    def stream(self) -> int:
        return int(self.lib.b200tau_stream(self.ctx) or 0)

    @property
    def last_launch_count(self) -> int:
        return int(self.lib.b200tau_last_launch_count(self.ctx))

    @property
    def last_fallback_count(self) -> int:
        """Mixed-precision jobs of the last solve re-solved by FP64 block LU."""
        return int(self.lib.b200tau_last_fallback_count(self.ctx))

    def set_refinement(self, prec: int, steps: int):
        """FP64 refinement steps of a precision (see b200tau_set_refinement)."""
        self._check(self.lib.b200tau_set_refinement(self.ctx, prec, steps))

    def set_mixed_engine(self, engine: int):
        """Trailing-update engine of the mixed path: ENGINE_TENSOR (tcgen05) or ENGINE_SIMT."""
        self._check(self.lib.b200tau_set_mixed_engine(self.ctx, engine))

    def set_mixed_fallback(self, enable: bool):
        """Re-solve unconverged mixed-precision jobs by FP64 block LU (default on)."""
        self._check(self.lib.b200tau_set_mixed_fallback(self.ctx, int(bool(enable))))

    def set_keep_factors(self, enable: bool):
        """Keep an FP64 solve's factors for the next solve_vjp on the same jobs."""
        self._check(self.lib.b200tau_set_keep_factors(self.ctx, int(bool(enable))))

    def set_graphs(self, enable: bool):
        """Each wave as one captured CUDA graph (default) or as separate launches."""
        self._check(self.lib.b200tau_set_graphs(self.ctx, int(bool(enable))))

    def set_paired_steps(self, min_rest: int):
        """Paired elimination steps (one tensor-core pass for two steps' trailing updates) while the
        trailing block has at least min_rest columns; 0 turns them off (default 768)."""
        self._check(self.lib.b200tau_set_paired_steps(self.ctx, int(min_rest)))

    def autotune_paired_steps(self, jobs, candidates=None, reps: int = 2):
        """Time mixed solves of `jobs` at each paired-steps threshold (default 0, 512, 768, 1024,
        1280, 1536), keep the fastest as the setting; returns (chosen, {candidate: ms})."""
        cand = [0, 512, 768, 1024, 1280, 1536] if candidates is None else [int(c) for c in candidates]
        ca = np.ascontiguousarray(cand, np.int32)
        ms = np.zeros(len(cand), np.float32)
        chosen = ctypes.c_int()
        self._check(self.lib.b200tau_autotune_paired_steps(self.ctx, ctypes.cast(jobs, ctypes.c_void_p), len(jobs),
                                                           _ptr(ca), len(cand), int(reps),
                                                           ctypes.byref(chosen), _ptr(ms)))
        return chosen.value, {c: float(t) for c, t in zip(cand, ms)}

    def autotune_paired_steps_by_size(self, jobs, sample: int = 64, candidates=(0, 768, 1280), reps: int = 2):
        """Tune the paired-steps threshold per size bucket (N rounded up to 64) of a mixed batch:
        for each bucket, autotune_paired_steps on up to `sample` of its jobs; waves whose largest N
        falls in a tuned bucket then use its threshold.  Returns {bucket: (chosen, {candidate: ms})}."""
        buckets = {}
        for j in jobs:
            n = self.atom_n[j.atom]
            buckets.setdefault((n + 63) // 64 * 64, []).append(j)
        table = {}
        for bucket in sorted(buckets, reverse=True):
            sub = buckets[bucket][:sample]
            table[bucket] = self.autotune_paired_steps((Job * len(sub))(*sub), candidates, reps)
        return table

    def set_pivoting(self, mode: int):
        """Row pivoting of the elimination: PIVOT_AUTO (default), PIVOT_BLOCK or PIVOT_PANEL."""
        self._check(self.lib.b200tau_set_pivoting(self.ctx, mode))

    def set_build_wait(self, polls: int):
        """Bound of the KKR build's first wait on its table copy (0: give up at once); a wait
        that runs out makes the call return ERR_TIMEOUT (see b200tau_set_build_wait)."""
        self._check(self.lib.b200tau_set_build_wait(self.ctx, int(polls)))

    def set_mixed_sweep(self, sweep: int):
        """Arithmetic of the mixed path's correction solve: SWEEP_FP32 (default) or SWEEP_FP64."""
        self._check(self.lib.b200tau_set_mixed_sweep(self.ctx, sweep))

    def set_profiling(self, enable: bool):
        self._check(self.lib.b200tau_set_profiling(self.ctx, int(bool(enable))))

    def profile_read(self):
        """(device ms, launches, algorithmic FLOPs) of the timed trailing-update launches."""
        ms, n, fl = ctypes.c_double(), ctypes.c_long(), ctypes.c_double()
        self._check(self.lib.b200tau_profile_read(self.ctx, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(fl)))
        return ms.value, n.value, fl.value

    def profile_phases(self) -> dict:
        """Device ms per phase since profiling was enabled: KKR build, elimination, refinement."""
        ms = (ctypes.c_double * 3)()
        self._check(self.lib.b200tau_profile_phases(self.ctx, ms))
        return {"build_ms": ms[0], "eliminate_ms": ms[1], "refine_ms": ms[2]}

    # -- uploads (DeviceStorage / DeviceAtom) ----------------------------------------------
    def upload_tmat(self, tmat_store: np.ndarray):
        """tmat_store: (nstore, group_size, blk) complex128 == column-major (blk*group, nstore)."""
        ts = np.ascontiguousarray(tmat_store, np.complex128)
        nstore, group, blk = ts.shape
        self._check(self.lib.b200tau_upload_tmat(self.ctx, _ptr(ts), blk * group, nstore, blk))

    def set_atom(self, atom: int, liz_pos: np.ndarray, liz_lmax, liz_store_idx, ubr=None, ubrd=None):
        pos = np.ascontiguousarray(np.asarray(liz_pos, np.float64).T)  # (L, 3) == column-major 3 x L
        lm = np.ascontiguousarray(liz_lmax, np.int32)
        si = np.ascontiguousarray(liz_store_idx, np.int32)
        u = None if ubr is None else np.ascontiguousarray(ubr, np.complex128)
        ud = None if ubrd is None else np.ascontiguousarray(ubrd, np.complex128)
        self._check(self.lib.b200tau_set_atom(self.ctx, atom, pos.shape[0], _ptr(pos), _ptr(lm), _ptr(si),
                                              None if u is None else _ptr(u),
                                              None if ud is None else _ptr(ud)))
        self.atom_n[atom] = self.n_spin_cant * int(sum((int(l) + 1) ** 2 for l in lm))

    def load_problem(self, prob: workloads.Problem, atom: int = 0, upload_tmat: bool = True):
        if upload_tmat:
            self.upload_tmat(prob.tmat_store)
        self.set_atom(atom, prob.liz_pos, prob.liz_lmax, prob.liz_store_idx, prob.ubr, prob.ubrd)

    # -- solves ---------------------------------------------------------------------------
    def solve_jobs(self, jobs, prec: int = PREC_FP64) -> np.ndarray:
        """Batched solve; returns (njobs, kkrsz_ns^2) complex tau00_l (column-major blocks)."""
        n = len(jobs)
        out = np.zeros((max(n, 1), self.kkrsz_ns * self.kkrsz_ns), np.complex128)
        self._check(self.lib.b200tau_solve(self.ctx, ctypes.cast(jobs, ctypes.c_void_p), n, prec, _ptr(out)))
        return out[:n]

    def solve_jobs_device(self, jobs, out_dev_ptr: int, prec: int = PREC_FP64):
        """Enqueue a batched solve writing to device memory (no host synchronisation)."""
        self._check(self.lib.b200tau_solve_device(self.ctx, ctypes.cast(jobs, ctypes.c_void_p), len(jobs), prec,
                                                  ctypes.c_void_p(out_dev_ptr)))

    def sync(self):
        self._check(self.lib.b200tau_sync(self.ctx))

    def calculate_tau_matrix(self, atom: int, ispin: int, energy: complex, iie: int,
                             prec: int = PREC_FP64) -> np.ndarray:
        """tau00_l of one (atom, energy, spin) as calculateTauMatrix writes it (flat, kkrsz_ns^2)."""
        return self.solve_jobs(make_jobs([(atom, iie, ispin, energy)]), prec)[0]

    def calculate_all_tau_matrices(self, atoms, energies, iies=None, prec: int = PREC_FP64) -> np.ndarray:
        """tau00_l for every local atom x energy (x spin when collinear-polarised), batched.
        Returns (n_energies, n_spin, n_atoms, kkrsz_ns^2)."""
        atoms = list(atoms)
        energies = np.asarray(energies, np.complex128).reshape(-1)
        iies = list(range(energies.size)) if iies is None else list(iies)
        nspin = 2 if (self.n_spin_pola != self.n_spin_cant) else 1
        specs = [(a, iie, s, e) for iie, e in zip(iies, energies) for s in range(nspin) for a in atoms]
        out = self.solve_jobs(make_jobs(specs), prec)
        return out.reshape(energies.size, nspin, len(atoms), -1)

    def solve_tau00_dense(self, m: np.ndarray, t0: np.ndarray, prec: int = PREC_FP64) -> np.ndarray:
        """tau00 = [m^-1 [t0; 0]]_00 for a KKR matrix m (numpy [row, col], central block first)."""
        m = np.asarray(m, np.complex128)
        n = m.shape[0]
        b = t0.shape[0]
        mf = np.asfortranarray(m)
        t0f = np.asfortranarray(np.asarray(t0, np.complex128))
        out = np.zeros((b, b), np.complex128, order="F")
        self._check(self.lib.b200tau_solve_dense(self.ctx, mf.ctypes.data_as(ctypes.c_void_p), n, n,
                                                 t0f.ctypes.data_as(ctypes.c_void_p), b, prec,
                                                 out.ctypes.data_as(ctypes.c_void_p)))
        return np.array(out)

    def solve_vjp(self, jobs, taubar: np.ndarray, num_liz, want_logdet: bool = True):
        """Adjoint of each job's raw tau00 (b200tau_solve_vjp).

        taubar: (njobs, b, b) cotangents ([row, col]).  num_liz: LIZ size of each job's atom.
        Returns (tau00 (njobs, b, b), tbar, dlogdet) with tbar / dlogdet a list per job of
        (L, b, b) arrays [site, row, col] in the store layout (holomorphic: no conjugation)."""
        n = len(jobs)
        b = self.kkrsz_ns
        tb = np.ascontiguousarray(np.asarray(taubar, np.complex128).reshape(n, b, b).transpose(0, 2, 1))
        tau = np.zeros((n, b, b), np.complex128)
        nblk = int(np.sum(num_liz))
        g = np.zeros((nblk, b, b), np.complex128)
        d = np.zeros((nblk, b, b), np.complex128) if want_logdet else None
        self._check(self.lib.b200tau_solve_vjp(self.ctx, ctypes.cast(jobs, ctypes.c_void_p), n, _ptr(tb),
                                               _ptr(tau), _ptr(g), None if d is None else _ptr(d)))
        offs = np.concatenate([[0], np.cumsum(num_liz)]).astype(int)
        # stored column-major: [blk, col, row] -> [blk, row, col]
        tau = tau.transpose(0, 2, 1)
        gl = [g[offs[k]:offs[k + 1]].transpose(0, 2, 1).copy() for k in range(n)]
        dl = None if d is None else [d[offs[k]:offs[k + 1]].transpose(0, 2, 1).copy() for k in range(n)]
        return tau.copy(), gl, dl

    def solve_tau_full(self, atom: int, iie: int, ispin: int, energy: complex, n: int) -> np.ndarray:
        """Full tau = M^-1 T (numpy [row, col], reference site order): solveTauFullzgetrf's
        contract (linearSolvers_CPU.cpp:125-144), as the Kubo current matrix uses it."""
        jobs = make_jobs([(atom, iie, ispin, energy)])
        out = np.zeros((n * n,), np.complex128)
        self._check(self.lib.b200tau_solve_tau_full(self.ctx, ctypes.cast(jobs, ctypes.c_void_p), _ptr(out), n))
        return out.reshape(n, n).T.copy()

    def build_kkr(self, atom: int, iie: int, ispin: int, energy: complex, n: int) -> np.ndarray:
        """The device-built KKR matrix in the reference's site order (numpy [row, col])."""
        jobs = make_jobs([(atom, iie, ispin, energy)])
        out = np.zeros((n * n,), np.complex128)
        self._check(self.lib.b200tau_build_kkr(self.ctx, ctypes.cast(jobs, ctypes.c_void_p), _ptr(out), n))
        return out.reshape(n, n).T.copy()
