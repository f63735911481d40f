/*
 * b200tau: B200-native (sm_100a) multiple-scattering tau00 solve for LSMS.
 *
 * C ABI of the drop-in for LSMS's per-atom, per-energy solve
 *   M = 1 - t G0 over the local interaction zone (LIZ),
 *   tau00 = [M^-1]_00 t_0  (central kkrsz_ns x kkrsz_ns block),
 * returned as the reference returns it in tau00_l: (tau00 - t_0), rotated into
 * the local spin frame when n_spin_cant == 2.
 *
 * Reference interfaces replaced (paths inside mstsuite/lsms):
 *   calculateTauMatrix      src/MultipleScattering/calculateTauMatrix.cpp:320-837
 *   calculateAllTauMatrices src/MultipleScattering/calculateTauMatrix.cpp:841-945
 *   buildKKRMatrix*         src/MultipleScattering/buildKKRMatrix_CPU.cpp:621-646,
 *                           src/MultipleScattering/buildKKRMatrix_CUDA.cu:958-991
 *   solveTau00*             src/MultipleScattering/linearSolvers_CPU.cpp:76-331,
 *                           src/MultipleScattering/linearSolvers_CUDA.cu:182-469
 *   DeviceStorage / DeviceAtom uploads
 *                           src/Accelerator/DeviceStorage.cu:284-303,341-404
 *
 * Conventions
 *   - Complex numbers are interleaved (re, im) doubles, layout-compatible with
 *     std::complex<double>.  Matrices are column-major like Matrix<Complex>.
 *   - Every function returns B200TAU_OK (0) or an error code; the message of
 *     the last failure of a context is b200tau_last_error(ctx).  Nothing calls
 *     exit() or abort().
 *   - Host pointers passed in are read during the call only; nothing retains
 *     them after it returns.
 *   - One context per host thread (a context owns one CUDA stream); calls on
 *     one context are serialised by the caller.
 */
#ifndef B200TAU_H
#define B200TAU_H

#ifdef __cplusplus
extern "C" {
#endif

#define B200TAU_OK 0
#define B200TAU_ERR_ARG 1       /* bad argument (size, index, NULL pointer) */
#define B200TAU_ERR_CUDA 2      /* CUDA runtime error */
#define B200TAU_ERR_OOM 3       /* device allocation failed */
#define B200TAU_ERR_SINGULAR 4  /* zero pivot in a diagonal block or in 1 - Delta */
#define B200TAU_ERR_TIMEOUT 5   /* a device-side wait exceeded its bound */
#define B200TAU_ERR_STATE 6     /* call order (e.g. solve before upload) */

#define B200TAU_PREC_FP64 0  /* all arithmetic in FP64 */
#define B200TAU_PREC_MIXED 1 /* FP32/TF32 trailing updates + FP64 refinement */

#define B200TAU_ENGINE_TENSOR 0 /* mixed path: tcgen05 TF32 hi/lo trailing update (default) */
#define B200TAU_ENGINE_SIMT 1   /* mixed path: FP32 CUDA-core trailing update (cross-check) */

#define B200TAU_SWEEP_FP64 0 /* mixed path: correction solve in FP64 arithmetic on FP32 factors */
#define B200TAU_SWEEP_FP32 1 /* mixed path: correction solve in FP32, as zcgesv (default) */

#define B200TAU_PIVOT_AUTO 0  /* PANEL for MIXED factors from N = 3000 up, else BLOCK (default) */
#define B200TAU_PIVOT_BLOCK 1 /* pivots inside each 64 x 64 diagonal block */
#define B200TAU_PIVOT_PANEL 2 /* pivots from the whole remaining column of each 64-column panel */

typedef struct b200tau_ctx b200tau_ctx;

/* One solve: what calculateTauMatrix receives besides the shared state
 * (calculateTauMatrix.cpp:320-323: localAtomIndex, ispin, energy, prel, iie). */
typedef struct b200tau_job {
  int atom;         /* index previously given to b200tau_set_atom */
  int iie;          /* energy index inside the uploaded tmatStore group */
  int ispin;        /* spin channel (collinear spin-polarised: 0 or 1) */
  int reserved;     /* must be 0 */
  double energy[2]; /* complex energy, Ry */
  double prel[2];   /* sqrt(E (1 + E c2inv)), calculateTauMatrix.cpp:846 */
} b200tau_job;

/* Create a context on CUDA device `device` for maxlmax `lmax` (<= 3 supported
 * in this build), n_spin_cant in {1,2}, n_spin_pola in {1,2}
 * (LSMSSystemParameters fields, SystemParameters.hpp:126,76-77).  Builds the
 * Gaunt / i^l / Legendre tables (Coeficients.hpp:21-107) on the device. */
int b200tau_create(b200tau_ctx **ctx, int device, int lmax, int n_spin_cant,
                   int n_spin_pola);
void b200tau_destroy(b200tau_ctx *ctx);
const char *b200tau_last_error(const b200tau_ctx *ctx);

/* The context's CUDA stream (cudaStream_t) for callers that order their own
 * work against device-resident solves. */
void *b200tau_stream(b200tau_ctx *ctx);

/* Upload LocalTypeInfo::tmatStore (SystemParameters.hpp:260-262): column-major
 * (ld x nstore) complex, ld = blk_size * group_size, blk_size =
 * (2 (lmax+1)^2)^2 (buildLIZandCommLists.cpp:552-555).  Replaces
 * DeviceStorage::copyTmatStoreToDevice (DeviceStorage.cu:284-303). */
int b200tau_upload_tmat(b200tau_ctx *ctx, const double *tmat_store, long ld,
                        int nstore, int blk_size);

/* Register atom `atom`'s LIZ (AtomData fields, AtomData.hpp:440-445,466):
 * liz_pos 3 x num_liz column-major (LIZPos), liz_lmax and liz_store_idx
 * (LIZlmax, LIZStoreIdx), and the spin frame ubr/ubrd (4 complex each, may
 * be NULL when n_spin_cant == 1).  Replaces DeviceAtom::copyFromAtom
 * (DeviceStorage.cu:341-404). */
int b200tau_set_atom(b200tau_ctx *ctx, int atom, int num_liz,
                     const double *liz_pos, const int *liz_lmax,
                     const int *liz_store_idx, const double *ubr,
                     const double *ubrd);

/* Iterative-refinement steps for a precision (0..16).  Each step computes the FP64 residual
 * R = [0; t0] - M X against the unmodified KKR matrix and applies the correction from the
 * stored block factors (the refinement of the reference's zcgesv / cusolverDnIRSXgesv
 * solvers, linearSolvers_CPU.cpp:148-174, linearSolvers_CUDA.cu:424-469, on the N x b
 * system).  Defaults: FP64 1 step, MIXED 10 steps, of which each job runs only as many as it
 * needs: after every step, a job whose estimated remaining error (the relative size c of the
 * correction just applied times its contraction c / c_previous) is below 1e-12 of tau00 stops.
 * A MIXED job whose corrections stop shrinking, or that has not converged after the last step,
 * is re-solved by FP64 block LU (b200tau_last_fallback_count).  FP64 with 0 steps takes tau00
 * directly from the Schur complement like zblock_lu. */
int b200tau_set_refinement(b200tau_ctx *ctx, int prec, int steps);

/* Engine of the mixed path's trailing update (B200TAU_ENGINE_*). */
int b200tau_set_mixed_engine(b200tau_ctx *ctx, int engine);

/* Arithmetic of the mixed path's correction solve Y = F^-1 R between FP64 residuals
 * (B200TAU_SWEEP_*).  The residual R = B - M X and the update X += Y are FP64 either way. */
int b200tau_set_mixed_sweep(b200tau_ctx *ctx, int sweep);

/* Solve `njobs` (atom, energy, spin) problems in one batched device pass and
 * write each job's tau00_l (kkrsz_ns^2 complex, the layout calculateTauMatrix
 * writes through its tau00_l argument) to host memory at
 * tau00_l + 2 * kkrsz_ns^2 * j.  `prec` is B200TAU_PREC_*. */
int b200tau_solve(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs,
                  int prec, double *tau00_l);

/* As b200tau_solve, but tau00_l_dev is device memory and the call returns
 * once the work is enqueued on the context's stream (inputs already resident
 * from upload_tmat / set_atom).  The call does not wait for the device, not
 * between waves and not for the FP64 re-solve of unconverged MIXED jobs, so
 * several calls can be queued ahead.  It waits only when a call first needs (or
 * outgrows) a workspace buffer, which it then allocates.  Errors detected on
 * the device (a singular pivot of any job of the last call, a bounded wait that
 * ran out) are reported by the next b200tau_sync. */
int b200tau_solve_device(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs,
                         int prec, double *tau00_l_dev);
int b200tau_sync(b200tau_ctx *ctx);

/* Solver-only entry, the contract of solveTau00zblocklu_cpp / solveTau00zgesv
 * (linearSolvers_CPU.cpp:76-96,261-331): given a host KKR matrix m (n x n,
 * column-major, leading dimension ldm, central site first) and the central
 * t-matrix t0 (b x b), write tau00 = [m^-1 [t0; 0]]_00 (b x b, NOT minus t0,
 * unrotated) to host memory. */
int b200tau_solve_dense(b200tau_ctx *ctx, const double *m, int n, int ldm,
                        const double *t0, int b, int prec, double *tau00);

/* Allocation-free variant of b200tau_solve_dense, for callers that cannot call cudaMalloc:
 * programs whose GPU memory is owned by another allocator (memory reserved up front for an
 * application pool, where an allocation inside this library would fail or fragment it) and
 * latency-critical paths that cannot accept cudaMalloc/cudaFree's implicit synchronisation.
 * No counterpart in the reference.
 *   m (n x n, leading dimension ldm, central site first), t0 (b x b) and tau00 (b x b output,
 *   raw tau00 as b200tau_solve_dense) are DEVICE pointers owned by the caller; the FP64 path
 *   with one refinement step runs on `stream` (a cudaStream_t, NULL = default stream) and the
 *   call returns after synchronising that stream.
 *   No context, no cudaMalloc/cudaFree: all scratch lives in one fixed file-scope device array
 *   of about 8.9 MB that every GPU loading the library keeps until the process exits.
 *   Limits: n <= 512, b <= 32; larger sizes return B200TAU_ERR_ARG.
 *   The array's device address is looked up once per device by the first call on that device,
 *   so make that first call before any stream capture.  All calls share the array (the call
 *   clears what must start at zero); calls that overlap on the GPU race and must be serialised. */
int b200tau_solve_dense_noalloc(const double *m, int n, int ldm, const double *t0, int b,
                                double *tau00, void *stream);

/* Full tau = M^-1 T of one job, T = blockdiag(t_j) over every LIZ site j: the contract of the
 * reference's solveTauFullzgetrf (src/MultipleScattering/linearSolvers_CPU.cpp:125-144; cuSOLVER
 * variant linearSolvers_CUDA.cu:331-361), which the Kubo current matrix calls
 * (src/Kubo/CurrentMatrix.cpp:184-222).  tau_full is n x n complex, column-major, host memory, in
 * the reference's site order (central site first), n = n_spin_cant * nrmat of the job's atom.
 * FP64 block factors of M (pivoting as b200tau_set_pivoting), M^-1 formed from them on the device,
 * then each block column scaled by its site's t-matrix.  Two documented differences from the
 * reference, both invisible when every site has the same lmax and the tmatStore group holds one
 * energy (Kubo's use): t_j comes from the job's energy iie (the reference always reads the
 * group's first energy) and each site's block has the site's own size (the reference places
 * kkrsz_ns x kkrsz_ns blocks at multiples of kkrsz_ns). */
int b200tau_solve_tau_full(b200tau_ctx *ctx, const b200tau_job *job, double *tau_full, int n);

/* Build only: the KKR matrix M = 1 - t G for one job in the reference's site
 * order (central site first), written to host memory (n x n, ld = n) where
 * n = n_spin_cant * nrmat.  Parity hook for buildKKRMatrix*; not on the hot
 * path.  Returns B200TAU_ERR_ARG if m_out's n does not match. */
int b200tau_build_kkr(b200tau_ctx *ctx, const b200tau_job *job, double *m_out,
                      int n);

/* Keep the factors of a forward solve for the adjoint (1), or not (0, the default).  While on, a
 * PREC_FP64 b200tau_solve / b200tau_solve_device whose jobs fit one wave (and whose matrices are
 * eliminated with BLOCK pivoting) leaves its KKR matrices, FP64 block factors and refined
 * solutions in the workspace, and the next b200tau_solve_vjp on the same jobs in the same order
 * reuses them: no KKR build, no elimination, no refinement, only M^-1 from the kept factors and
 * the per-site contractions.  Any other call on the context (another solve, an upload, a dense,
 * full-tau or build call) drops them; so does the vjp that uses them.  The forward pass of an
 * LSMS energy point then pays one factorisation for tau00 and its derivatives.  No counterpart in
 * the reference. */
int b200tau_set_keep_factors(b200tau_ctx *ctx, int enable);

/* Reverse-mode derivatives, for each job, of tau00 and of ln det M with respect to the
 * t-matrix t_j of every LIZ site j, from the FP64 block factors of the job's own forward solve
 * (one factorisation; M^-1 is formed from the factors; with b200tau_set_keep_factors those of the
 * preceding forward solve of the same jobs).  No counterpart in the reference.
 *   taubar  (in)  b x b cotangent on the raw tau00 = [M^-1]_00 t_0 of each job (not minus t0,
 *                 unrotated), jobs one after another (2 b^2 doubles per job).
 *   tau00   (out) that tau00 per job, or NULL.
 *   tbar    (out) sum_ab taubar_ab d tau00_ab / d (t_j)_xy as a b x b block per LIZ site
 *                 (holomorphic convention: no conjugation);
 *   dlogdet (out) d ln det M / d (t_j)_xy per LIZ site, same layout, or NULL.
 * Gradient blocks are column-major b x b in the t-matrix store layout (row s kkrsz + lm; zero
 * for lm >= (lmax_j + 1)^2), in LIZ order (site 0 first); job k's blocks start at block
 * sum_{i<k} num_liz(atom of job i).  A caller wanting the torch/JAX convention for a real loss
 * conjugates: grad_t = conj(tbar(conj(grad_tau))). */
int b200tau_solve_vjp(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs,
                      const double *taubar, double *tau00, double *tbar,
                      double *dlogdet);

/* The Gaunt numbers this library builds its G0 tables from (host-only, no GPU needed):
 * cgnt[l3/2 + (lmax+1) * (j1 + kk * j2)], kk = (lmax+1)^2, the layout of the reference's
 * GauntCoeficients::cgnt (Coeficients.hpp:37-92, cgaunt_c.f90:31).  cgnt must hold
 * (lmax+1) * kk * kk doubles; entries outside the l3 range are 0. */
int b200tau_gaunt_numbers(int lmax, double *cgnt);

/* Kernel-time accounting of the dominant kernel (the trailing-update launches of the block
 * elimination).  While enabled, each such launch is bracketed by CUDA events on the context
 * stream; b200tau_profile_read returns the summed device time (ms), the number of timed
 * launches and their algorithmic FLOPs (8 (N-k-kb)^2 kb per job and step) since enabling.
 * Enabling resets the totals. */
int b200tau_set_profiling(b200tau_ctx *ctx, int enable);
int b200tau_profile_read(b200tau_ctx *ctx, double *ms, long *launches, double *flops);
/* Device time per phase of the solves since profiling was enabled, from CUDA events on the
 * context stream: ms3[0] KKR build, ms3[1] block elimination, ms3[2] refinement and tau00_l. */
int b200tau_profile_phases(b200tau_ctx *ctx, double *ms3);

/* Number of kernel launches the last solve issued (for launch accounting). */
long b200tau_last_launch_count(const b200tau_ctx *ctx);

/* Number of jobs of the last solve whose mixed-precision refinement did not converge (the FP32
 * factors cannot refine a condition number much beyond ~1e5) and that were re-solved by FP64
 * block LU of their KKR matrix instead. */
long b200tau_last_fallback_count(const b200tau_ctx *ctx);

/* Turn that FP64 re-solve off (0) or on (1, the default).  Off, an unconverged MIXED job
 * returns its last refinement iterate. */
int b200tau_set_mixed_fallback(b200tau_ctx *ctx, int enable);

/* Run each wave of b200tau_solve / b200tau_solve_device as one CUDA graph (1, the default) or as
 * separate kernel launches (0).  A wave's pipeline (KKR build, block elimination, refinement,
 * tau00_l) is captured on first use of its shape (job count, sizes, buffers) and replayed for every
 * later wave of that shape, so a call costs the host a few copies and one or two graph launches.
 * Profiling (b200tau_set_profiling) times the separate launches instead.  No counterpart in the
 * reference. */
int b200tau_set_graphs(b200tau_ctx *ctx, int enable);

/* Paired elimination steps (MIXED, either pivoting): while the trailing block after the second
 * of two 64-column steps has at least min_rest columns, both steps' updates of it are applied in
 * one tensor-core pass (K = 128 complex), so its FP32 read-modify-write, which bounds the update,
 * happens once per two steps; the strips the second step needs first are updated separately.
 * The factors, and so the refinement and tau00, are those of single steps.  min_rest = 0 turns
 * it off; default 768.  No counterpart in the reference. */
int b200tau_set_paired_steps(b200tau_ctx *ctx, int min_rest);

/* Autotuner of that threshold for a workload: solves `jobs` (MIXED) with each candidate min_rest
 * (NULL candidates: 0, 512, 768, 1024, 1280, 1536; at most 16), one untimed solve and then `reps`
 * timed ones (1..16) per candidate, each timed on the context's stream from the first launch to
 * the last of the call, and keeps the candidate with the fastest of its timed solves for the jobs'
 * size bucket (their largest N rounded up to 64): later waves whose largest N falls in that bucket
 * use it, other sizes keep b200tau_set_paired_steps' value (which also clears every tuned bucket).
 * The threshold in force for the bucket before the call stays unless a candidate is at least 2%
 * faster than it.  The choice goes to *chosen (if non-NULL) and the per-candidate ms (fastest
 * timed solve) to ms_out[ncand] (if non-NULL).  Outputs of the solves are discarded.  On an error
 * nothing is recorded.  No counterpart in the reference, whose tuning knob is the block size of
 * its block LU (zblockLUSize, calculateTauMatrix.cpp:726-736). */
int b200tau_autotune_paired_steps(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs,
                                  const int *candidates, int ncand, int reps, int *chosen,
                                  float *ms_out);

/* Row pivoting of the block elimination (B200TAU_PIVOT_*), both precisions.  BLOCK pivots inside
 * each 64 x 64 diagonal block, as the reference's GPU solver inverts its diagonal blocks
 * (zblock_lu_cuda_c.cu:218-259).  PANEL picks each 64-column step's rows from the whole
 * remaining column: the diagonal block's own rows and the rows of largest magnitude in the panel
 * (256 candidates) go through a partial-pivoting elimination, whose pivot rows then move into
 * place in every column.  That approaches LAPACK's zgetrf over the column (the reference's CPU
 * path pivots with zgetrf inside blocks of ~N/3 rows, zblock_lu_cpp.cpp:58,
 * linearSolvers_CPU.cpp:270), at the cost of the selection and the row moves; ill-conditioned
 * matrices need it for the MIXED refinement to converge.  Pivots never come from the central site's rows, so FP64 with 0
 * refinement steps still reads tau00 from the Schur complement.  b200tau_solve_vjp always
 * uses BLOCK. */
int b200tau_set_pivoting(b200tau_ctx *ctx, int mode);

/* Bound, in polls, of the first wait of every KKR-build CTA on the copy of the angular tables
 * into its shared memory (default 1 << 24; 0 makes that wait give up at once).  A CTA whose wait
 * runs out records it, still waits (with a far longer bound) for its copy to land before it
 * exits, and leaves its block column of M unbuilt; the call then returns B200TAU_ERR_TIMEOUT
 * (outputs are written but meaningless).  It exists to exercise that reporting: every bounded
 * device wait of the library reports the same way.  No counterpart in the reference, which has
 * no bounded waits (it aborts, src/Accelerator/zblock_lu_cuda_c.cu:30-52). */
int b200tau_set_build_wait(b200tau_ctx *ctx, long polls);

#ifdef __cplusplus
}
#endif

#endif /* B200TAU_H */
