// Internal declarations shared by the b200tau CUDA sources.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace b200 {

constexpr int kMaxLmax = 3;                                     // maxlmax supported
constexpr int kMaxKK = (kMaxLmax + 1) * (kMaxLmax + 1);          // 16
constexpr int kMaxB = 2 * kMaxKK;                                // kkrsz_ns <= 32
constexpr int kMaxLend = 2 * kMaxLmax;                          // 6
constexpr int kNdlm = (kMaxLend + 1) * (kMaxLend + 2) / 2;       // 28 P_lm values
constexpr int kNdlj = (kMaxLend + 1) * (kMaxLend + 1);           // 49 D_lm values
constexpr int kMaxTerms = kMaxLmax + 1;                          // Gaunt terms per G element
constexpr int kNb = 64;                                         // elimination block width
// Panel pivoting (pivot.cu): candidate rows of a step's partial-pivoting elimination.
constexpr int kPivCands = 256;
// Per-job pivot buffer of panel pivoting (ints), for leading dimension ld:
//   [0, ld)                  perm: the original row at each physical row position
//   [ld, 2 ld)               rowpos: the physical position of each original row (after elimination)
//   [2 ld, 2 ld + 1 + 4 kNb) the step's row moves: count, kNb*2 destinations, kNb*2 sources
//   [.., + ld)               the step's row magnitudes over the panel columns (float bits)
__host__ __device__ constexpr int pivot_moves_offset(int ld) { return 2 * ld; }
__host__ __device__ constexpr int pivot_mags_offset(int ld) { return 2 * ld + 1 + 4 * kNb; }
__host__ __device__ constexpr int pivot_ints(int ld) { return pivot_mags_offset(ld) + ld; }
// Columns of one tile of the tensor-core trailing update (tc_update.cu).
constexpr int kTcTileCols = 256;
// A refining job stops once its estimated remaining error on tau00 is below this fraction of
// max|tau00|: 100x below the mixed path's 1e-10 accuracy target.
constexpr double kRefineTol = 1e-12;
// JobDev::conv values (0: still refining)
constexpr int kConverged = 1;
constexpr int kDiverged = 2;  // the corrections stopped shrinking (numerical)
constexpr int kAborted = 3;   // a bounded wait of a dataflow sweep ran out on this job
// Bits of the context's device error word: a bounded wait ran out in the KKR build's table copy,
// in the tensor-core trailing update, or in a dataflow sweep of the refinement.
constexpr int kErrBuildWait = 1;
constexpr int kErrUpdateWait = 2;
constexpr int kErrSweepWait = 8;
// Polls of a bounded wait: the default bound of the first wait on the KKR build's table copy, and
// the far longer bound of a wait that only drains copies or tensor-core work still in flight
// after an earlier wait gave up (a CTA never exits with such work outstanding).
constexpr long kTablePolls = 1L << 24;
constexpr long kDrainPolls = 1L << 26;

// Angular-momentum tables for G_ij (makegij_c.f:79-128, buildKKRMatrix_CPU.cpp:144-176),
// laid out as a gather list: G(lm2, lm1) = pi4 * i^rot * sum_q coef[q] * D[didx[q]]
// with the terms in the reference's summation order (l3 descending).
// Staged into shared memory with one bulk (TMA) copy, so the size is a multiple of 16.
struct alignas(16) AngularTables {
  double coef[kMaxKK * kMaxKK * kMaxTerms];  // Gaunt numbers cgnt(l3/2, lm1, lm2)
  int didx[kMaxKK * kMaxKK * kMaxTerms];     // index l3 (l3+1) + m2 - m1 into D
  int nterm[kMaxKK * kMaxKK];                // number of l3 terms
  int rot[kMaxKK * kMaxKK];                  // illp(lm2, lm1) = i^rot
  double ilp1_re[kMaxLend + 2];              // i^(l+1)
  double ilp1_im[kMaxLend + 2];
  double plm_mm[kMaxLend + 2];               // sqrt((2m+1)/(2m))
  double plm_m1[kMaxLend + 2];               // sqrt(2m+1)
  double plm_a[kNdlm + 4];                   // a_lm (index l(l+1)/2+m)
  double plm_b[kNdlm + 4];                   // b_lm
  double pi4;
  int lmax;
  int pad_[1];
};
static_assert(sizeof(AngularTables) % 16 == 0, "bulk-copy size must be a multiple of 16");

// Host-side table construction (angular.cpp).  Returns 0 on success.
int build_angular_tables(int lmax, AngularTables *out);
// Gaunt numbers cgnt[l3/2 + (lmax+1)*(j1 + kk*j2)], exposed for tests.
void gaunt_numbers(int lmax, double *cgnt);

// One solve as the device sees it.  Matrices are column-major complex.
// Site order inside M: LIZ sites 1..L-1 first, the central site 0 last, so that
// eliminating the first n = N - b columns leaves the Schur complement
// S = M00 - M0r Mrr^-1 Mr0 = 1 - Delta in the trailing b x b block.
//
// M  : the KKR matrix in FP64, kept unmodified when refinement is on (residuals).
// F  : the factor storage (FP64 `double2` or FP32 `float2`, see the launcher's type); the block
//      elimination runs in place on F.  F may alias M (FP64, no refinement).
// X  : N x b solution (FP64), R : N x b residual, Y : N x b correction (FP64), ld = ld.
struct JobDev {
  double2 energy;
  double2 prel;
  const double *pos;     // 3 x L (device)
  const int *lmax;       // L
  const int *store;      // L (tmatStore column per site)
  const int *perm;       // L: perm[p] = LIZ site at position p (site 0 last)
  const int *off;        // L+1: row/column offset of position p
  double2 *M;
  void *F;
  double2 *X;
  double2 *R;
  double2 *Y;
  const double2 *t0;     // central t-matrix (b x b, ld t0_ld)
  double2 *out;          // b*b complex result
  int *conv;             // refinement converged flag (set on the device, skips later rounds)
  double *cnorm;         // relative size of the previous refinement correction (0 before round 1)
  double2 ubr[4];
  double2 ubrd[4];
  int L, N, n, b;
  int ld;
  int iie, ispin;
  int t0_ld;
  int out_mode;          // 0: tau00_l (tau00 - t0, rotated); 1: raw tau00
  int inactive;          // 1: every kernel skips this record (a converged job in the FP64 re-solve)
  int slot;              // workspace slot of F (the z coordinate of the factor tensor maps)
  int pad_[1];
  // adjoint (b200tau_solve_vjp) only
  double2 *V;            // N x N workspace for M^-1 (ld)
  const double2 *taubar; // b x b cotangent on tau00
  double2 *tbar;         // L blocks of b x b, LIZ site order: d<taubar, tau00>/d t_site
  double2 *dlogdet;      // L blocks of b x b: d ln det M / d t_site (may be null)
  int *err;              // the context's device error word (kErr* bits), or null
  int *piv;              // panel pivoting's buffer (pivot_ints(ld) ints), null: pivots inside the
                         // 64 x 64 diagonal blocks only
};

struct BuildParams {
  const AngularTables *tables;  // device
  const double2 *tmat;          // device tmatStore, column-major (tmat_ld x nstore)
  long tmat_ld;
  int blk;                      // blkSizeTmatStore
  int kkrsz;                    // (maxlmax+1)^2
  int ns;                       // n_spin_cant
  int npola;                    // n_spin_pola
  int f_kind;                   // 0: no F copy (F aliases M), 1: FP64 copy, 2: FP32 copy
  const unsigned char *tdiag;   // [(store * group + iie) * 2 + ispin]: t block exactly diagonal
  int group;                    // energies in the uploaded tmatStore group
  int g_mode;                   // 1: write the structure constants G (no t factor, zero diagonal
                                // blocks) into M instead of M = 1 - t G (adjoint)
  long table_polls;             // bound of the first wait on the table copy (kTablePolls)
};

enum FactorKind { kFactorFP64 = 0, kFactorFP32 = 1 };

// Optional CUDA-event bracketing of the trailing-update launches (the dominant kernel), on the
// launching stream.  `ev` holds `cap` events; pairs (start, stop) are recorded from `used`.
struct KernelTimer {
  cudaEvent_t *ev = nullptr;
  int cap = 0;
  int used = 0;
};

// Operand packs and TMA descriptors of the tensor-core trailing update (tc_update.cu).
// Per wave slot: A pack 2 ld rows x kTcKMax floats (hi and lo), B pack ld rows x kTcKMax floats.
struct TcMaps {
  CUtensorMap tA_hi, tA_lo, tB_hi, tB_lo;
  CUtensorMap tB2_hi, tB2_lo;  // the B packs in 128-column boxes: one CTA's half of a pair tile
  CUtensorMap tF;   // the wave's FP32 factor slots as floats {2 ld, ld, slots}, box {128, kTcPieceCols, 1}
  CUtensorMap tFw;  // the same slots, box {32, kTcPieceCols, 1}: one epilogue warp's rows of a piece
  CUtensorMap tFu;  // the same slots, box {32, 32, 1}, MN-major TF32 swizzle: a quarter of a sweep unit
  float *a_hi = nullptr, *a_lo = nullptr, *b_hi = nullptr, *b_lo = nullptr;
  size_t a_slot = 0, b_slot = 0;  // floats per slot
  int *counters = nullptr;        // tile counters of the pair update, kTcCountersPerStep per step
  int counter_slots = 0;
};
constexpr int kTcCountersPerStep = 8;
// K floats per TMA box of the operand packs (128-byte rows, 128-byte swizzle)
constexpr int kTcChunk = 32;
// floats per operand-pack row: the real K of up to two 64-column elimination steps, whose updates
// of the trailing block the tensor-core kernels can apply in one pass
constexpr int kTcKMax = 4 * kNb;
// columns of F per TMA reduce-add of the update's epilogue
constexpr int kTcPieceCols = 32;
size_t tc_smem_bytes();
int tc_num_sms();
cudaError_t tc_prepare();
// Pack + tensor-core update A22 -= A21 W for step k of every job in the wave (FP32 factors).
cudaError_t launch_tc_step(const TcMaps &maps, const JobDev *jobs, int njobs, int k, int max_N, int *err,
                           cudaStream_t s);
// The operand packs of an update of the trailing block of step k_last by the steps kA, kA + 64,
// ... (nblk of them, k_last the last): A = the columns of those steps below row k_last + kb,
// B (if pack_b) = their rows right of column k_last + kb.  nblk = 1 is a single step (kA = k_last).
// The two halves: the hi/lo operand packs of step k (A21, and W unless the W = D A12 tiles wrote
// theirs), and the update of the tiles of `part` (0 all, 1 the first 256 rows of the first tile
// column, which hold the next diagonal block, 2 the others; 3 the first tile column, which holds
// the next step's whole panel, 4 the other tile columns) on at most max_grid SMs (0: all).
// Parts 0, 2 and 4 run on CTA pairs and take their tiles from maps.counters, which the
// elimination zeroes before its first step (launch_tc_counters_reset).
cudaError_t launch_tc_pack(const TcMaps &maps, const JobDev *jobs, int njobs, int kA, int nblk, int k_last,
                           int max_N, cudaStream_t s, bool pack_b);
// The update of the trailing block of step k by the last nblk steps (their packs from
// launch_tc_pack and the W = D A12 tiles), restricted to the tiles of `part`.
cudaError_t launch_tc_update(const TcMaps &maps, const JobDev *jobs, int njobs, int k, int max_N, int *err,
                             cudaStream_t s, int part, int max_grid, int nblk = 1);
cudaError_t launch_tc_counters_reset(const TcMaps &maps, cudaStream_t s);
// A second stream and two events for the elimination's look-ahead (all null: none).
struct Lookahead {
  cudaStream_t s2 = nullptr;
  cudaEvent_t panel = nullptr, diag = nullptr;
  // Paired steps (FP32 factors, either pivoting): while the trailing block after the second of
  // two steps has at least pair_min_rest columns, the two steps' updates of it are applied in one
  // tensor-core pass of K = 128 complex (0: never).  min_n: the smallest n of the wave's jobs
  // (every job must have both steps).
  int pair_min_rest = 0;
  int min_n = 0;
};
// default pair_min_rest: paired steps pay for their strip updates once the trailing block's
// read-modify-write they save is larger (on the 31-point N = 2160 contour 768 measured best of
// 0, 768, 1024 and 1400)
constexpr int kPairMinRest = 768;

// cudaFuncSetAttribute(fn, MaxDynamicSharedMemorySize, bytes) on the current device, skipped when
// an earlier call on this device already allowed at least `bytes` (a per-launch host call costs
// more than the launch itself).
cudaError_t ensure_smem_attr(const void *fn, int bytes);
template <typename K>
inline cudaError_t ensure_smem(K *kernel, int bytes) {
  return ensure_smem_attr(reinterpret_cast<const void *>(kernel), bytes);
}

// Launchers (return cudaGetLastError of the launches).  `launches` accumulates the number of
// kernels enqueued.
cudaError_t launch_kkr_build(const JobDev *jobs, int njobs, int max_L, const BuildParams &p,
                             int *err_flags, cudaStream_t s, long *launches);
// flags[(store * group + iie) * 2 + ispin] = 1 when that b x b t block of the device tmatStore
// (column-major, leading dimension ld per store column) has no non-zero off-diagonal element;
// spin 1 is written as 0 unless the store is collinear spin-polarised (`colpol`).
cudaError_t launch_tdiag_flags(const double2 *tmat, long ld, int nstore, int group, int b, int kkrsz, bool colpol,
                               unsigned char *flags, cudaStream_t s);
// Block elimination of F over the first n columns (all jobs of the wave).
// With FP32 factors and `tc` non-null the trailing update runs on the tensor cores (tc_update.cu).
// `sparse_jobs`: most records are inactive (the FP64 re-solve), so the trailing update runs on a
// small looping grid instead of one CTA per tile.  `panel`: the records carry pivot buffers and
// every step picks its rows by panel pivoting (pivot.cu).
cudaError_t launch_eliminate(FactorKind fk, const JobDev *jobs, int njobs, int max_n, int max_N,
                             int *info, cudaStream_t s, long *launches, KernelTimer *timer,
                             const TcMaps *tc, int *err, bool sparse_jobs = false,
                             const Lookahead *la = nullptr, bool panel = false);
// Panel pivoting (pivot.cu), for the records with a pivot buffer: the identity permutation; the
// selection that picks step k's kb rows from [k, n) and writes the step's row moves; those moves
// applied to columns [c0, c1) of F; and the final row positions for the residual.
cudaError_t launch_pivot_init(const JobDev *jobs, int njobs, cudaStream_t s, long *launches);
cudaError_t launch_panel_select(FactorKind fk, const JobDev *jobs, int njobs, int k, int max_n, cudaStream_t s,
                                long *launches);
cudaError_t launch_row_moves(FactorKind fk, const JobDev *jobs, int njobs, int k, int c0, int c1, int max_N,
                             cudaStream_t s, long *launches);
cudaError_t launch_pivot_finish(const JobDev *jobs, int njobs, cudaStream_t s, long *launches);
// F = M (n x n, leading dimension ld) converted to the factor type.
cudaError_t launch_copy_to_factor(FactorKind fk, const double2 *M, void *F, int n, int ld, cudaStream_t s);
// FP64 re-solve of the mixed jobs whose refinement did not converge, on the device: out[w] is
// jobs[w] with F at f64 + w * f64_stride (an FP64 copy of M is made there) and no converged flag,
// or an inactive record when jobs[w] converged; `count` accumulates the re-solved jobs.  Without
// `panel` the records lose their pivot buffer (the re-solve pivots inside the diagonal blocks).
cudaError_t launch_fallback_prepare(const JobDev *jobs, JobDev *out, int njobs, double2 *f64, size_t f64_stride,
                                    int max_N, int *count, bool panel, cudaStream_t s, long *launches);
// tau00 from the Schur block directly (no refinement): out = S^-1 t0 (- t0, rotated).
cudaError_t launch_finalize_direct(FactorKind fk, const JobDev *jobs, int njobs, int ns, int kkrsz,
                                   int *info, cudaStream_t s, long *launches);
// Iterative refinement of X for M X = [0; t0]: initial solve from the factors, then `steps`
// rounds of R = B - M X (FP64), Y = F^-1 R, X += Y; then out from X[n:N].
// `fp32_sweep` (FP32 factors only) runs the correction solve in FP32 arithmetic, as LAPACK's
// zcgesv does; the residual and X += Y stay FP64.
cudaError_t launch_solve_refine(FactorKind fk, const JobDev *jobs, int njobs, int max_n, int max_N,
                                int b, int steps, int ns, int kkrsz, int *info, cudaStream_t s,
                                long *launches, bool fp32_sweep = false, const CUtensorMap *fmap = nullptr);
// The same in pieces, for a driver that drops converged jobs between rounds: the initial solve
// X = F^-1 [0; t0], one refinement round (with the convergence check when `check`), and tau00_l.
cudaError_t launch_refine_begin(FactorKind fk, const JobDev *jobs, int njobs, int max_n, int max_N, int b,
                                int *info, cudaStream_t s, long *launches, bool fp32_sweep = false,
                                const CUtensorMap *fmap = nullptr);
// `active_hint` (> 0): about how many of the jobs are still refining, which sizes the dataflow
// sweeps' clusters; the launches still cover all njobs, so any value is correct.  `active`
// (njobs + 1 ints of device scratch, optional): the residual first lists the jobs still refining
// there and spreads its CTAs over them alone.
cudaError_t launch_refine_round(FactorKind fk, const JobDev *jobs, int njobs, int max_n, int max_N, int b,
                                bool check, int *info, cudaStream_t s, long *launches, bool fp32_sweep = false,
                                const CUtensorMap *fmap = nullptr, int active_hint = 0, int *active = nullptr);
cudaError_t launch_refine_end(const JobDev *jobs, int njobs, int ns, int kkrsz, cudaStream_t s, long *launches);
// One block sweep of the correction solve for all jobs, one thread-block cluster per job
// (sweep.cu): forward (R -> Y over the D_k, A21_k factors) or backward (Y over the W_k factors,
// X (+)= Y).  `fp32_arith` selects FP32 arithmetic on FP32 factors.  max_N bounds the jobs' N.
cudaError_t launch_sweep(FactorKind fk, const JobDev *jobs, int njobs, int b, int max_N, bool forward, int mode,
                         bool fp32_arith, const CUtensorMap *fmap, cudaStream_t s, int active_hint = 0);
// The dataflow sweeps for FP32 factors in FP32 arithmetic with b <= 16 (sweep_flow.cu), operand
// units loaded through `fmap` (TcMaps::tFu over the jobs' factor slots).  Sets *launched when it
// took the launch; false (and cudaSuccess) without a map or when the shape does not fit its
// shared-memory layout, and the caller runs launch_sweep's step-synchronous kernels instead.
cudaError_t launch_flow_sweep(const JobDev *jobs, int njobs, int b, int max_N, bool forward, int mode,
                              const CUtensorMap *fmap, cudaStream_t s, bool *launched, int active_hint = 0);
// Graph node of the mixed path's FP64 re-solve gate: sets `h` to 1 when any of the njobs records
// has not converged (its conv word is not kConverged), else 0.
cudaError_t add_fallback_gate_node(cudaGraph_t g, cudaGraphNode_t *node, const JobDev *jobs, int njobs,
                                   cudaGraphConditionalHandle h);
// The device tmatStore as the kernels that read t blocks see it: the b x b block of (store,
// energy iie, spin) at tmat + store tmat_ld + iie blk + jsm(spin), leading dimension bstore.
struct TmatView {
  const double2 *tmat;
  long tmat_ld;
  int blk, kkrsz, ns, bstore;
  int colpol;  // collinear spin-polarised: spin 1's block follows spin 0's
  __host__ __device__ long jsm(int ispin) const { return colpol ? (long)kkrsz * kkrsz * ispin : 0; }
};
// Full tau = M^-1 T into M's storage (positions order), from V = M^-1 (or (P M)^-1 with panel
// pivoting) and the sites' t-matrices; the contract of the reference's solveTauFullzgetrf.
cudaError_t launch_tau_full(const JobDev *jobs, int njobs, int max_L, int max_N, const TmatView &tv, cudaStream_t s,
                            long *launches);
// Adjoint (adjoint.cu), FP64 factors: V = M^-1 from the block factors in F, then per LIZ site the
// tau00 cotangent pull-back and d ln det M / d t (needs G in M, X refined, V).
cudaError_t launch_inverse(const JobDev *jobs, int njobs, int max_n, int max_N, cudaStream_t s, long *launches);
cudaError_t launch_vjp_assemble(const JobDev *jobs, int njobs, int max_L, int kkrsz, int ns, cudaStream_t s,
                                long *launches);

}  // namespace b200
