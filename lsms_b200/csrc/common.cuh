// Internal declarations shared by the b200tau CUDA sources.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace b200 {

constexpr int kMaxLmax = 3;                                     // maxlmax supported
constexpr int kMaxKK = (kMaxLmax + 1) * (kMaxLmax + 1);          // 16
constexpr int kMaxB = 2 * kMaxKK;                                // kkrsz_ns <= 32
constexpr int kMaxLend = 2 * kMaxLmax;                          // 6
constexpr int kNdlm = (kMaxLend + 1) * (kMaxLend + 2) / 2;       // 28 P_lm values
constexpr int kNdlj = (kMaxLend + 1) * (kMaxLend + 1);           // 49 D_lm values
constexpr int kMaxTerms = kMaxLmax + 1;                          // Gaunt terms per G element

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
// Gaunt numbers cgnt[l3/2 + (lmax+1)*(j1 + kk*j2)] and the i-factors, exposed for tests.
void gaunt_numbers(int lmax, double *cgnt);

// One solve as the device sees it.  Matrices are column-major complex (double2).
// Site order inside M: LIZ sites 1..L-1 first, the central site 0 last, so that
// eliminating the first n = N - b columns leaves the Schur complement
// S = M00 - M0r Mrr^-1 Mr0 = 1 - Delta in the trailing b x b block.
struct JobDev {
  double2 energy;
  double2 prel;
  const double *pos;     // 3 x L (device)
  const int *lmax;       // L
  const int *store;      // L (tmatStore column per site)
  const int *perm;       // L: perm[p] = LIZ site at position p (site 0 last)
  const int *off;        // L+1: row/column offset of position p
  double2 *M;            // workspace, ld = ld
  const double2 *t0;     // central t-matrix (b x b, ld t0_ld) for the finalize step
  double2 *out;          // b*b complex result
  float2 *Mf;            // FP32 working copy (mixed precision), ld = ld
  double2 *X;            // N x b solution (mixed precision refinement), ld = ld
  double2 *R;            // N x b residual / correction (mixed precision), ld = ld
  double2 ubr[4];
  double2 ubrd[4];
  int L, N, n, b;
  int ld;
  int iie, ispin;
  int t0_ld;
  int out_mode;          // 0: tau00_l (tau00 - t0, rotated); 1: raw tau00
  int pad_[3];
};

struct BuildParams {
  const AngularTables *tables;  // device
  const double2 *tmat;          // device tmatStore, column-major (tmat_ld x nstore)
  long tmat_ld;
  int blk;                      // blkSizeTmatStore
  int kkrsz;                    // (maxlmax+1)^2
  int ns;                       // n_spin_cant
  int npola;                    // n_spin_pola
};

// Launchers (return cudaGetLastError of the launch).
cudaError_t launch_kkr_build(const JobDev *jobs, int njobs, int max_L, const BuildParams &p,
                             int *err_flags, cudaStream_t s);
cudaError_t launch_lu_fp64(const JobDev *jobs, int njobs, int max_n, int max_N, int nb,
                           int *info, cudaStream_t s, long *launches);
cudaError_t launch_finalize(const JobDev *jobs, int njobs, int ns, int kkrsz, int *info,
                            cudaStream_t s);

}  // namespace b200
