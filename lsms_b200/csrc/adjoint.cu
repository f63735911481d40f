// Reverse-mode derivatives of tau00 and of ln det M with respect to every LIZ site's t-matrix,
// from the FP64 block factors of the forward solve (no second factorisation).
//
// With M = 1 - T G (T = blockdiag(t_j), G the structure constants, G_jj = 0), X = M^-1 [0; t_0]
// (tau00 = X_0, positions with the central site last) and a cotangent taubar on tau00, the
// holomorphic pull-back (no conjugation: delta<taubar, tau00> = sum_j sum_ab tbar_j,ab dt_j,ab) is
//   Lambda = M^-T E_0 taubar,   Z = G X,
//   tbar_j = Lambda_j Z_j^T  (+ Lambda_0 for the central site, which also enters through t_0),
// and d ln det M = tr(M^-1 dM) = -sum_j tr(dt_j (G M^-1)_jj) gives
//   dlogdet_j = -((G M^-1)_jj)^T.
// The reference has no derivative code; these follow from dM = -dT G and d(M^-1) = -M^-1 dM M^-1.
//
// Work: V = M^-1 by the block factors applied to the identity (forward and backward passes of
// batched 64 x 64 FP64 GEMM tiles, ~(2/3) N^3 complex multiply-adds per job), G rebuilt into M's
// storage by the build kernel, then one CTA per (site, job) contracts its row block of G with X
// and with its column block of V (2 N b^2 multiply-adds) and forms the small products.

#include <cuda_runtime.h>

#include "common.cuh"
#include "cplx.cuh"
#include "gj.cuh"

namespace b200 {
namespace {

using namespace cx;

constexpr int kT = 64;   // GEMM tile
constexpr int kKc = 16;  // K chunk
enum { kOverwrite = 0, kSubtract = 1 };

struct GemmView {
  const double2 *A;
  const double2 *B;
  double2 *C;
  int lda, ldb, ldc;
  int m, n, K;
};

// C (m x n) = A B  [kOverwrite, C may alias B: a CTA reads all of its B tile before writing]
// C (m x n) -= A B [kSubtract]
// 64 x 64 complex tile per CTA, 256 threads, 4 x 4 FP64 complex accumulators per thread, operands
// double-buffered through shared memory in K chunks of 16.
template <class Op, int MODE>
__global__ void __launch_bounds__(256) zgemm_view_kernel(const JobDev *__restrict__ jobs, int k, Op op) {
  const JobDev &J = jobs[blockIdx.z];
  GemmView g;
  if (!op(J, k, g)) return;
  const int row0 = blockIdx.y * kT, col0 = blockIdx.x * kT;
  if (row0 >= g.m || col0 >= g.n) return;
  const int m = min(kT, g.m - row0), n = min(kT, g.n - col0), K = g.K;
  const double2 *__restrict__ Ab = g.A + row0;
  const double2 *__restrict__ Bb = g.B + (size_t)col0 * g.ldb;
  double2 *Cb = g.C + row0 + (size_t)col0 * g.ldc;
  extern __shared__ __align__(16) unsigned char zsm[];
  double2(*As)[kKc][kT] = reinterpret_cast<double2(*)[kKc][kT]>(zsm);  // As[buf][kk][row]
  double2(*Bs)[kKc][kT] = reinterpret_cast<double2(*)[kKc][kT]>(zsm + 2 * kKc * kT * sizeof(double2));
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const double2 zero = make_double2(0.0, 0.0);
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = zero;
  double2 ra[4], rb[4];
  auto load_chunk = [&](int kc) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;
      const int ar = e & 63, ak = e >> 6;
      ra[q] = (ar < m && kc + ak < K) ? Ab[(size_t)ar + (size_t)(kc + ak) * g.lda] : zero;
      const int bk = e & 15, bc = e >> 4;
      rb[q] = (bc < n && kc + bk < K) ? Bb[(size_t)(kc + bk) + (size_t)bc * g.ldb] : zero;
    }
  };
  auto store_chunk = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;
      As[buf][e >> 6][e & 63] = ra[q];
      Bs[buf][e & 15][e >> 4] = rb[q];
    }
  };
  const int nchunks = (K + kKc - 1) / kKc;
  load_chunk(0);
  store_chunk(0);
  __syncthreads();
  for (int ch = 0; ch < nchunks; ++ch) {
    const int buf = ch & 1;
    if (ch + 1 < nchunks) load_chunk((ch + 1) * kKc);
#pragma unroll
    for (int kk = 0; kk < kKc; ++kk) {
      double2 a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[buf][kk][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
    }
    if (ch + 1 < nchunks) store_chunk(buf ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int c = ty + 16 * j;
    if (c >= n) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = tx + 16 * i;
      if (r >= m) continue;
      double2 *dst = Cb + (size_t)r + (size_t)c * g.ldc;
      *dst = MODE == kOverwrite ? acc[i][j] : csub(*dst, acc[i][j]);
    }
  }
}

// --- the passes of V = M^-1 = U^-1 S^-1 L^-1 over the block factors in F (positions order) ---
// forward step k:  V_k = D_k V_k  (columns [0, k + kb): L^-1 is lower triangular)
struct OpInvDiag {
  __device__ bool operator()(const JobDev &J, int k, GemmView &g) const {
    if (k >= J.n) return false;
    const int kb = min(kNb, J.n - k);
    const double2 *F = static_cast<const double2 *>(J.F);
    g.A = F + (size_t)k + (size_t)k * J.ld;
    g.B = J.V + k;
    g.C = J.V + k;
    g.lda = g.ldb = g.ldc = J.ld;
    g.m = kb;
    g.n = k + kb;
    g.K = kb;
    return true;
  }
};
// forward step k:  V[k+kb:N, 0:k+kb] -= A21_k V_k
struct OpInvLower {
  __device__ bool operator()(const JobDev &J, int k, GemmView &g) const {
    if (k >= J.n) return false;
    const int kb = min(kNb, J.n - k);
    const double2 *F = static_cast<const double2 *>(J.F);
    g.A = F + (size_t)(k + kb) + (size_t)k * J.ld;
    g.B = J.V + k;
    g.C = J.V + (k + kb);
    g.lda = g.ldb = g.ldc = J.ld;
    g.m = J.N - k - kb;
    g.n = k + kb;
    g.K = kb;
    return g.m > 0;
  }
};
// V_c = S^-1 V_c with S^-1 staged in the Y buffer (b x b, leading dimension ld)
struct OpSchurApply {
  __device__ bool operator()(const JobDev &J, int, GemmView &g) const {
    g.A = J.Y;
    g.B = J.V + J.n;
    g.C = J.V + J.n;
    g.lda = g.ldb = g.ldc = J.ld;
    g.m = J.b;
    g.n = J.N;
    g.K = J.b;
    return true;
  }
};
// backward, block at k (k < 0: the central block):  V[0:k, :] -= W[0:k, k:k+kb] V_k
struct OpInvUpper {
  __device__ bool operator()(const JobDev &J, int k, GemmView &g) const {
    int kb;
    if (k < 0) {
      k = J.n;
      kb = J.b;
    } else {
      if (k >= J.n) return false;
      kb = min(kNb, J.n - k);
    }
    if (k == 0) return false;
    const double2 *F = static_cast<const double2 *>(J.F);
    g.A = F + (size_t)k * J.ld;
    g.B = J.V + k;
    g.C = J.V;
    g.lda = g.ldb = g.ldc = J.ld;
    g.m = k;
    g.n = J.N;
    g.K = kb;
    return true;
  }
};

// V = identity (N x N); one CTA per column
__global__ void __launch_bounds__(256) identity_kernel(const JobDev *__restrict__ jobs) {
  const JobDev &J = jobs[blockIdx.y];
  const int c = blockIdx.x;
  if (c >= J.N) return;
  for (int r = threadIdx.x; r < J.N; r += 256)
    J.V[(size_t)r + (size_t)c * J.ld] = make_double2(r == c ? 1.0 : 0.0, 0.0);
}

// S^-1 (the trailing b x b block of F) into the Y buffer
__global__ void __launch_bounds__(256) schur_inverse_kernel(const JobDev *__restrict__ jobs) {
  const JobDev &J = jobs[blockIdx.x];
  const int b = J.b, n = J.n, ld = J.ld;
  __shared__ double2 A[kMaxB][2 * kMaxB + 1];
  __shared__ int s_piv;
  __shared__ double2 s_dinv;
  const double2 *S = static_cast<const double2 *>(J.F) + (size_t)n + (size_t)n * ld;
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int c = e / b, r = e - c * b;
    A[r][c] = S[r + (size_t)c * ld];
    A[r][b + c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  gj_solve_smem(A, b, &s_piv, &s_dinv);  // a singular S was already reported by the forward solve
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int c = e / b, r = e - c * b;
    J.Y[(size_t)r + (size_t)c * ld] = A[r][b + c];
  }
}

template <class Op, int MODE>
cudaError_t gemm_launch(const JobDev *jobs, int njobs, int k, int max_m, int max_n, cudaStream_t s,
                        long *launches) {
  if (max_m <= 0 || max_n <= 0) return cudaSuccess;
  const int smem = 4 * kKc * kT * (int)sizeof(double2);
  cudaError_t e = ensure_smem(zgemm_view_kernel<Op, MODE>, smem);
  if (e != cudaSuccess) return e;
  zgemm_view_kernel<Op, MODE><<<dim3((max_n + kT - 1) / kT, (max_m + kT - 1) / kT, njobs), 256, smem, s>>>(jobs, k, Op());
  if (launches) *launches += 1;
  return cudaGetLastError();
}

// One CTA per (LIZ position p, job): with G in M's storage, X refined and V = M^-1,
//   Z = G[p, :] X (bp x b),  H = G[p, :] V[:, p] (bp x bp),  Lambda = V[c, p]^T taubar (bp x b),
//   tbar_site = Lambda Z^T (+ Lambda for the central site),  dlogdet_site = -H^T,
// written as b x b blocks in the t-matrix store layout (row s kkrsz + lm for the site's lm < kk,
// zero elsewhere).  bp = ns kk <= kMaxB.
constexpr int kAk = 32;  // K chunk of the contraction
constexpr int kVjpSmem =
    (int)sizeof(double2) * (kMaxB * (kAk + 1) + 2 * kAk * (kMaxB + 1)) > (int)sizeof(double2) * 3 * kMaxB * (kMaxB + 1)
        ? (int)sizeof(double2) * (kMaxB * (kAk + 1) + 2 * kAk * (kMaxB + 1))
        : (int)sizeof(double2) * 3 * kMaxB * (kMaxB + 1);

__global__ void __launch_bounds__(256) vjp_assemble_kernel(const JobDev *__restrict__ jobs, int kkrsz, int ns) {
  const JobDev &J = jobs[blockIdx.y];
  const int p = blockIdx.x;
  if (p >= J.L) return;
  const int off = J.off[p], bp = J.off[p + 1] - off;
  const int site = J.perm[p];
  const int kk = bp / ns;
  const int N = J.N, n = J.n, b = J.b, ld = J.ld;
  // K-chunk staging (G rows of the site, X, V columns of the site), then Z, H and Lambda in the
  // same shared memory (vjp_smem_bytes)
  extern __shared__ __align__(16) unsigned char vsm[];
  double2(*Gs)[kAk + 1] = reinterpret_cast<double2(*)[kAk + 1]>(vsm);
  double2(*Xs)[kMaxB + 1] = reinterpret_cast<double2(*)[kMaxB + 1]>(vsm + sizeof(double2) * kMaxB * (kAk + 1));
  double2(*Vs)[kMaxB + 1] = Xs + kAk;
  double2(*Zs)[kMaxB + 1] = reinterpret_cast<double2(*)[kMaxB + 1]>(vsm);
  double2(*Hs)[kMaxB + 1] = Zs + kMaxB;
  double2(*Ls)[kMaxB + 1] = Hs + kMaxB;  // Lambda
  const int tid = threadIdx.x;
  // each thread owns up to 4 entries of Z (bp x b) and of H (bp x bp): entry e = tid + 256 q
  double2 zacc[4], hacc[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) zacc[q] = hacc[q] = make_double2(0.0, 0.0);
  for (int kc = 0; kc < N; kc += kAk) {
    for (int e = tid; e < bp * kAk; e += 256) {
      const int i = e % bp, kq = e / bp;
      Gs[i][kq] = kc + kq < N ? J.M[(size_t)(off + i) + (size_t)(kc + kq) * ld] : make_double2(0.0, 0.0);
    }
    for (int e = tid; e < kAk * b; e += 256) {
      const int kq = e % kAk, c = e / kAk;
      Xs[kq][c] = kc + kq < N ? J.X[(size_t)(kc + kq) + (size_t)c * ld] : make_double2(0.0, 0.0);
    }
    for (int e = tid; e < kAk * bp; e += 256) {
      const int kq = e % kAk, c = e / kAk;
      Vs[kq][c] = kc + kq < N ? J.V[(size_t)(kc + kq) + (size_t)(off + c) * ld] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + 256 * q;
      if (e < bp * b) {
        const int i = e % bp, c = e / bp;
        for (int kq = 0; kq < kAk; ++kq) zacc[q] = cfma(Gs[i][kq], Xs[kq][c], zacc[q]);
      }
      if (e < bp * bp) {
        const int i = e % bp, c = e / bp;
        for (int kq = 0; kq < kAk; ++kq) hacc[q] = cfma(Gs[i][kq], Vs[kq][c], hacc[q]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {  // (the last barrier of the K loop freed the staging memory)
    const int e = tid + 256 * q;
    if (e < bp * b) Zs[e % bp][e / bp] = zacc[q];
    if (e < bp * bp) Hs[e % bp][e / bp] = hacc[q];
  }
  // Lambda[i][c] = sum_r V[n + r][off + i] taubar[r][c]
  for (int e = tid; e < bp * b; e += 256) {
    const int i = e % bp, c = e / bp;
    double2 s = make_double2(0.0, 0.0);
    for (int r = 0; r < b; ++r)
      s = cfma(J.V[(size_t)(n + r) + (size_t)(off + i) * ld], J.taubar[r + (size_t)c * b], s);
    Ls[i][c] = s;
  }
  __syncthreads();
  double2 *tb = J.tbar + (size_t)site * b * b;
  double2 *dl = J.dlogdet ? J.dlogdet + (size_t)site * b * b : nullptr;
  for (int e = tid; e < b * b; e += 256) {
    const int R = e % b, C = e / b;  // store layout row and column
    const int sr = R / kkrsz, lr = R - sr * kkrsz, sc = C / kkrsz, lc = C - sc * kkrsz;
    double2 tv = make_double2(0.0, 0.0), dv = make_double2(0.0, 0.0);
    if (lr < kk && lc < kk) {
      const int i = sr * kk + lr, j = sc * kk + lc;  // local indices in the site block
      for (int c = 0; c < b; ++c) tv = cfma(Ls[i][c], Zs[j][c], tv);
      if (site == 0) tv = make_double2(tv.x + Ls[i][j].x, tv.y + Ls[i][j].y);
      dv = make_double2(-Hs[j][i].x, -Hs[j][i].y);
    }
    tb[e] = tv;
    if (dl) dl[e] = dv;
  }
}

// Full tau = M^-1 T (T = blockdiag of the sites' t-matrices, positions order) into M's storage:
// one CTA per (256 rows, position p, job), one row per thread; a thread reads the bp elements of
// its row in the position's column block of M^-1 and writes the bp products with t_p.  With panel
// pivoting V holds (P M)^-1, and column j of M^-1 is column rowpos[j] of V.
__global__ void __launch_bounds__(256) tau_full_kernel(const JobDev *__restrict__ jobs, TmatView tv) {
  const JobDev &J = jobs[blockIdx.z];
  const int p = blockIdx.y;
  if (p >= J.L || J.inactive) return;
  const int off = J.off[p], bp = J.off[p + 1] - off;
  const int site = J.perm[p];
  const int kk = bp / tv.ns;  // (lmax + 1)^2 of the site
  __shared__ double2 ts[kMaxB][kMaxB + 1];
  // the site's t block, rows / columns s kk + l for the site's own l < kk (the build's gather)
  const double2 *tb = tv.tmat + (long)J.store[site] * tv.tmat_ld + (long)J.iie * tv.blk + tv.jsm(J.ispin);
  for (int e = threadIdx.x; e < bp * bp; e += 256) {
    const int r = e % bp, c = e / bp;
    const int sr = r / kk, lr = r - sr * kk, sc = c / kk, lc = c - sc * kk;
    ts[r][c] = tb[(sr * tv.kkrsz + lr) + (long)(sc * tv.kkrsz + lc) * tv.bstore];
  }
  __syncthreads();
  const int r = blockIdx.x * 256 + threadIdx.x;
  if (r >= J.N) return;
  const int *__restrict__ rowpos = J.piv != nullptr ? J.piv + J.ld : nullptr;
  double2 v[kMaxB];
#pragma unroll
  for (int k = 0; k < kMaxB; ++k) {
    const int j = off + k;
    const int col = k < bp ? (rowpos != nullptr ? rowpos[j] : j) : 0;
    v[k] = k < bp ? J.V[(size_t)r + (size_t)col * J.ld] : make_double2(0.0, 0.0);
  }
  for (int c = 0; c < bp; ++c) {
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < kMaxB; ++k)
      if (k < bp) acc = cfma(v[k], ts[k][c], acc);
    J.M[(size_t)r + (size_t)(off + c) * J.ld] = acc;
  }
}

}  // namespace

cudaError_t launch_tau_full(const JobDev *jobs, int njobs, int max_L, int max_N, const TmatView &tv, cudaStream_t s,
                            long *launches) {
  if (njobs <= 0) return cudaSuccess;
  tau_full_kernel<<<dim3((max_N + 255) / 256, max_L, njobs), 256, 0, s>>>(jobs, tv);
  if (launches) *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_inverse(const JobDev *jobs, int njobs, int max_n, int max_N, cudaStream_t s, long *launches) {
  if (njobs <= 0) return cudaSuccess;
  cudaError_t e;
  identity_kernel<<<dim3(max_N, njobs), 256, 0, s>>>(jobs);
  if (launches) *launches += 1;
  for (int k = 0; k < max_n; k += kNb) {
    if ((e = gemm_launch<OpInvDiag, kOverwrite>(jobs, njobs, k, kNb, k + kNb, s, launches)) != cudaSuccess) return e;
    if ((e = gemm_launch<OpInvLower, kSubtract>(jobs, njobs, k, max_N - k - 1, k + kNb, s, launches)) != cudaSuccess)
      return e;
  }
  schur_inverse_kernel<<<njobs, 256, 0, s>>>(jobs);
  if (launches) *launches += 1;
  if ((e = gemm_launch<OpSchurApply, kOverwrite>(jobs, njobs, 0, kMaxB, max_N, s, launches)) != cudaSuccess) return e;
  if ((e = gemm_launch<OpInvUpper, kSubtract>(jobs, njobs, -1, max_n, max_N, s, launches)) != cudaSuccess) return e;
  for (int k = ((max_n - 1) / kNb) * kNb; k >= 0 && max_n > 0; k -= kNb)
    if ((e = gemm_launch<OpInvUpper, kSubtract>(jobs, njobs, k, k, max_N, s, launches)) != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t launch_vjp_assemble(const JobDev *jobs, int njobs, int max_L, int kkrsz, int ns, cudaStream_t s,
                                long *launches) {
  if (njobs <= 0) return cudaSuccess;
  cudaError_t e = ensure_smem(vjp_assemble_kernel, kVjpSmem);
  if (e != cudaSuccess) return e;
  vjp_assemble_kernel<<<dim3(max_L, njobs), 256, kVjpSmem, s>>>(jobs, kkrsz, ns);
  if (launches) *launches += 1;
  return cudaGetLastError();
}

}  // namespace b200
