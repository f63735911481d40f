// Plain-FP64 block elimination for tau00 (batched over jobs).
//
// Restates the reference's block LU contract (zblock_lu_cpp.cpp:19-86, zblock_lu_CPU.f:2-82,
// block_inverse.cpp:24-47, tau_inv_postproc.f:1-77 / linearSolvers_CPU.cpp:299-330):
//   Delta = M0r Mrr^-1 Mr0,  tau00 = (1 - Delta)^-1 t0,  tau00_l = rotate(tau00 - t0).
// The reference eliminates bottom-up with pivoting restricted to each diagonal block (zgetrf on
// the block, zgetrs on its block row, zgemm on the rest; its CUDA variant
// zblock_lu_cuda_c.cu:56-353 re-blocks to 55 columns and inverts each diagonal block).
// Here M is stored with the central site last and eliminated top-down in nb-column steps:
//   1. diag_inverse_kernel  D = A11^-1 by Gauss-Jordan with partial pivoting inside the block
//                           (one CTA per job, block in shared memory),
//   2. zgemm_tile<kOverwrite>  W = D * A12 in place over the block row,
//   3. zgemm_tile<kSubtract>   A22 -= A21 * W over the trailing matrix (the O(N^3) part).
// After n = N - b columns the trailing b x b block holds 1 - Delta; finalize_kernel solves
// (1 - Delta) tau00 = t0 by Gauss-Jordan and writes tau00_l.

#include <cuda_runtime.h>

#include "common.cuh"

namespace b200 {
namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }
__device__ __forceinline__ double2 crecip(double2 a) {
  // 1/a with scaling against overflow of |a|^2
  const double s = fmax(fabs(a.x), fabs(a.y));
  const double ar = a.x / s, ai = a.y / s;
  const double d = ar * ar + ai * ai;
  return make_double2(ar / (d * s), -ai / (d * s));
}

// ---------------------------------------------------------------------------------------------
// 1. In-place Gauss-Jordan inverse of the kb x kb diagonal block at (k, k), kb <= NB.
// ---------------------------------------------------------------------------------------------
template <int NB>
__global__ void __launch_bounds__(256) diag_inverse_kernel(const JobDev *__restrict__ jobs, int k,
                                                           int *info) {
  const JobDev &J = jobs[blockIdx.x];
  if (k >= J.n) return;
  const int kb = min(NB, J.n - k);
  extern __shared__ __align__(16) double2 dyn_smem[];
  double2(*A)[NB + 1] = reinterpret_cast<double2(*)[NB + 1]>(dyn_smem);  // A[row][col]
  __shared__ int perm[NB];
  __shared__ int s_piv;
  __shared__ double2 s_dinv;
  double2 *__restrict__ Mk = J.M + (size_t)k + (size_t)k * J.ld;
  const int tid = threadIdx.x;
  for (int e = tid; e < kb * kb; e += blockDim.x) {
    const int c = e / kb, r = e - c * kb;
    A[r][c] = Mk[r + (size_t)c * J.ld];
  }
  __syncthreads();
  bool singular = false;
  for (int p = 0; p < kb; ++p) {
    if (tid < 32) {  // pivot search |re|+|im| over rows p..kb-1 (izamax convention)
      double best = -1.0;
      int bi = p;
      for (int r = p + tid; r < kb; r += 32) {
        const double v = cabs1(A[r][p]);
        if (v > best) {
          best = v;
          bi = r;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (tid == 0) {
        s_piv = bi;
        perm[p] = bi;
      }
    }
    __syncthreads();
    const int pv = s_piv;
    if (pv != p)
      for (int c = tid; c < kb; c += blockDim.x) {
        const double2 t = A[p][c];
        A[p][c] = A[pv][c];
        A[pv][c] = t;
      }
    __syncthreads();
    if (tid == 0) {
      const double2 d = A[p][p];
      if (d.x == 0.0 && d.y == 0.0) {
        s_dinv = make_double2(0.0, 0.0);
      } else {
        s_dinv = crecip(d);
      }
    }
    __syncthreads();
    const double2 dinv = s_dinv;
    if (dinv.x == 0.0 && dinv.y == 0.0) singular = true;
    // column-owner mapping: thread handles column c = tid % kb, rows r = tid / kb + q * (256/kb)
    const int c = tid % NB;
    const int r0 = tid / NB;
    constexpr int RS = 256 / NB;
    double2 rowp = make_double2(0.0, 0.0);
    double2 f[NB / RS];
    if (c < kb) {
      rowp = (c == p) ? dinv : cmul(A[p][c], dinv);
#pragma unroll
      for (int q = 0; q < NB / RS; ++q) {
        const int r = r0 + q * RS;
        f[q] = (r < kb) ? A[r][p] : make_double2(0.0, 0.0);
      }
    }
    __syncthreads();
    if (c < kb) {
#pragma unroll
      for (int q = 0; q < NB / RS; ++q) {
        const int r = r0 + q * RS;
        if (r >= kb) continue;
        if (r == p) {
          A[r][c] = rowp;
        } else {
          const double2 base = (c == p) ? make_double2(0.0, 0.0) : A[r][c];
          A[r][c] = csub(base, cmul(f[q], rowp));
        }
      }
    }
    __syncthreads();
  }
  // undo the row interchanges as column interchanges, last first
  for (int p = kb - 1; p >= 0; --p) {
    const int pv = perm[p];
    if (pv != p)
      for (int r = tid; r < kb; r += blockDim.x) {
        const double2 t = A[r][p];
        A[r][p] = A[r][pv];
        A[r][pv] = t;
      }
    __syncthreads();
  }
  for (int e = tid; e < kb * kb; e += blockDim.x) {
    const int c = e / kb, r = e - c * kb;
    Mk[r + (size_t)c * J.ld] = A[r][c];
  }
  if (singular && tid == 0) atomicCAS(&info[blockIdx.x], 0, k + 1);
}

// ---------------------------------------------------------------------------------------------
// 2./3. Complex FP64 GEMM tile, C (m x n) = A (m x K) * B (K x n)  [kOverwrite, in place over B]
//                               C (m x n) -= A (m x K) * B (K x n) [kSubtract]
// 64 x 64 complex tile per CTA, 256 threads, 4 x 4 complex accumulators per thread; operands
// double-buffered through shared memory in K-chunks of 16.  Thread (tx, ty) owns rows tx + 16 i
// and columns ty + 16 j so that C / A accesses of consecutive lanes hit consecutive rows of the
// column-major matrix (256-byte segments).
// ---------------------------------------------------------------------------------------------
constexpr int kTile = 64;
constexpr int kKc = 16;
enum { kOverwrite = 0, kSubtract = 1 };

template <int MODE>
__global__ void __launch_bounds__(256) zgemm_tile_kernel(const JobDev *__restrict__ jobs, int k, int nb) {
  const JobDev &J = jobs[blockIdx.z];
  const int N = J.N, ld = J.ld;
  if (k >= J.n) return;
  const int kb = min(nb, J.n - k);
  const int K = kb;
  int row0, m, col0, n;
  const double2 *Ab;
  const double2 *Bb;
  double2 *Cb;
  // block row W = D A12 covers columns k+kb .. N-1 and rows k .. k+kb-1
  col0 = k + kb + blockIdx.x * kTile;
  n = N - col0;
  if (n <= 0) return;
  if (MODE == kOverwrite) {
    if (blockIdx.y != 0) return;
    row0 = k;
    m = kb;
    Ab = J.M + (size_t)k + (size_t)k * ld;  // D (kb x kb)
  } else {
    row0 = k + kb + blockIdx.y * kTile;
    m = N - row0;
    if (m <= 0) return;
    Ab = J.M + (size_t)row0 + (size_t)k * ld;  // A21
  }
  Bb = J.M + (size_t)k + (size_t)col0 * ld;  // A12 / W
  Cb = J.M + (size_t)row0 + (size_t)col0 * ld;
  m = min(m, kTile);
  n = min(n, kTile);

  extern __shared__ __align__(16) double2 dyn_smem[];
  double2(*As)[kKc][kTile] = reinterpret_cast<double2(*)[kKc][kTile]>(dyn_smem);  // As[buf][kk][row]
  double2(*Bs)[kKc][kTile] =
      reinterpret_cast<double2(*)[kKc][kTile]>(dyn_smem + 2 * kKc * kTile);  // Bs[buf][kk][col]
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;

  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);

  // global -> register staging: A chunk kKc x 64 rows (4 per thread), B chunk kKc x 64 cols.
  double2 ra[4], rb[4];
  auto load_chunk = [&](int kc) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;  // 0..1023
      // A: row = e % 64, kk = e / 64
      const int ar = e & 63, ak = e >> 6;
      const int kg = kc + ak;
      ra[q] = (ar < m && kg < K) ? Ab[(size_t)ar + (size_t)kg * ld] : make_double2(0.0, 0.0);
      // B: kk = e % 16, col = e / 16
      const int bk = e & 15, bc = e >> 4;
      const int kg2 = kc + bk;
      rb[q] = (bc < n && kg2 < K) ? Bb[(size_t)kg2 + (size_t)bc * ld] : make_double2(0.0, 0.0);
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
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x = fma(a[i].x, b[j].x, acc[i][j].x);
          acc[i][j].x = fma(-a[i].y, b[j].y, acc[i][j].x);
          acc[i][j].y = fma(a[i].x, b[j].y, acc[i][j].y);
          acc[i][j].y = fma(a[i].y, b[j].x, acc[i][j].y);
        }
    }
    if (ch + 1 < nchunks) store_chunk(buf ^ 1);
    __syncthreads();
  }
  // epilogue (for kOverwrite, every read of B = C happened before the last __syncthreads)
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int c = ty + 16 * j;
    if (c >= n) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = tx + 16 * i;
      if (r >= m) continue;
      double2 *dst = Cb + (size_t)r + (size_t)c * ld;
      if (MODE == kOverwrite) {
        *dst = acc[i][j];
      } else {
        const double2 cv = *dst;
        *dst = make_double2(cv.x - acc[i][j].x, cv.y - acc[i][j].y);
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Finalize: S = trailing b x b block (= 1 - Delta); tau00 = S^-1 t0 by Gauss-Jordan on [S | t0]
// (tau_inv_postproc.f:36-49); out = tau00 - t0, rotated by trgtol for n_spin_cant = 2
// (tau00Postprocess.cpp:52-101, trgtol.f:3-110), or raw tau00 (out_mode 1).
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) finalize_kernel(const JobDev *__restrict__ jobs, int ns,
                                                       int kkrsz, int *info) {
  const JobDev &J = jobs[blockIdx.x];
  const int b = J.b;
  __shared__ double2 A[kMaxB][2 * kMaxB + 1];
  __shared__ int s_piv;
  __shared__ double2 s_dinv;
  const int tid = threadIdx.x;
  const double2 *S = J.M + (size_t)J.n + (size_t)J.n * J.ld;
  for (int e = tid; e < b * b; e += blockDim.x) {
    const int c = e / b, r = e - c * b;
    A[r][c] = S[r + (size_t)c * J.ld];
    const double2 t = J.t0[r + (size_t)c * J.t0_ld];
    A[r][b + c] = t;
  }
  __syncthreads();
  bool singular = false;
  for (int p = 0; p < b; ++p) {
    if (tid < 32) {
      double best = -1.0;
      int bi = p;
      for (int r = p + tid; r < b; r += 32) {
        const double v = cabs1(A[r][p]);
        if (v > best) {
          best = v;
          bi = r;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (tid == 0) s_piv = bi;
    }
    __syncthreads();
    const int pv = s_piv;
    if (pv != p)
      for (int c = tid; c < 2 * b; c += blockDim.x) {
        const double2 t = A[p][c];
        A[p][c] = A[pv][c];
        A[pv][c] = t;
      }
    __syncthreads();
    if (tid == 0) {
      const double2 d = A[p][p];
      s_dinv = (d.x == 0.0 && d.y == 0.0) ? make_double2(0.0, 0.0) : crecip(d);
    }
    __syncthreads();
    const double2 dinv = s_dinv;
    if (dinv.x == 0.0 && dinv.y == 0.0) singular = true;
    // scale row p, then eliminate column p from every other row
    for (int c = tid; c < 2 * b; c += blockDim.x) A[p][c] = cmul(A[p][c], dinv);
    __syncthreads();
    for (int e = tid; e < b * 2 * b; e += blockDim.x) {
      const int r = e / (2 * b), c = e - r * 2 * b;
      if (r == p || c <= p) continue;
      A[r][c] = csub(A[r][c], cmul(A[r][p], A[p][c]));
    }
    __syncthreads();
    for (int r = tid; r < b; r += blockDim.x)
      if (r != p) A[r][p] = make_double2(0.0, 0.0);
    __syncthreads();
  }
  if (singular) {
    if (tid == 0) atomicCAS(&info[blockIdx.x], 0, -1);
  }
  double2 *out = J.out;
  if (J.out_mode == 1) {
    for (int e = tid; e < b * b; e += blockDim.x) {
      const int c = e / b, r = e - c * b;
      out[e] = A[r][b + c];
    }
    return;
  }
  // d = tau00 - t0
  for (int e = tid; e < b * b; e += blockDim.x) {
    const int c = e / b, r = e - c * b;
    A[r][c] = csub(A[r][b + c], J.t0[r + (size_t)c * J.t0_ld]);
  }
  __syncthreads();
  if (ns == 1) {
    for (int e = tid; e < b * b; e += blockDim.x) {
      const int c = e / b, r = e - c * b;
      out[e] = A[r][c];
    }
  } else {
    // ml(:,:,k) = (u d ud) spin block k, k column-major over the 2x2 spin matrix
    const int nr = kkrsz;
    for (int e = tid; e < 4 * nr * nr; e += blockDim.x) {
      const int kblk = e / (nr * nr);
      const int rem = e - kblk * nr * nr;
      const int c = rem / nr, r = rem - c * nr;
      const int ia = kblk & 1, jb = kblk >> 1;
      double2 s = make_double2(0.0, 0.0);
      for (int pp = 0; pp < 2; ++pp)
        for (int qq = 0; qq < 2; ++qq) {
          const double2 f = cmul(J.ubr[ia + 2 * pp], J.ubrd[qq + 2 * jb]);
          const double2 g = A[pp * nr + r][qq * nr + c];
          const double2 fg = cmul(f, g);
          s.x += fg.x;
          s.y += fg.y;
        }
      out[e] = s;
    }
  }
}

}  // namespace

cudaError_t launch_lu_fp64(const JobDev *jobs, int njobs, int max_n, int max_N, int nb,
                           int *info, cudaStream_t s, long *launches) {
  if (nb != 64) return cudaErrorInvalidValue;
  const int smem_diag = 64 * 65 * (int)sizeof(double2);
  const int smem_gemm = 4 * kKc * kTile * (int)sizeof(double2);
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(diag_inverse_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem_diag)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(zgemm_tile_kernel<kOverwrite>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem_gemm)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(zgemm_tile_kernel<kSubtract>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem_gemm)) != cudaSuccess)
    return e;
  for (int k = 0; k < max_n; k += nb) {
    diag_inverse_kernel<64><<<njobs, 256, smem_diag, s>>>(jobs, k, info);
    const int rest = max_N - k - 1;
    const int tiles = (rest + kTile - 1) / kTile;
    if (tiles > 0) {
      zgemm_tile_kernel<kOverwrite><<<dim3(tiles, 1, njobs), 256, smem_gemm, s>>>(jobs, k, nb);
      zgemm_tile_kernel<kSubtract><<<dim3(tiles, tiles, njobs), 256, smem_gemm, s>>>(jobs, k, nb);
    }
    if (launches) *launches += 3;
  }
  return cudaGetLastError();
}

cudaError_t launch_finalize(const JobDev *jobs, int njobs, int ns, int kkrsz, int *info,
                            cudaStream_t s) {
  finalize_kernel<<<njobs, 256, 0, s>>>(jobs, ns, kkrsz, info);
  return cudaGetLastError();
}

}  // namespace b200
