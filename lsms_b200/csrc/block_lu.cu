// Block elimination and iterative refinement for tau00 (batched over jobs).
//
// Restates the reference's block LU contract (zblock_lu_cpp.cpp:19-86, zblock_lu_CPU.f:2-82,
// block_inverse.cpp:24-47, tau_inv_postproc.f:1-77 / linearSolvers_CPU.cpp:299-330):
//   Delta = M0r Mrr^-1 Mr0,  tau00 = (1 - Delta)^-1 t0,  tau00_l = rotate(tau00 - t0).
// The reference eliminates bottom-up with pivoting restricted to each diagonal block (zgetrf on
// the block, zgetrs on its block row, zgemm on the rest; its CUDA variant
// zblock_lu_cuda_c.cu:56-353 re-blocks to 55 columns and inverts each diagonal block).
// Here M is stored with the central site last and eliminated top-down in 64-column steps on the
// factor storage F (FP64 or FP32):
//   diag_inverse_kernel   D = A11^-1, Gauss-Jordan with partial pivoting inside the block (FP64)
//   zgemm_tile<kOverwrite> W = D A12 in place over the block row
//   zgemm_tile<kSubtract>  A22 -= A21 W over the trailing matrix (the O(N^3) part; the mixed path
//                          replaces this launch by the tensor-core kernel in tc_update.cu)
// After n = N - b columns the trailing b x b block holds S = 1 - Delta and F holds, in place, the
// block factors {D_k in the diagonal blocks, A21_k below them, W_k to their right}.
// Without refinement, finalize solves S tau00 = t0.  With refinement (the reference's zcgesv /
// cusolverDnIRSXgesv idea, linearSolvers_CPU.cpp:148-174, linearSolvers_CUDA.cu:424-469, applied
// to the N x b system M X = [0; t0]):
//   X = F^-1 B;  repeat: R = B - M X (FP64, M unmodified), Y = F^-1 R, X += Y;
// where F^-1 is a forward sweep (Y_k = D_k R_k, R_below -= A21_k Y_k), the S solve, and a backward
// sweep (Y_above -= W Y_k), each one launch with a thread-block cluster per job (sweep.cu).
// tau00 = X[n:N].

#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "cplx.cuh"
#include "gj.cuh"

namespace b200 {
namespace {

using namespace cx;

template <typename S> struct Vec2;
template <> struct Vec2<double> { using t = double2; };
template <> struct Vec2<float> { using t = float2; };

// ---------------------------------------------------------------------------------------------
// In-place inverse of the kb x kb diagonal block at (k, k) of F, kb <= 64: FP64 Gauss-Jordan with
// partial pivoting inside the block on |re| + |im| (izamax's measure; ties go to the lowest row).
// Rows are never interchanged: step p pivots on the not-yet-used row pv with the largest
// |A[pv][p]|, and the permutation is applied when the block is written back (for the in-place
// result P, A^-1[i][pv_k] = P[pv_i][k]).
// One Gauss-Jordan step as a single rank-1 update of the whole block, A[r][c] -= g_r u_c, with
//   u = row pv, except u_p = d + 1 (d = A[pv][p]);   g_r = A[r][p] / d (r != pv),  g_pv = 1 - 1/d:
// row pv becomes A[pv][c] / d, column p becomes -A[r][p] / d, and A[pv][p] becomes 1/d, as the
// in-place inverse needs, with no special cases in the update.
// Layout: warp w holds columns 8w .. 8w + 7 and lane l rows l and l + 32, in registers (the step
// loop is not unrolled: an unrolled body outgrows the instruction caches).  Per step the warp
// holding column p finds the pivot (warp argmax) and publishes g; after the one block barrier of
// the step, in every warp the lane holding row pv publishes u over the warp's columns (a per-warp
// slot in shared memory, read only by that warp) and all lanes apply the update.
// ---------------------------------------------------------------------------------------------
// Pivot search key of a row: |re| + |im| (non-negative doubles order as their bit patterns; NaN
// counts as 0) with its 6 low mantissa bits replaced by 63 - row, so that the largest key is the
// largest value, ties - and values within 2^-46 relative of each other - going to the lowest row.
__device__ __forceinline__ unsigned long long pivot_key(double v, int row) {
  v = (v == v) ? v : 0.0;
  return ((unsigned long long)__double_as_longlong(v) & ~63ull) | (unsigned long long)(63 - row);
}

constexpr int kDiagThreads = 256;
constexpr int kDiagWarps = kDiagThreads / 32;
static_assert(kDiagWarps * 8 == kNb && kNb == 64, "diagonal inverse layout: 8 columns per warp, 2 rows per lane");

// PER_SM = blocks per SM the register budget allows: 1 (the update's chains unconstrained, for the
// elimination that keeps one SM per job free for the inverses) or 2 (two per SM, for the
// elimination with panel pivoting, which leaves fewer SMs to them).
template <typename T, int PER_SM>
__global__ void __launch_bounds__(kDiagThreads, PER_SM) diag_inverse_kernel(const JobDev *__restrict__ jobs, int k,
                                                                            int *info) {
  constexpr int NB = kNb;
  const JobDev &J = jobs[blockIdx.x];
  if (k >= J.n || J.inactive) return;
  const int kb = min(NB, J.n - k);
  extern __shared__ __align__(16) double2 dyn_smem[];
  double2(*As)[NB + 1] = reinterpret_cast<double2(*)[NB + 1]>(dyn_smem);  // staging As[row][col]
  __shared__ double2 s_g[2][NB];              // the step's row factors g, by step parity
  __shared__ double2 s_row[kDiagWarps][8];    // per warp: u over the warp's columns
  __shared__ int s_pvp[2];
  __shared__ int s_sing[2];
  __shared__ int s_pv[NB], s_inv[NB];
  T *__restrict__ Fk = static_cast<T *>(J.F) + (size_t)k + (size_t)k * J.ld;
  const int tid = threadIdx.x;
  constexpr int kPer = NB * NB / kDiagThreads;  // entries per thread of a full block
  if (kb == NB) {
    // all of a thread's loads in flight at once (a loop over them waits out one DRAM round trip
    // per entry)
    double2 v[kPer];
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int e = tid + i * kDiagThreads;
      v[i] = ldc(Fk + (e % NB) + (size_t)(e / NB) * J.ld);
    }
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int e = tid + i * kDiagThreads;
      As[e % NB][e / NB] = v[i];
    }
  } else {
    for (int e = tid; e < kb * kb; e += kDiagThreads) {
      const int cc = e / kb, r = e - cc * kb;
      As[r][cc] = ldc(Fk + r + (size_t)cc * J.ld);
    }
  }
  if (tid < NB) s_inv[tid] = tid;  // every entry in range whatever the pivots
  __syncthreads();
  const int w = tid >> 5, l = tid & 31;
  double2 a[2][8];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int r = l + 32 * i, c = 8 * w + j;
      a[i][j] = (r < kb && c < kb) ? As[r][c] : make_double2(0.0, 0.0);
    }
  // rows already pivoted on (rows past kb count as used, so they are never chosen)
  bool used0 = l >= kb, used1 = l + 32 >= kb;
  bool singular = false;
#pragma unroll 1
  for (int p = 0; p < kb; ++p) {
    const int par = p & 1;
    if (w == (p >> 3)) {
      // column p & 7 of this warp's registers (opaque copies: the compiler otherwise turns the
      // selection into an indexed local-memory load)
      double2 x0 = make_double2(0.0, 0.0), x1 = x0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        double2 t0 = a[0][j], t1 = a[1][j];
        asm volatile("" : "+d"(t0.x), "+d"(t0.y), "+d"(t1.x), "+d"(t1.y));
        if (j == (p & 7)) {
          x0 = t0;
          x1 = t1;
        }
      }
      // the pivot: the unused row of largest |re| + |im| as the largest 64-bit key (pivot_key),
      // two warp max-reductions (high word, then the low word among the lanes holding the high max)
      const unsigned long long k0 = used0 ? 0ull : pivot_key(cabs1(x0), l);
      const unsigned long long k1 = used1 ? 0ull : pivot_key(cabs1(x1), l + 32);
      const unsigned long long kl = k0 > k1 ? k0 : k1;
      const unsigned hi = (unsigned)(kl >> 32);
      const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
      const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? (unsigned)kl : 0u);
      // kb - p unused rows remain, so the key names one of them (a row < kb)
      const int pv = min(63 - (int)(mlo & 63u), kb - 1);
      const double2 xs = (pv >> 5) ? x1 : x0;
      double2 d;
      d.x = __shfl_sync(0xffffffffu, xs.x, pv & 31);
      d.y = __shfl_sync(0xffffffffu, xs.y, pv & 31);
      // 1/d = conj(d) / |d|^2 in every lane (pivots of these blocks are far from the FP64 range limits)
      const bool zero = d.x == 0.0 && d.y == 0.0;
      double2 dinv = make_double2(0.0, 0.0);
      if (!zero) {
        const double rr = 1.0 / (d.x * d.x + d.y * d.y);
        dinv = make_double2(d.x * rr, -d.y * rr);
      }
      s_g[par][l] = (l == pv) ? make_double2(1.0 - dinv.x, -dinv.y) : cmul(x0, dinv);
      s_g[par][l + 32] = (l + 32 == pv) ? make_double2(1.0 - dinv.x, -dinv.y) : cmul(x1, dinv);
      if (l == 0) {
        s_pvp[par] = pv;
        s_sing[par] = zero ? 1 : 0;
        s_pv[p] = pv;
      }
    }
    __syncthreads();
    const int pv = s_pvp[par];
    if (s_sing[par]) singular = true;
    const int pl = pv & 31, pi = pv >> 5;
    if (l == pl) {  // publish u over this warp's columns, then mark row pv used
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        double2 v = pi ? a[1][jj] : a[0][jj];
        if (8 * w + jj == p) v.x += 1.0;
        s_row[w][jj] = v;
      }
      if (pi) used1 = true;
      else used0 = true;
    }
    __syncwarp();
    const double2 g0 = s_g[par][l], g1 = s_g[par][l + 32];
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
      const double2 u = s_row[w][jj];
      a[0][jj].x = fma(-g0.x, u.x, a[0][jj].x);
      a[0][jj].x = fma(g0.y, u.y, a[0][jj].x);
      a[0][jj].y = fma(-g0.x, u.y, a[0][jj].y);
      a[0][jj].y = fma(-g0.y, u.x, a[0][jj].y);
      a[1][jj].x = fma(-g1.x, u.x, a[1][jj].x);
      a[1][jj].x = fma(g1.y, u.y, a[1][jj].x);
      a[1][jj].y = fma(-g1.x, u.y, a[1][jj].y);
      a[1][jj].y = fma(-g1.y, u.x, a[1][jj].y);
    }
  }
  __syncthreads();
  if (tid < kb) s_inv[s_pv[tid]] = tid;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int r = l + 32 * i, c = 8 * w + j;
      if (r < kb && c < kb) As[s_inv[r]][s_pv[c]] = a[i][j];
    }
  __syncthreads();
  if (kb == NB) {
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int e = tid + i * kDiagThreads;
      stc(Fk + (e % NB) + (size_t)(e / NB) * J.ld, As[e % NB][e / NB]);
    }
  } else {
    for (int e = tid; e < kb * kb; e += kDiagThreads) {
      const int cc = e / kb, r = e - cc * kb;
      stc(Fk + r + (size_t)cc * J.ld, As[r][cc]);
    }
  }
  if (singular && tid == 0) atomicCAS(&info[blockIdx.x], 0, k + 1);
}

template <typename T>
void launch_diag_inverse(bool packed, const JobDev *jobs, int njobs, int k, int *info, int smem, cudaStream_t s) {
  if (packed) diag_inverse_kernel<T, 2><<<njobs, kDiagThreads, smem, s>>>(jobs, k, info);
  else diag_inverse_kernel<T, 1><<<njobs, kDiagThreads, smem, s>>>(jobs, k, info);
}

// ---------------------------------------------------------------------------------------------
// Complex GEMM tile on F (SIMT), C (m x n) = A (m x K) B (K x n)  [kOverwrite, in place over B]
//                                C (m x n) -= A (m x K) B (K x n) [kSubtract]
// 64 x 64 complex tile per CTA, 256 threads, 4 x 4 complex accumulators per thread in the storage
// precision S; operands double-buffered through shared memory in K-chunks of 16.  Thread (tx, ty)
// owns rows tx + 16 i and columns ty + 16 j so consecutive lanes touch consecutive rows of the
// column-major matrix.
// ---------------------------------------------------------------------------------------------
constexpr int kTile = 64;
constexpr int kKc = 16;
enum { kOverwrite = 0, kSubtract = 1 };

// Optional second output of the W = D A12 tiles (FP32, tensor-core path): W's hi/lo TF32 split in
// the K-major operand layout of the trailing update (column c of the trailing block at
// b + z * slot + c * kTcKMax + k_off floats, (re, im) of row p at 2 p), job z = the launch's job
// index.  With shift_k >= 0 the trailing block is that of the next step shift_k (its columns
// start kb(shift_k) further right; W's columns left of it are not packed), and this step's rows
// go to K offset k_off: the first half of a two-step update's operand.
struct PackB {
  float *hi = nullptr, *lo = nullptr;
  size_t slot = 0;
  int shift_k = -1;
  int k_off = 0;
};

__device__ __forceinline__ float tf32_round(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

template <typename S, int MODE>
__device__ __forceinline__ void zgemm_tile_body(const JobDev &J, int k, int bx, int by, int bx0, int by0,
                                                const PackB &pk = PackB(), int z = 0) {
  using T = typename Vec2<S>::t;
  const int N = J.N, ld = J.ld;
  if (k >= J.n || J.inactive) return;
  const int kb = min(kNb, J.n - k);
  const int K = kb;
  T *__restrict__ F = static_cast<T *>(J.F);
  int row0, m;
  const T *Ab;
  const int col0 = k + kb + (bx + bx0) * kTile;
  int n = N - col0;
  if (n <= 0) return;
  if (MODE == kOverwrite) {
    if (by != 0) return;
    row0 = k;
    m = kb;
    Ab = F + (size_t)k + (size_t)k * ld;  // D (kb x kb)
  } else {
    row0 = k + kb + (by + by0) * kTile;
    m = N - row0;
    if (m <= 0) return;
    Ab = F + (size_t)row0 + (size_t)k * ld;  // A21
  }
  const T *Bb = F + (size_t)k + (size_t)col0 * ld;  // A12 / W
  T *Cb = F + (size_t)row0 + (size_t)col0 * ld;
  m = min(m, kTile);
  n = min(n, kTile);

  extern __shared__ __align__(16) unsigned char zsm[];
  T(*As)[kKc][kTile] = reinterpret_cast<T(*)[kKc][kTile]>(zsm);  // As[buf][kk][row]
  T(*Bs)[kKc][kTile] = reinterpret_cast<T(*)[kKc][kTile]>(zsm + 2 * kKc * kTile * sizeof(T));
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const T zero = {S(0), S(0)};

  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = zero;

  T ra[4], rb[4];
  auto load_chunk = [&](int kc) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + q * 256;
      const int ar = e & 63, ak = e >> 6;
      const int kg = kc + ak;
      ra[q] = (ar < m && kg < K) ? Ab[(size_t)ar + (size_t)kg * ld] : zero;
      const int bk = e & 15, bc = e >> 4;
      const int kg2 = kc + bk;
      rb[q] = (bc < n && kg2 < K) ? Bb[(size_t)kg2 + (size_t)bc * ld] : zero;
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
      T a[4], b[4];
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
  // for kOverwrite every read of B = C happened before the last __syncthreads
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int c = ty + 16 * j;
    if (c >= n) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = tx + 16 * i;
      if (MODE == kOverwrite && sizeof(S) == 4 && pk.hi != nullptr) {
        // rows past kb pack as zero
        const int shift = pk.shift_k >= 0 ? min(kNb, J.n - pk.shift_k) : 0;
        const int prow = (bx + bx0) * kTile + c - shift;
        if (prow >= 0) {
          const float wr = r < m ? (float)acc[i][j].x : 0.f, wi = r < m ? (float)acc[i][j].y : 0.f;
          const float hr = tf32_round(wr), hi = tf32_round(wi);
          const size_t o = (size_t)z * pk.slot + (size_t)prow * kTcKMax + pk.k_off;
          reinterpret_cast<float2 *>(pk.hi + o)[r] = make_float2(hr, hi);
          reinterpret_cast<float2 *>(pk.lo + o)[r] = make_float2(wr - hr, wi - hi);
        }
      }
      if (r >= m) continue;
      T *dst = Cb + (size_t)r + (size_t)c * ld;
      if (MODE == kOverwrite) {
        *dst = acc[i][j];
      } else {
        const T cv = *dst;
        *dst = T{cv.x - acc[i][j].x, cv.y - acc[i][j].y};
      }
    }
  }
}

// One output tile per (bx, by, job).  Launched either with that 3-D grid, or with a smaller 1-D
// grid whose CTAs loop over the tiles (the FP64 re-solve of a mixed wave, where most jobs are
// inactive and a full grid would spend its time launching CTAs that exit at once).
// Two resident CTAs per SM: with K = 64 per step each CTA runs only four K-chunks, so its operand
// prologue and C read-modify-write latencies are hidden by the other CTA's FMAs.
// Tiles start at column tile bx0 and row tile by0 of the step's trailing block.
template <typename S, int MODE>
__global__ void __launch_bounds__(256, 2) zgemm_tile_kernel(const JobDev *__restrict__ jobs, int k, int tx, int ty,
                                                            int nj, PackB pk, int bx0, int by0 = 0) {
  if (gridDim.z == (unsigned)nj && gridDim.x == (unsigned)tx && gridDim.y == (unsigned)ty) {
    zgemm_tile_body<S, MODE>(jobs[blockIdx.z], k, blockIdx.x, blockIdx.y, bx0, by0, pk, blockIdx.z);
    return;
  }
  // looping grid: jobs one after another (an inactive job costs one check), its tiles spread
  // over the CTAs
  const int nblk = gridDim.x * gridDim.y * gridDim.z;
  const int b0 = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  for (int bz = 0; bz < nj; ++bz) {
    const JobDev &J = jobs[bz];
    if (J.inactive || k >= J.n) continue;
    for (int vb = b0; vb < tx * ty; vb += nblk) zgemm_tile_body<S, MODE>(J, k, vb % tx, vb / tx, bx0, by0);
  }
}


// Step k's update of the two strips a paired step k2 = k + 64 needs before its own W (block
// pivoting): block column k2 below its diagonal block (CTAs x < t1: row tiles 1 .. t1) and block
// row k2 right of it (x >= t1: column tiles 1 .. t1), one grid of 2 t1 x njobs CTAs, so that the
// last wave of one strip shares the GPU with the other.
template <typename S>
__global__ void __launch_bounds__(256, 2) zgemm_strips_kernel(const JobDev *__restrict__ jobs, int k, int t1) {
  const int x = blockIdx.x;
  if (x < t1) zgemm_tile_body<S, kSubtract>(jobs[blockIdx.z], k, 0, x, 0, 1);
  else zgemm_tile_body<S, kSubtract>(jobs[blockIdx.z], k, x - t1, 0, 1, 0);
}

// out = tau00 (out_mode 1) or rotate(tau00 - t0) (out_mode 0), tau00 in A[r][b + c].
__device__ void write_out(const JobDev &J, double2 (*A)[2 * kMaxB + 1], int ns, int kkrsz) {
  const int tid = threadIdx.x;
  const int b = J.b;
  double2 *out = J.out;
  if (J.out_mode == 1) {
    for (int e = tid; e < b * b; e += blockDim.x) {
      const int c = e / b, r = e - c * b;
      out[e] = A[r][b + c];
    }
    return;
  }
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
    // trgtol.f:3-110: ml(:,:,k) = (u d ud) spin block k, k column-major over the 2x2 spin matrix
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
          const double2 fg = cmul(f, A[pp * nr + r][qq * nr + c]);
          s.x += fg.x;
          s.y += fg.y;
        }
      out[e] = s;
    }
  }
}

// tau00 = S^-1 t0 from the Schur block in F (no refinement).
template <typename T>
__global__ void __launch_bounds__(256) finalize_direct_kernel(const JobDev *__restrict__ jobs, int ns,
                                                              int kkrsz, int *info) {
  const JobDev &J = jobs[blockIdx.x];
  const int b = J.b;
  __shared__ double2 A[kMaxB][2 * kMaxB + 1];
  __shared__ int s_piv;
  __shared__ double2 s_dinv;
  const T *Sb = static_cast<const T *>(J.F) + (size_t)J.n + (size_t)J.n * J.ld;
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int c = e / b, r = e - c * b;
    A[r][c] = ldc(Sb + r + (size_t)c * J.ld);
    A[r][b + c] = J.t0[r + (size_t)c * J.t0_ld];
  }
  __syncthreads();
  if (gj_solve_smem(A, b, &s_piv, &s_dinv) && threadIdx.x == 0) atomicCAS(&info[blockIdx.x], 0, -1);
  write_out(J, A, ns, kkrsz);
}

// out from X[n:N] (refined tau00).
__global__ void __launch_bounds__(256) finalize_from_x_kernel(const JobDev *__restrict__ jobs, int ns,
                                                              int kkrsz) {
  const JobDev &J = jobs[blockIdx.x];
  if (J.inactive) return;
  // a dataflow sweep whose bounded wait ran out aborted this job: report it in the error word
  if (threadIdx.x == 0 && J.conv != nullptr && J.err != nullptr && *J.conv == kAborted)
    atomicOr(J.err, kErrSweepWait);
  const int b = J.b;
  __shared__ double2 A[kMaxB][2 * kMaxB + 1];
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int c = e / b, r = e - c * b;
    A[r][b + c] = J.X[(size_t)(J.n + r) + (size_t)c * J.ld];
  }
  __syncthreads();
  write_out(J, A, ns, kkrsz);
}

// ---------------------------------------------------------------------------------------------
// Refinement pieces.  X, R, Y are N x b FP64 column-major with leading dimension ld.
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ bool converged(const JobDev &J) { return cx::converged(J.conv); }

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}

// R = B - M X with B = [0; t0] (rows n..N-1 hold t0), FP64.  The product is FP64 bound (b complex
// multiply-adds per 16-byte element of M) and runs on the FP64 tensor cores (mma.sync m8n8k4
// f64): as real products, [Rr | Ri] = Mr [Xr | Xi] + Mi [-Xi | Xr], four 8 x 8 x 4 MMAs per row
// tile and 8-column block per K step of 4, a few instructions per 1024 FMAs where DFMAs take 32.
// Each warp owns ROWS / 4 rows (8-row tiles) x BC columns of accumulators.  M and X stream
// through a three-stage cp.async ring in shared memory (kResK columns of M and rows of X per
// stage), so two stages of loads are in flight while one is multiplied.
// BC = 16 or 32 is the padded column count (b <= BC).
constexpr int kResK = 8;       // K per stage
constexpr int kResStages = 3;

constexpr int kResThreads = 128;  // four CTAs per SM, so a round on a few jobs still spans the GPU
template <int BC>
__host__ __device__ constexpr int residual_rows() {
  return kResThreads * 16 / BC;
}
template <int BC>
__host__ __device__ constexpr int residual_smem_bytes() {
  return kResStages * kResK * (residual_rows<BC>() + BC) * (int)sizeof(double2);
}

// D (8 x 8) += A (8 x 4) B (4 x 8) in FP64 on the tensor cores, per warp: lane l holds
// a = A[l / 4][l % 4], b = B[l % 4][l / 4] and D[l / 4][2 (l % 4) + i] in d_i.
__device__ __forceinline__ void dmma_884(double &d0, double &d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// The jobs of a wave still refining: list[0] = their number, list[1..] their indices in order.
// One warp.
__global__ void active_list_kernel(const JobDev *__restrict__ jobs, int njobs, int *list) {
  const int lane = threadIdx.x;
  int count = 0;
  for (int base = 0; base < njobs; base += 32) {
    const int w = base + lane;
    const bool a = w < njobs && !converged(jobs[w]) && !jobs[w].inactive;
    const unsigned mask = __ballot_sync(0xffffffffu, a);
    if (a) list[1 + count + __popc(mask & ((1u << lane) - 1u))] = w;
    count += __popc(mask);
  }
  if (lane == 0) list[0] = count;
}

// Without a list: grid (jobs, row blocks), converged jobs leave at once.  With `active` (from
// active_list_kernel): a 1-D grid whose first count x rowblocks CTAs take (active job i % count,
// row block i / count), so the jobs still refining spread evenly over the SMs; the rest leave.
template <int BC>
__global__ void __launch_bounds__(kResThreads, 4) residual_kernel(const JobDev *__restrict__ jobs,
                                                                  const int *__restrict__ active, int rowblocks) {
  constexpr int ROWS = residual_rows<BC>();  // rows per CTA
  constexpr int RT = ROWS / 32;              // 8-row tiles per warp (four warps)
  constexpr int NB = BC / 8;                 // 8-column blocks
  static_assert(kResThreads == 128 && RT * 32 == ROWS && NB * 8 == BC && kResK % 4 == 0, "residual layout");
  int jw = blockIdx.x, rb = blockIdx.y;
  if (active != nullptr) {
    const int cnt = active[0], i = blockIdx.x;
    if (i >= cnt * rowblocks) return;
    jw = active[1 + i % cnt];
    rb = i / cnt;
  }
  const JobDev &J = jobs[jw];
  if (converged(J) || J.inactive) return;
  const int N = J.N, ld = J.ld, b = J.b;
  const int row0 = rb * ROWS;
  if (row0 >= N) return;
  extern __shared__ __align__(16) unsigned char rsm[];
  double2(*Ms)[kResK][ROWS] = reinterpret_cast<double2(*)[kResK][ROWS]>(rsm);
  double2(*Xs)[kResK][BC] =
      reinterpret_cast<double2(*)[kResK][BC]>(rsm + sizeof(double2) * kResStages * kResK * ROWS);
  const int tid = threadIdx.x;
  const int lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int wrow = (tid >> 5) * (8 * RT);  // the warp's first row within the CTA's rows
  const double2 *__restrict__ M = J.M;
  const double2 *__restrict__ X = J.X;
  const double2 zero = make_double2(0.0, 0.0);
  // columns [k0, k0 + kResK) of M (rows of the CTA) and rows [k0, k0 + kResK) of X into stage st;
  // entries past N or b read as zero
  auto stage = [&](int k0, int st) {
    for (int e = tid; e < kResK * ROWS; e += kResThreads) {
      const int kk = e / ROWS, rr = e - kk * ROWS;
      const int gk = k0 + kk, grr = row0 + rr;
      if (gk < N && grr < N) cp_async16(&Ms[st][kk][rr], M + (size_t)grr + (size_t)gk * ld);
      else Ms[st][kk][rr] = zero;
    }
    for (int e = tid; e < kResK * BC; e += kResThreads) {
      const int kk = e % kResK, c = e / kResK;
      const int gk = k0 + kk;
      if (c < b && gk < N) cp_async16(&Xs[st][kk][c], X + (size_t)gk + (size_t)c * ld);
      else Xs[st][kk][c] = zero;
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  double ar[RT][NB][2], ai[RT][NB][2];  // M X, real and imaginary parts
#pragma unroll
  for (int r = 0; r < RT; ++r)
#pragma unroll
    for (int j = 0; j < NB; ++j) ar[r][j][0] = ar[r][j][1] = ai[r][j][0] = ai[r][j][1] = 0.0;
  const int nst = (N + kResK - 1) / kResK;
#pragma unroll
  for (int q = 0; q < kResStages - 1; ++q) {
    if (q < nst) stage(q * kResK, q);
    else asm volatile("cp.async.commit_group;" ::: "memory");
  }
  for (int q = 0; q < nst; ++q) {
    asm volatile("cp.async.wait_group %0;" ::"n"(kResStages - 2) : "memory");
    __syncthreads();  // stage q landed for every thread; stage q - 1 is no longer read
    const int nq = q + kResStages - 1;
    if (nq < nst) stage(nq * kResK, nq % kResStages);
    else asm volatile("cp.async.commit_group;" ::: "memory");
    const int st = q % kResStages;
#pragma unroll
    for (int ks = 0; ks < kResK; ks += 4) {
      double2 xv[NB];
#pragma unroll
      for (int j = 0; j < NB; ++j) xv[j] = Xs[st][ks + t][8 * j + g];
#pragma unroll
      for (int r = 0; r < RT; ++r) {
        const double2 mv = Ms[st][ks + t][wrow + 8 * r + g];
#pragma unroll
        for (int j = 0; j < NB; ++j) {
          dmma_884(ar[r][j][0], ar[r][j][1], mv.x, xv[j].x);
          dmma_884(ar[r][j][0], ar[r][j][1], mv.y, -xv[j].y);
          dmma_884(ai[r][j][0], ai[r][j][1], mv.x, xv[j].y);
          dmma_884(ai[r][j][0], ai[r][j][1], mv.y, xv[j].x);
        }
      }
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  // with panel pivoting the factors are those of P M: row gr of R goes to its physical row
  const int *__restrict__ rowpos = J.piv != nullptr ? J.piv + ld : nullptr;
#pragma unroll
  for (int r = 0; r < RT; ++r) {
    const int gr = row0 + wrow + 8 * r + g;
    if (gr >= N) continue;
    const int dst = rowpos != nullptr ? rowpos[gr] : gr;
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int c = 8 * j + 2 * t + i;
        if (c >= b) continue;
        const double2 bv = (gr >= J.n) ? J.t0[(gr - J.n) + (size_t)c * J.t0_ld] : zero;
        J.R[(size_t)dst + (size_t)c * ld] = make_double2(bv.x - ar[r][j][i], bv.y - ai[r][j][i]);
      }
  }
}

// Y[n:N] = S^-1 rhs with rhs = R[n:N] (mode 1) or t0 (mode 0, which also zeroes Y[0:n]).
template <typename T>
__global__ void __launch_bounds__(256) schur_solve_kernel(const JobDev *__restrict__ jobs, int mode,
                                                          int *info) {
  const JobDev &J = jobs[blockIdx.x];
  if ((mode == 1 && converged(J)) || J.inactive) return;
  const int b = J.b, n = J.n, ld = J.ld;
  __shared__ double2 A[kMaxB][2 * kMaxB + 1];
  __shared__ int s_piv;
  __shared__ double2 s_dinv;
  const T *Sb = static_cast<const T *>(J.F) + (size_t)n + (size_t)n * ld;
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int c = e / b, r = e - c * b;
    A[r][c] = ldc(Sb + r + (size_t)c * ld);
    A[r][b + c] = mode == 0 ? J.t0[r + (size_t)c * J.t0_ld] : J.R[(size_t)(n + r) + (size_t)c * ld];
  }
  if (mode == 0)
    for (int e = threadIdx.x; e < n * b; e += blockDim.x) {
      const int r = e % n, c = e / n;
      J.Y[(size_t)r + (size_t)c * ld] = make_double2(0.0, 0.0);
    }
  __syncthreads();
  if (gj_solve_smem(A, b, &s_piv, &s_dinv) && threadIdx.x == 0) atomicCAS(&info[blockIdx.x], 0, -1);
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int c = e / b, r = e - c * b;
    J.Y[(size_t)(n + r) + (size_t)c * ld] = A[r][b + c];
  }
}

// CTAs of the looping trailing-update grid (two per SM)
constexpr int kSparseGrid = 2 * 148;

// Step k: W = D A12 (with W's operand pack) and A21's pack on s, then the update of the tile holding
// the next diagonal block; s2 waits for it and inverts that block while s updates the other tiles;
// s waits for the inverse before step k + 1.  Only the diagonal inverse moves off s, so the packs of step k + 1 are
// written after every tile of step k has read those of step k.
// With panel pivoting the first update covers the whole first tile column (the next step's panel,
// every row), the second stream also runs the next step's row selection and applies its row moves to
// the columns left of the other tiles, and the main stream applies them to the other columns once
// their update is done.
template <typename T, typename S>
cudaError_t eliminate_lookahead(const JobDev *jobs, int njobs, int max_n, int max_N, int *info, cudaStream_t s,
                                long *launches, KernelTimer *timer, const TcMaps &tc, int *err, const Lookahead &la,
                                int smem_diag, int smem_gemm, bool panel) {
  cudaError_t e;
  const FactorKind fk = sizeof(T) == sizeof(double2) ? kFactorFP64 : kFactorFP32;
  // SMs left to the second stream's work during the interior update.  The update is a persistent
  // kernel with a fixed share of tiles per CTA, so a CTA of it that cannot start (an inverse took
  // its SM) delays the whole launch: without panel pivoting the inverses, which the scheduler may
  // spread one per SM, get one SM per job.  With panel pivoting the row selection (one block per
  // SM) runs first on the second stream, in waves over the SMs left to it, and the inverses then
  // pack at their occupancy: one wave of those is enough, and the update keeps more SMs.
  int per_sm = 1;
  if (panel && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, diag_inverse_kernel<T, 2>, kDiagThreads,
                                                               smem_diag) != cudaSuccess ||
                per_sm < 1)) {
    cudaGetLastError();
    per_sm = 1;
  }
  const int free_sms = std::min((njobs + per_sm - 1) / per_sm, tc_num_sms() / 2);
  if (panel) {
    if ((e = launch_pivot_init(jobs, njobs, s, launches)) != cudaSuccess) return e;
    if ((e = launch_panel_select(fk, jobs, njobs, 0, max_n, s, launches)) != cudaSuccess) return e;
    if ((e = launch_row_moves(fk, jobs, njobs, 0, 0, max_N, max_N, s, launches)) != cudaSuccess) return e;
  }
  launch_diag_inverse<T>(panel, jobs, njobs, 0, info, smem_diag, s);
  if (launches) *launches += 1;
  for (int k = 0; k < max_n; k += kNb) {
    const int rest = max_N - k - 1;
    const int tiles = (rest + kTile - 1) / kTile;
    const bool next = k + kNb < max_n;
    const int k2 = k + kNb;
    // Paired steps k and k2: the update of the trailing block after k2 by both steps in one pass
    // (its FP32 read-modify-write, which bounds the update, once per two steps).  Step k's update
    // of the strips that step k2 needs first (block column k2, which holds the next diagonal
    // block, and block row k2) runs as SIMT tiles; the factors left in F are those of two
    // single steps.
    // With panel pivoting the pair keeps every row's pending update the same when step k2's rows
    // move: block column k2 is updated by step k (all rows) before step k2's selection, and block
    // row k2 only after its row moves, so that at the moves every row below step k still owes
    // step k's update right of block column k2 (done for all of them by the combined pass) and
    // the moves carry A21_k's rows with them.
    if (panel && la.pair_min_rest > 0 && k2 < la.min_n && k2 + kNb < max_n &&
        max_N - k2 - kNb >= la.pair_min_rest) {
      const int tiles2 = (max_N - k2 - 1 + kTile - 1) / kTile;
      const int split2 = k2 + kNb + kTcTileCols;
      PackB pk0;  // W(k): its columns right of block column k2 -> K half 0 of the pair's B operand
      pk0.hi = tc.b_hi;
      pk0.lo = tc.b_lo;
      pk0.slot = tc.b_slot;
      pk0.shift_k = k2;
      zgemm_tile_kernel<S, kOverwrite><<<dim3(tiles, 1, njobs), 256, smem_gemm, s>>>(jobs, k, tiles, 1, njobs, pk0, 0);
      // step k on block column k2, every row below step k (the diagonal block included)
      zgemm_tile_kernel<S, kSubtract><<<dim3(1, tiles, njobs), 256, smem_gemm, s>>>(jobs, k, 1, tiles, njobs,
                                                                                   PackB(), 0, 0);
      if ((e = launch_panel_select(fk, jobs, njobs, k2, max_n, s, launches)) != cudaSuccess) return e;
      if ((e = launch_row_moves(fk, jobs, njobs, k2, 0, max_N, max_N, s, launches)) != cudaSuccess) return e;
      // the inverse of the moved diagonal block beside step k's update of block row k2
      if ((e = cudaEventRecord(la.panel, s)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(la.s2, la.panel, 0)) != cudaSuccess) return e;
      launch_diag_inverse<T>(true, jobs, njobs, k2, info, smem_diag, la.s2);
      if ((e = cudaEventRecord(la.diag, la.s2)) != cudaSuccess) return e;
      if (tiles > 1)
        zgemm_tile_kernel<S, kSubtract><<<dim3(tiles - 1, 1, njobs), 256, smem_gemm, s>>>(jobs, k, tiles - 1, 1,
                                                                                         njobs, PackB(), 1, 0);
      if ((e = cudaStreamWaitEvent(s, la.diag, 0)) != cudaSuccess) return e;
      PackB pk1;  // W(k2) -> K half 1
      pk1.hi = tc.b_hi;
      pk1.lo = tc.b_lo;
      pk1.slot = tc.b_slot;
      pk1.k_off = 2 * kNb;
      zgemm_tile_kernel<S, kOverwrite><<<dim3(tiles2, 1, njobs), 256, smem_gemm, s>>>(jobs, k2, tiles2, 1, njobs,
                                                                                     pk1, 0);
      const bool timed = timer && timer->used + 2 <= timer->cap;
      if (timed) cudaEventRecord(timer->ev[timer->used++], s);
      if ((e = launch_tc_pack(tc, jobs, njobs, k, 2, k2, max_N, s, false)) != cudaSuccess) return e;
      if ((e = launch_tc_update(tc, jobs, njobs, k2, max_N, err, s, 3, 0, 2)) != cudaSuccess) return e;
      // the next step's selection, its moves left of the tiles still being updated, its inverse
      if ((e = cudaEventRecord(la.panel, s)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(la.s2, la.panel, 0)) != cudaSuccess) return e;
      if ((e = launch_panel_select(fk, jobs, njobs, k2 + kNb, max_n, la.s2, launches)) != cudaSuccess) return e;
      if ((e = launch_row_moves(fk, jobs, njobs, k2 + kNb, 0, split2, max_N, la.s2, launches)) != cudaSuccess)
        return e;
      launch_diag_inverse<T>(true, jobs, njobs, k2 + kNb, info, smem_diag, la.s2);
      if ((e = cudaEventRecord(la.diag, la.s2)) != cudaSuccess) return e;
      if ((e = launch_tc_update(tc, jobs, njobs, k2, max_N, err, s, 4, tc_num_sms() - free_sms, 2)) != cudaSuccess)
        return e;
      if (timed) cudaEventRecord(timer->ev[timer->used++], s);
      if ((e = cudaStreamWaitEvent(s, la.diag, 0)) != cudaSuccess) return e;
      if ((e = launch_row_moves(fk, jobs, njobs, k2 + kNb, split2, max_N, max_N, s, launches)) != cudaSuccess)
        return e;
      // W(k), the column strip, the row strip, k2's inverse, W(k2), the pack, the two update
      // launches, the next inverse (selections and moves count themselves)
      if (launches) *launches += 7 + (tiles > 1 ? 1 : 0);
      k = k2;  // the loop's increment moves past k2
      continue;
    }
    if (!panel && la.pair_min_rest > 0 && k2 < la.min_n && k2 + kNb < max_n &&
        max_N - k2 - kNb >= la.pair_min_rest) {
      const int tiles2 = (max_N - k2 - 1 + kTile - 1) / kTile;
      const bool next2 = k2 + kNb < max_n;
      PackB pk0;  // W(k): its columns right of block column k2 -> K half 0 of the pair's B operand
      pk0.hi = tc.b_hi;
      pk0.lo = tc.b_lo;
      pk0.slot = tc.b_slot;
      pk0.shift_k = k2;
      zgemm_tile_kernel<S, kOverwrite><<<dim3(tiles, 1, njobs), 256, smem_gemm, s>>>(jobs, k, tiles, 1, njobs, pk0, 0);
      // step k on block column k2 (all rows below step k) and on block row k2 (right of it): first
      // the diagonal block of k2, whose inverse then runs on the second stream beside the rest of
      // the two strips
      zgemm_tile_kernel<S, kSubtract><<<dim3(1, 1, njobs), 256, smem_gemm, s>>>(jobs, k, 1, 1, njobs, PackB(), 0, 0);
      if ((e = cudaEventRecord(la.panel, s)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(la.s2, la.panel, 0)) != cudaSuccess) return e;
      launch_diag_inverse<T>(false, jobs, njobs, k2, info, smem_diag, la.s2);
      if ((e = cudaEventRecord(la.diag, la.s2)) != cudaSuccess) return e;
      if (tiles > 1) zgemm_strips_kernel<S><<<dim3(2 * (tiles - 1), 1, njobs), 256, smem_gemm, s>>>(jobs, k, tiles - 1);
      if ((e = cudaStreamWaitEvent(s, la.diag, 0)) != cudaSuccess) return e;
      PackB pk1;  // W(k2) -> K half 1
      pk1.hi = tc.b_hi;
      pk1.lo = tc.b_lo;
      pk1.slot = tc.b_slot;
      pk1.k_off = 2 * kNb;
      zgemm_tile_kernel<S, kOverwrite><<<dim3(tiles2, 1, njobs), 256, smem_gemm, s>>>(jobs, k2, tiles2, 1, njobs,
                                                                                     pk1, 0);
      const bool timed = timer && timer->used + 2 <= timer->cap;
      if (timed) cudaEventRecord(timer->ev[timer->used++], s);
      if ((e = launch_tc_pack(tc, jobs, njobs, k, 2, k2, max_N, s, false)) != cudaSuccess) return e;
      if ((e = launch_tc_update(tc, jobs, njobs, k2, max_N, err, s, 1, 0, 2)) != cudaSuccess) return e;
      if (next2) {
        if ((e = cudaEventRecord(la.panel, s)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(la.s2, la.panel, 0)) != cudaSuccess) return e;
        launch_diag_inverse<T>(false, jobs, njobs, k2 + kNb, info, smem_diag, la.s2);
        if ((e = cudaEventRecord(la.diag, la.s2)) != cudaSuccess) return e;
      }
      if ((e = launch_tc_update(tc, jobs, njobs, k2, max_N, err, s, 2, next2 ? tc_num_sms() - free_sms : 0, 2)) !=
          cudaSuccess)
        return e;
      if (timed) cudaEventRecord(timer->ev[timer->used++], s);
      if (next2 && (e = cudaStreamWaitEvent(s, la.diag, 0)) != cudaSuccess) return e;
      // W(k), the diagonal block, its inverse, W(k2), the pack, the two update launches (+ the
      // two strips in one launch, + the next inverse)
      if (launches) *launches += 7 + (tiles > 1 ? 1 : 0) + (next2 ? 1 : 0);
      k = k2;  // the loop's increment moves past k2
      continue;
    }
    if (tiles > 0) {
      PackB pk;
      pk.hi = tc.b_hi;
      pk.lo = tc.b_lo;
      pk.slot = tc.b_slot;
      zgemm_tile_kernel<S, kOverwrite><<<dim3(tiles, 1, njobs), 256, smem_gemm, s>>>(jobs, k, tiles, 1, njobs, pk, 0);
      const bool timed = timer && timer->used + 2 <= timer->cap;
      if (timed) cudaEventRecord(timer->ev[timer->used++], s);
      if ((e = launch_tc_pack(tc, jobs, njobs, k, 1, k, max_N, s, false)) != cudaSuccess) return e;
      if ((e = launch_tc_update(tc, jobs, njobs, k, max_N, err, s, panel ? 3 : 1, 0)) != cudaSuccess) return e;
      // the next step's columns left of the tiles still being updated: [0, k + 64 + one tile)
      const int split = k + kNb + kTcTileCols;
      if (next) {
        if ((e = cudaEventRecord(la.panel, s)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(la.s2, la.panel, 0)) != cudaSuccess) return e;
        if (panel) {
          if ((e = launch_panel_select(fk, jobs, njobs, k + kNb, max_n, la.s2, launches)) != cudaSuccess) return e;
          if ((e = launch_row_moves(fk, jobs, njobs, k + kNb, 0, split, max_N, la.s2, launches)) != cudaSuccess)
            return e;
        }
        launch_diag_inverse<T>(panel, jobs, njobs, k + kNb, info, smem_diag, la.s2);
        if ((e = cudaEventRecord(la.diag, la.s2)) != cudaSuccess) return e;
      }
      if ((e = launch_tc_update(tc, jobs, njobs, k, max_N, err, s, panel ? 4 : 2,
                                next ? tc_num_sms() - free_sms : 0)) != cudaSuccess)
        return e;
      if (timed) cudaEventRecord(timer->ev[timer->used++], s);  // the update kernels only
      if (next && (e = cudaStreamWaitEvent(s, la.diag, 0)) != cudaSuccess) return e;
      if (next && panel && (e = launch_row_moves(fk, jobs, njobs, k + kNb, split, max_N, max_N, s, launches)) !=
                               cudaSuccess)
        return e;
      if (launches) *launches += next ? 5 : 4;
    } else if (next) {
      if (panel) {
        if ((e = launch_panel_select(fk, jobs, njobs, k + kNb, max_n, s, launches)) != cudaSuccess) return e;
        if ((e = launch_row_moves(fk, jobs, njobs, k + kNb, 0, max_N, max_N, s, launches)) != cudaSuccess) return e;
      }
      launch_diag_inverse<T>(panel, jobs, njobs, k + kNb, info, smem_diag, s);
      if (launches) *launches += 1;
    }
  }
  if (panel && (e = launch_pivot_finish(jobs, njobs, s, launches)) != cudaSuccess) return e;
  return cudaGetLastError();
}

template <typename T, typename S>
cudaError_t eliminate_impl(const JobDev *jobs, int njobs, int max_n, int max_N, int *info, cudaStream_t s,
                           long *launches, KernelTimer *timer, const TcMaps *tc, int *err, bool sparse_jobs,
                           const Lookahead *la, bool panel) {
  const FactorKind fk = sizeof(T) == sizeof(double2) ? kFactorFP64 : kFactorFP32;
  const int smem_diag = kNb * (kNb + 1) * (int)sizeof(double2);
  const int smem_gemm = 4 * kKc * kTile * (int)sizeof(T);
  cudaError_t e;
  if ((e = ensure_smem(diag_inverse_kernel<T, 1>, smem_diag)) != cudaSuccess)
    return e;
  if ((e = ensure_smem(diag_inverse_kernel<T, 2>, smem_diag)) != cudaSuccess)
    return e;
  if ((e = ensure_smem(zgemm_tile_kernel<S, kOverwrite>, smem_gemm)) != cudaSuccess)
    return e;
  if ((e = ensure_smem(zgemm_tile_kernel<S, kSubtract>, smem_gemm)) != cudaSuccess)
    return e;
  if ((e = ensure_smem(zgemm_strips_kernel<S>, smem_gemm)) != cudaSuccess)
    return e;
  // Look-ahead (tensor-core path): the update of step k first covers the tile holding the next
  // step's diagonal block; the next diagonal inverse then runs on the second stream while the other
  // tiles are updated on SMs left free for it (the inverses take one SM per job).
  if (tc != nullptr && la != nullptr && la->s2 != nullptr && !sparse_jobs)
    return eliminate_lookahead<T, S>(jobs, njobs, max_n, max_N, info, s, launches, timer, *tc, err, *la, smem_diag,
                                     smem_gemm, panel);
  if (panel && (e = launch_pivot_init(jobs, njobs, s, launches)) != cudaSuccess) return e;
  for (int k = 0; k < max_n; k += kNb) {
    if (panel) {
      if ((e = launch_panel_select(fk, jobs, njobs, k, max_n, s, launches)) != cudaSuccess) return e;
      if ((e = launch_row_moves(fk, jobs, njobs, k, 0, max_N, max_N, s, launches)) != cudaSuccess) return e;
    }
    launch_diag_inverse<T>(panel, jobs, njobs, k, info, smem_diag, s);
    const int rest = max_N - k - 1;
    const int tiles = (rest + kTile - 1) / kTile;
    if (launches) *launches += 1;
    if (tiles > 0) {
      zgemm_tile_kernel<S, kOverwrite><<<dim3(tiles, 1, njobs), 256, smem_gemm, s>>>(jobs, k, tiles, 1, njobs,
                                                                                   PackB(), 0);
      const bool timed = timer && timer->used + 2 <= timer->cap;
      if (timed) cudaEventRecord(timer->ev[timer->used++], s);
      if (tc != nullptr) {
        if ((e = launch_tc_step(*tc, jobs, njobs, k, max_N, err, s)) != cudaSuccess) return e;
        if (launches) *launches += 1;  // pack + update
      } else {
        if (sparse_jobs)
          zgemm_tile_kernel<S, kSubtract><<<std::min(tiles * tiles * njobs, kSparseGrid), 256, smem_gemm, s>>>(
              jobs, k, tiles, tiles, njobs, PackB(), 0);
        else
          zgemm_tile_kernel<S, kSubtract><<<dim3(tiles, tiles, njobs), 256, smem_gemm, s>>>(jobs, k, tiles, tiles,
                                                                                           njobs, PackB(), 0);
      }
      if (timed) cudaEventRecord(timer->ev[timer->used++], s);
      if (launches) *launches += 2;
    }
  }
  if (panel && (e = launch_pivot_finish(jobs, njobs, s, launches)) != cudaSuccess) return e;
  return cudaGetLastError();
}

template <typename T>
cudaError_t sweep_solve(const JobDev *jobs, int njobs, int b, int max_N, int mode, int *info, cudaStream_t s,
                        long *launches, bool fp32, const CUtensorMap *fmap, int active_hint = 0) {
  const FactorKind fk = sizeof(T) == sizeof(double2) ? kFactorFP64 : kFactorFP32;
  cudaError_t e;
  // forward (skipped for the initial solve: B is zero above the central block)
  if (mode == 1) {
    if ((e = launch_sweep(fk, jobs, njobs, b, max_N, true, mode, fp32, fmap, s, active_hint)) != cudaSuccess)
      return e;
    if (launches) *launches += 1;
  }
  schur_solve_kernel<T><<<njobs, 256, 0, s>>>(jobs, mode, info);
  if ((e = launch_sweep(fk, jobs, njobs, b, max_N, false, mode, fp32, fmap, s, active_hint)) != cudaSuccess)
    return e;
  if (launches) *launches += 2;
  return cudaSuccess;
}

// After a refinement round: c = max|correction| / max|tau00| on the tau00 block.  A job whose
// correction stops shrinking (c >= c_prev) is marked kDiverged and skipped from then on; the
// host re-solves such jobs, and those not converged after the last round, by FP64 block LU.  The error left
// after applying the correction is about c times the contraction factor of the refinement,
// estimated as c / c_prev from the previous round; the job is converged when c * min(1, c / c_prev)
// is below tol, and later rounds skip it.
__global__ void __launch_bounds__(256) converge_check_kernel(const JobDev *__restrict__ jobs, double tol) {
  const JobDev &J = jobs[blockIdx.x];
  if (J.conv == nullptr || converged(J) || J.inactive) return;
  const int b = J.b, n = J.n, ld = J.ld;
  double my = 0.0, mx = 0.0;
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int r = e % b, c = e / b;
    const size_t idx = (size_t)(n + r) + (size_t)c * ld;
    my = fmax(my, cabs1(J.Y[idx]));
    mx = fmax(mx, cabs1(J.X[idx]));
  }
  __shared__ double sy[256], sx[256];
  sy[threadIdx.x] = my;
  sx[threadIdx.x] = mx;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      sy[threadIdx.x] = fmax(sy[threadIdx.x], sy[threadIdx.x + o]);
      sx[threadIdx.x] = fmax(sx[threadIdx.x], sx[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double c = sx[0] > 0.0 ? sy[0] / sx[0] : 0.0;
    const double prev = J.cnorm ? *J.cnorm : 0.0;
    const double est = prev > 0.0 ? c * fmin(1.0, c / prev) : c;
    if (est <= tol) *J.conv = kConverged;
    else if (prev > 0.0 && c >= prev) *J.conv = kDiverged;  // no contraction: stop refining
    if (J.cnorm) *J.cnorm = c;
  }
}

template <typename T>
__global__ void copy_to_factor_kernel(const double2 *__restrict__ M, T *__restrict__ F, int n, int ld) {
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const size_t c = e / n, r = e - c * n;
    stc(F + r + c * ld, M[r + c * ld]);
  }
}

// The FP64 re-solve records of a mixed wave (launch_fallback_prepare).
__global__ void fallback_prepare_kernel(const JobDev *__restrict__ jobs, JobDev *__restrict__ out, int njobs,
                                        double2 *f64, size_t f64_stride, int *count, int panel) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= njobs) return;
  JobDev J = jobs[w];
  const bool conv = J.conv != nullptr && *J.conv == kConverged;
  if (conv) {
    J.inactive = 1;
  } else {
    J.F = f64 + (size_t)w * f64_stride;
    J.conv = nullptr;  // the FP64 rounds run unconditionally
    J.cnorm = nullptr;
    if (!panel) J.piv = nullptr;  // pivots inside the diagonal blocks: rows stay in place
    atomicAdd(count, 1);
  }
  out[w] = J;
}

// The re-solve gate of a mixed wave: the graph's conditional body (the FP64 re-solve) runs only
// when some record has not converged.
__global__ void fallback_gate_kernel(const JobDev *__restrict__ jobs, int njobs, cudaGraphConditionalHandle h) {
  int any = 0;
  for (int w = threadIdx.x; w < njobs; w += blockDim.x) {
    const int *c = jobs[w].conv;
    any |= (c == nullptr || *c != kConverged) ? 1 : 0;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

// F = M (FP64, N x N) for the active records; CTAs (blockIdx.x) stride over the columns of job
// blockIdx.y
__global__ void __launch_bounds__(256) copy_jobs_to_factor_kernel(const JobDev *__restrict__ jobs) {
  const JobDev &J = jobs[blockIdx.y];
  if (J.inactive) return;
  double2 *F = static_cast<double2 *>(J.F);
  for (int c = blockIdx.x; c < J.N; c += gridDim.x)
    for (int r = threadIdx.x; r < J.N; r += 256) F[(size_t)r + (size_t)c * J.ld] = J.M[(size_t)r + (size_t)c * J.ld];
}

}  // namespace

cudaError_t launch_fallback_prepare(const JobDev *jobs, JobDev *out, int njobs, double2 *f64, size_t f64_stride,
                                    int max_N, int *count, bool panel, cudaStream_t s, long *launches) {
  if (njobs <= 0) return cudaSuccess;
  fallback_prepare_kernel<<<(njobs + 63) / 64, 64, 0, s>>>(jobs, out, njobs, f64, f64_stride, count, panel ? 1 : 0);
  copy_jobs_to_factor_kernel<<<dim3(std::min(max_N, 64), njobs), 256, 0, s>>>(out);
  if (launches) *launches += 2;
  return cudaGetLastError();
}

cudaError_t add_fallback_gate_node(cudaGraph_t g, cudaGraphNode_t *node, const JobDev *jobs, int njobs,
                                   cudaGraphConditionalHandle h) {
  cudaKernelNodeParams kp = {};
  void *args[3] = {&jobs, &njobs, &h};
  kp.func = reinterpret_cast<void *>(fallback_gate_kernel);
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(256);
  kp.sharedMemBytes = 0;
  kp.kernelParams = args;
  return cudaGraphAddKernelNode(node, g, nullptr, 0, &kp);
}

cudaError_t launch_copy_to_factor(FactorKind fk, const double2 *M, void *F, int n, int ld, cudaStream_t s) {
  const int blocks = 148 * 8;
  if (fk == kFactorFP64)
    copy_to_factor_kernel<double2><<<blocks, 256, 0, s>>>(M, static_cast<double2 *>(F), n, ld);
  else
    copy_to_factor_kernel<float2><<<blocks, 256, 0, s>>>(M, static_cast<float2 *>(F), n, ld);
  return cudaGetLastError();
}

cudaError_t launch_eliminate(FactorKind fk, const JobDev *jobs, int njobs, int max_n, int max_N, int *info,
                             cudaStream_t s, long *launches, KernelTimer *timer, const TcMaps *tc,
                             int *err, bool sparse_jobs, const Lookahead *la, bool panel) {
  if (fk == kFactorFP64)
    return eliminate_impl<double2, double>(jobs, njobs, max_n, max_N, info, s, launches, timer, nullptr, err,
                                           sparse_jobs, nullptr, panel);
  if (tc) {
    cudaError_t e = tc_prepare();
    if (e == cudaSuccess) e = launch_tc_counters_reset(*tc, s);
    if (e != cudaSuccess) return e;
  }
  return eliminate_impl<float2, float>(jobs, njobs, max_n, max_N, info, s, launches, timer, tc, err, sparse_jobs,
                                       la, panel);
}

cudaError_t launch_finalize_direct(FactorKind fk, const JobDev *jobs, int njobs, int ns, int kkrsz, int *info,
                                   cudaStream_t s, long *launches) {
  if (fk == kFactorFP64)
    finalize_direct_kernel<double2><<<njobs, 256, 0, s>>>(jobs, ns, kkrsz, info);
  else
    finalize_direct_kernel<float2><<<njobs, 256, 0, s>>>(jobs, ns, kkrsz, info);
  if (launches) *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_refine_begin(FactorKind fk, const JobDev *jobs, int njobs, int max_n, int max_N, int b,
                                int *info, cudaStream_t s, long *launches, bool fp32_sweep,
                                const CUtensorMap *fmap) {
  (void)max_n;
  const cudaError_t e = fk == kFactorFP64 ? sweep_solve<double2>(jobs, njobs, b, max_N, 0, info, s, launches, false, nullptr)
                                           : sweep_solve<float2>(jobs, njobs, b, max_N, 0, info, s, launches, fp32_sweep, fmap);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <int BC>
cudaError_t launch_residual(const JobDev *jobs, int njobs, int max_N, int *active, cudaStream_t s) {
  constexpr int sm = residual_smem_bytes<BC>();
  const cudaError_t e = ensure_smem(residual_kernel<BC>, sm);
  if (e != cudaSuccess) return e;
  const int rowblocks = (max_N + residual_rows<BC>() - 1) / residual_rows<BC>();
  if (active) {
    active_list_kernel<<<1, 32, 0, s>>>(jobs, njobs, active);
    residual_kernel<BC><<<njobs * rowblocks, kResThreads, sm, s>>>(jobs, active, rowblocks);
  } else {
    residual_kernel<BC><<<dim3(njobs, rowblocks), kResThreads, sm, s>>>(jobs, nullptr, rowblocks);
  }
  return cudaGetLastError();
}

cudaError_t launch_refine_round(FactorKind fk, const JobDev *jobs, int njobs, int max_n, int max_N, int b,
                                bool check, int *info, cudaStream_t s, long *launches, bool fp32_sweep,
                                const CUtensorMap *fmap, int active_hint, int *active) {
  (void)max_n;
  const cudaError_t e0 = b <= 16 ? launch_residual<16>(jobs, njobs, max_N, active, s)
                                 : launch_residual<32>(jobs, njobs, max_N, active, s);
  if (e0 != cudaSuccess) return e0;
  if (launches) *launches += active ? 2 : 1;
  const cudaError_t e = fk == kFactorFP64 ? sweep_solve<double2>(jobs, njobs, b, max_N, 1, info, s, launches, false, nullptr)
                                           : sweep_solve<float2>(jobs, njobs, b, max_N, 1, info, s, launches, fp32_sweep, fmap,
                                                                 active_hint);
  if (e != cudaSuccess) return e;
  if (check) {
    converge_check_kernel<<<njobs, 256, 0, s>>>(jobs, kRefineTol);
    if (launches) *launches += 1;
  }
  return cudaGetLastError();
}

cudaError_t launch_refine_end(const JobDev *jobs, int njobs, int ns, int kkrsz, cudaStream_t s, long *launches) {
  finalize_from_x_kernel<<<njobs, 256, 0, s>>>(jobs, ns, kkrsz);
  if (launches) *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_solve_refine(FactorKind fk, const JobDev *jobs, int njobs, int max_n, int max_N, int b,
                                int steps, int ns, int kkrsz, int *info, cudaStream_t s, long *launches,
                                bool fp32_sweep, const CUtensorMap *fmap) {
  cudaError_t e = launch_refine_begin(fk, jobs, njobs, max_n, max_N, b, info, s, launches, fp32_sweep, fmap);
  for (int it = 0; it < steps && e == cudaSuccess; ++it)
    e = launch_refine_round(fk, jobs, njobs, max_n, max_N, b, it + 1 < steps, info, s, launches, fp32_sweep,
                            fmap);
  if (e != cudaSuccess) return e;
  return launch_refine_end(jobs, njobs, ns, kkrsz, s, launches);
}

}  // namespace b200
