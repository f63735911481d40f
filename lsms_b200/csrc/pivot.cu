// Panel pivoting of the block elimination: each 64-column step picks its diagonal-block rows from
// the whole remaining column, not from the 64 x 64 diagonal block alone.
//
// The reference's CPU solver pivots with LAPACK's zgetrf inside each of its nblk diagonal blocks
// of ~N/3 rows (zblock_lu_cpp.cpp:58, nblk = 3 at linearSolvers_CPU.cpp:270); its zgesv path
// (linearSolvers_CPU.cpp:76-96) pivots over the whole column.  Restricting the pivots of a 64-column
// step to its own diagonal block is enough for the collinear contour matrices, but the
// non-collinear N = 4320 matrices (condition numbers up to ~1e7) then lose most of the FP32
// factorisation's accuracy and the mixed refinement stalls.  Here step k's rows come from every
// candidate row [k, n), in two launches:
//   magnitudes  every row below the diagonal block gets max_j |re| + |im| over the panel columns
//               k..k+kb-1 (one thread per row, coalesced over the column-major panel);
//   selection   one CTA per job: the kPivCands - kb rows of largest magnitude (a radix select on
//               the float bits, compacted in row order, so the choice is deterministic) join the
//               kb rows of the diagonal block, and Gaussian elimination with partial pivoting
//               (GEPP) on these candidates' panel rows picks the kb pivot rows in pivot order.
// That is the node of communication-avoiding "tournament pivoting" with a magnitude filter in
// front: a row that is small in every panel column is not a candidate.  On the non-collinear
// N = 4320 matrices a numpy emulation of the whole mixed solve gives the first refinement round an
// error of 1.6e-3 .. 1e-2 with it, 1.6e-3 .. 5e-3 with a full tournament over all rows and
// 5e-3 .. 9e-2 with the pivots restricted to the diagonal block.
// The kb rows then move to positions k..k+kb-1 (the rows displaced from there take the vacated
// positions): a permutation of at most 2 kb rows, applied to every column of F, so the factor
// storage is that of LAPACK's P M = L U and the kernels of the elimination and of the sweeps run
// unchanged.  The permutation of the whole elimination is tracked per job (perm), and its inverse
// (rowpos) makes the refinement's residual land in the permuted row order.  Pivots come only from
// rows [k, n), never from the central site's rows, so the trailing b x b block still holds the
// Schur complement 1 - Delta.
//
// Selection arithmetic is FP32 on either factor type (it only ranks pivot magnitudes, |re| + |im|
// as izamax, ties to the earlier candidate); the factorisation itself is unchanged.

#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"

namespace b200 {
namespace {

constexpr int kSelThreads = 1024;                  // (candidate, 16-column group) per thread
constexpr int kGroups = kSelThreads / kPivCands;   // column groups of the panel
constexpr int kGroupCols = kNb / kGroups;          // 16
static_assert(kGroups * kGroupCols == kNb, "selection thread layout");

__device__ __forceinline__ float2 to_f2(double2 a) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ float2 to_f2(float2 a) { return a; }
__device__ __forceinline__ float cabs1f(float2 a) { return fabsf(a.x) + fabsf(a.y); }

// Row magnitudes below the diagonal block of step k: mags[row] = max_j |F[row, k + j]|_1 over the
// kb panel columns, as float bits (a NaN ranks as zero).
template <typename T>
__global__ void __launch_bounds__(256) panel_mags_kernel(const JobDev *__restrict__ jobs, int k) {
  const JobDev &J = jobs[blockIdx.y];
  if (J.inactive || J.piv == nullptr || k >= J.n) return;
  const int kb = min(kNb, J.n - k);
  const int row = k + kb + blockIdx.x * 256 + threadIdx.x;
  if (row >= J.n) return;
  const T *__restrict__ F = static_cast<const T *>(J.F);
  float m = 0.f;
  for (int j = 0; j < kb; ++j) {
    const float v = cabs1f(to_f2(F[(size_t)row + (size_t)(k + j) * J.ld]));
    m = v > m ? v : m;  // (a NaN compares false)
  }
  J.piv[pivot_mags_offset(J.ld) + row] = __float_as_int(m);
}

// Block-wide exclusive prefix sum of one int per thread (kSelThreads threads); returns the total.
__device__ __forceinline__ int block_scan(int v, int *s_warp, int &excl) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = s_warp[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    s_warp[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  const int total = s_warp[31];
  excl = (warp > 0 ? s_warp[warp - 1] : 0) + x - v;
  __syncthreads();  // s_warp is reused by the next scan
  return total;
}

// Step k's selection, one CTA per job (see the file comment); the kb pivot rows in pivot order
// become the step's row moves, also applied to the job's permutation.
template <typename T>
__global__ void __launch_bounds__(kSelThreads) panel_select_kernel(const JobDev *__restrict__ jobs, int k) {
  const JobDev &J = jobs[blockIdx.x];
  if (J.inactive || J.piv == nullptr || k >= J.n) return;
  const int kb = min(kNb, J.n - k);
  const int n = J.n, ld = J.ld;
  int *__restrict__ piv = J.piv;
  const unsigned *__restrict__ mags = reinterpret_cast<const unsigned *>(piv + pivot_mags_offset(ld));
  extern __shared__ __align__(16) unsigned char sel_smem[];
  float2(*A)[kPivCands] = reinterpret_cast<float2(*)[kPivCands]>(sel_smem);  // A[col][cand]
  __shared__ int s_cand[kPivCands];
  __shared__ int s_out[kNb];
  __shared__ int s_hist[256];
  __shared__ int s_warp[32];
  __shared__ unsigned s_prefix;
  __shared__ int s_remain;
  __shared__ float s_wv[2][kPivCands / 32];
  __shared__ int s_wi[2][kPivCands / 32];
  const int tid = threadIdx.x;

  // --- candidates: the diagonal block's rows, then the largest rows below it ---
  const int lo = k + kb, m2 = n - lo;  // rows below the diagonal block
  const int K2 = min(m2, kPivCands - kb);
  if (tid < kb) s_cand[tid] = k + tid;
  if (K2 == m2) {
    for (int i = tid; i < m2; i += kSelThreads) s_cand[kb + i] = lo + i;
  } else {
    // radix select (8 bits at a time, most significant first) of the K2-th largest key
    unsigned prefix = 0u, mask = 0u;
    int remain = K2;
    for (int shift = 24; shift >= 0; shift -= 8) {
      if (tid < 256) s_hist[tid] = 0;
      __syncthreads();
      for (int i = tid; i < m2; i += kSelThreads) {
        const unsigned key = mags[lo + i];
        if ((key & mask) == prefix) atomicAdd(&s_hist[(key >> shift) & 255u], 1);
      }
      __syncthreads();
      if (tid == 0) {
        int cum = 0, d = 0;
        for (d = 255; d > 0; --d) {
          if (cum + s_hist[d] >= remain) break;
          cum += s_hist[d];
        }
        s_prefix = prefix | ((unsigned)d << shift);
        s_remain = remain - cum;
      }
      __syncthreads();
      prefix = s_prefix;
      remain = s_remain;
      mask |= 255u << shift;
      __syncthreads();
    }
    // keys above the threshold, then `remain` of the keys equal to it, each in row order
    const int chunk = (m2 + kSelThreads - 1) / kSelThreads;
    const int r0 = min(m2, tid * chunk), r1 = min(m2, r0 + chunk);
    int ngt = 0, neq = 0;
    for (int i = r0; i < r1; ++i) {
      const unsigned key = mags[lo + i];
      ngt += key > prefix;
      neq += key == prefix;
    }
    int bgt = 0, beq = 0;
    const int tgt = block_scan(ngt, s_warp, bgt);
    block_scan(neq, s_warp, beq);
    for (int i = r0; i < r1; ++i) {
      const unsigned key = mags[lo + i];
      if (key > prefix) {
        s_cand[kb + bgt++] = lo + i;
      } else if (key == prefix) {
        if (beq < remain) s_cand[kb + tgt + beq] = lo + i;
        ++beq;
      }
    }
  }
  __syncthreads();
  const int R = kb + K2;  // candidates

  // --- GEPP on the candidates' panel rows ---
  if (R <= kb) {  // the last step: the block's own rows, in place
    if (tid < kb) s_out[tid] = k + tid;
    __syncthreads();
  } else {
    const T *__restrict__ F = static_cast<const T *>(J.F);
    const int r = tid & (kPivCands - 1), g = tid / kPivCands, c0 = g * kGroupCols;
    const int cand = r < R ? s_cand[r] : -1;
    for (int j = c0; j < c0 + kGroupCols; ++j)
      A[j][r] = (cand >= 0 && j < kb) ? to_f2(F[(size_t)cand + (size_t)(k + j) * ld]) : make_float2(0.f, 0.f);
    __syncthreads();
    bool taken = false;
    for (int p = 0; p < kb; ++p) {
      const int par = p & 1, gp = p / kGroupCols;
      if (g == gp) {  // the threads holding column p rank their rows: warp arg-max, ties low
        float v = -1.f;
        if (cand >= 0 && !taken) {
          v = cabs1f(A[p][r]);
          if (!(v == v)) v = 0.f;  // a NaN ranks as zero, so a row in range is still chosen
        }
        int idx = r;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const float ov = __shfl_xor_sync(0xffffffffu, v, o);
          const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
          if (ov > v || (ov == v && oi < idx)) {
            v = ov;
            idx = oi;
          }
        }
        if ((tid & 31) == 0) {
          s_wv[par][r >> 5] = v;
          s_wi[par][r >> 5] = idx;
        }
      }
      __syncthreads();
      float bv = s_wv[par][0];
      int bi = s_wi[par][0];
#pragma unroll
      for (int w = 1; w < kPivCands / 32; ++w) {
        const float ov = s_wv[par][w];
        const int oi = s_wi[par][w];
        if (ov > bv || (ov == bv && oi < bi)) {
          bv = ov;
          bi = oi;
        }
      }
      // R > kb > p candidates remain untaken, each ranked >= 0: bi is one of them
      if (r == bi) taken = true;
      if (tid == 0) s_out[p] = s_cand[bi];
      const int jlo = max(p + 1, c0), jhi = min(kb, c0 + kGroupCols);
      if (cand >= 0 && !taken && jlo < jhi) {
        const float2 d = A[p][bi];
        const float dd = d.x * d.x + d.y * d.y;
        float2 f = make_float2(0.f, 0.f);
        if (dd > 0.f) {
          const float2 a = A[p][r];
          f = make_float2((a.x * d.x + a.y * d.y) / dd, (a.y * d.x - a.x * d.y) / dd);
        }
        for (int j = jlo; j < jhi; ++j) {
          const float2 pj = A[j][bi];
          float2 x = A[j][r];
          x.x -= f.x * pj.x - f.y * pj.y;
          x.y -= f.x * pj.y + f.y * pj.x;
          A[j][r] = x;
        }
      }
      __syncthreads();
    }
  }
  if (tid != 0) return;
  // the moves that bring the pivot rows to k..k+kb-1 (pivot order) and the displaced rows to the
  // vacated positions; a permutation of at most 2 kb positions, also applied to perm
  int *mv = piv + pivot_moves_offset(ld);
  int *dst = mv + 1, *src = mv + 1 + 2 * kNb;
  // kb distinct rows in [k, n) by construction; anything else leaves the rows in place
  for (int p = 0; p < kb; ++p)
    if (s_out[p] < k || s_out[p] >= n) {
      mv[0] = 0;
      return;
    }
  int cnt = 0;
  unsigned long long in_s = 0ull;
  for (int p = 0; p < kb; ++p)
    if (s_out[p] - k < kb) in_s |= 1ull << (s_out[p] - k);
  for (int i = 0; i < kb; ++i)
    if (s_out[i] != k + i) {
      dst[cnt] = k + i;
      src[cnt] = s_out[i];
      ++cnt;
    }
  int vj = 0;
  for (int i = 0; i < kb; ++i)
    if (!((in_s >> i) & 1ull)) {
      while (vj < kb && s_out[vj] < k + kb) ++vj;  // the next vacated position, in pivot order
      if (vj == kb) break;  // (as many vacated positions as displaced rows: not reached)
      dst[cnt] = s_out[vj];
      src[cnt] = k + i;
      ++cnt;
      ++vj;
    }
  mv[0] = cnt;
  int old[2 * kNb];
  for (int c = 0; c < cnt; ++c) old[c] = piv[src[c]];
  for (int c = 0; c < cnt; ++c) piv[dst[c]] = old[c];
}

// The step's row moves applied to columns [c0, c1) of F: one warp per column reads every moved
// element, then writes it at its destination.
template <typename T>
__global__ void __launch_bounds__(256) row_move_kernel(const JobDev *__restrict__ jobs, int k, int c0, int c1) {
  const JobDev &J = jobs[blockIdx.y];
  if (J.inactive || J.piv == nullptr || k >= J.n) return;
  const int *__restrict__ mv = J.piv + pivot_moves_offset(J.ld);
  const int cnt = mv[0];
  if (cnt == 0) return;
  const int hi = min(c1, J.N);
  T *__restrict__ F = static_cast<T *>(J.F);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  int dst[4], src[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = lane + 32 * q;
    dst[q] = i < cnt ? mv[1 + i] : -1;
    src[q] = i < cnt ? mv[1 + 2 * kNb + i] : -1;
  }
  for (int c = c0 + blockIdx.x * nw + warp; c < hi; c += gridDim.x * nw) {
    T *col = F + (size_t)c * J.ld;
    T v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (src[q] >= 0) v[q] = col[src[q]];
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (dst[q] >= 0) col[dst[q]] = v[q];
    __syncwarp();
  }
}

__global__ void pivot_init_kernel(const JobDev *__restrict__ jobs) {
  const JobDev &J = jobs[blockIdx.x];
  if (J.inactive || J.piv == nullptr) return;
  for (int p = threadIdx.x; p < J.N; p += blockDim.x) J.piv[p] = p;
  if (threadIdx.x == 0) J.piv[pivot_moves_offset(J.ld)] = 0;
}

// rowpos: the physical row of every original row once the elimination is done.
__global__ void pivot_finish_kernel(const JobDev *__restrict__ jobs) {
  const JobDev &J = jobs[blockIdx.x];
  if (J.inactive || J.piv == nullptr) return;
  int *rowpos = J.piv + J.ld;
  for (int p = threadIdx.x; p < J.N; p += blockDim.x) rowpos[J.piv[p]] = p;
}

template <typename T>
cudaError_t select_impl(const JobDev *jobs, int njobs, int k, int max_n, cudaStream_t s, long *launches) {
  if (max_n - k <= 0) return cudaSuccess;
  const int m = max_n - k - kNb;  // rows below the diagonal block, at most
  const int smem = kNb * kPivCands * (int)sizeof(float2);
  cudaError_t e = ensure_smem(panel_select_kernel<T>, smem);
  if (e != cudaSuccess) return e;
  if (m > kPivCands - kNb) {  // magnitudes are ranked only when the candidates must be filtered
    panel_mags_kernel<T><<<dim3((m + 255) / 256, njobs), 256, 0, s>>>(jobs, k);
    if (launches) *launches += 1;
  }
  panel_select_kernel<T><<<njobs, kSelThreads, smem, s>>>(jobs, k);
  if (launches) *launches += 1;
  return cudaGetLastError();
}

template <typename T>
cudaError_t move_impl(const JobDev *jobs, int njobs, int k, int c0, int c1, int max_N, cudaStream_t s,
                      long *launches) {
  const int hi = std::min(c1, max_N);
  if (hi <= c0) return cudaSuccess;
  const int cols = hi - c0;
  const int per_cta = 8 * 4;  // 8 warps, 4 columns each
  const int grid = std::max(1, std::min((cols + per_cta - 1) / per_cta, 4 * 148 / std::max(1, njobs) + 1));
  row_move_kernel<T><<<dim3(grid, njobs), 256, 0, s>>>(jobs, k, c0, c1);
  if (launches) *launches += 1;
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_pivot_init(const JobDev *jobs, int njobs, cudaStream_t s, long *launches) {
  pivot_init_kernel<<<njobs, 256, 0, s>>>(jobs);
  if (launches) *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_panel_select(FactorKind fk, const JobDev *jobs, int njobs, int k, int max_n, cudaStream_t s,
                                long *launches) {
  return fk == kFactorFP64 ? select_impl<double2>(jobs, njobs, k, max_n, s, launches)
                           : select_impl<float2>(jobs, njobs, k, max_n, s, launches);
}

cudaError_t launch_row_moves(FactorKind fk, const JobDev *jobs, int njobs, int k, int c0, int c1, int max_N,
                             cudaStream_t s, long *launches) {
  return fk == kFactorFP64 ? move_impl<double2>(jobs, njobs, k, c0, c1, max_N, s, launches)
                           : move_impl<float2>(jobs, njobs, k, c0, c1, max_N, s, launches);
}

cudaError_t launch_pivot_finish(const JobDev *jobs, int njobs, cudaStream_t s, long *launches) {
  pivot_finish_kernel<<<njobs, 256, 0, s>>>(jobs);
  if (launches) *launches += 1;
  return cudaGetLastError();
}

}  // namespace b200
