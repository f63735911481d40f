// Panel pivoting of the block elimination: each 64-column step picks its diagonal-block rows from
// the whole remaining column, not from the 64 x 64 diagonal block alone.
//
// The reference's CPU solver pivots with LAPACK's zgetrf inside each of its nblk diagonal blocks
// of ~N/3 rows (zblock_lu_cpp.cpp:58, nblk = 3 at linearSolvers_CPU.cpp:270); its zgesv path
// (linearSolvers_CPU.cpp:76-96) pivots over the whole column.  Restricting the pivots of a 64-column
// step to its own diagonal block is enough for the collinear contour matrices, but the
// non-collinear N = 4320 matrices (condition numbers up to ~1e7) then lose most of the FP32
// factorisation's accuracy and the mixed refinement stalls.  Here the rows of step k come from a
// tournament over every candidate row [k, n) (communication-avoiding "tournament pivoting"):
//   leaves    every 256 candidate rows of the panel columns k..k+kb-1 run Gaussian elimination
//             with partial pivoting (GEPP) and nominate the kb rows it pivots on;
//   merges    the nominees of 4 nodes run GEPP again on their panel rows (re-read from F) and
//             nominate kb of them; repeated until one node is left.
// The root's kb rows then move to positions k..k+kb-1 (the rows displaced from there take the
// vacated positions): a permutation of at most 2 kb rows, applied to every column of F, so the
// factor storage is that of LAPACK's P M = L U and the kernels of the elimination and of the
// sweeps run unchanged.  The permutation of the whole elimination is tracked per job (perm), and
// its inverse (rowpos) makes the refinement's residual land in the permuted row order.  Pivots
// come only from rows [k, n), never from the central site's rows, so the trailing b x b block
// still holds the Schur complement 1 - Delta.
//
// Selection arithmetic is FP32 on either factor type (it only ranks pivot magnitudes, |re| + |im|
// as izamax, ties to the lower candidate); the factorisation itself is unchanged.

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "common.cuh"

namespace b200 {
namespace {

constexpr int kSelThreads = kPivLeafRows;  // one candidate row per thread
static_assert(kSelThreads == 256, "selection thread layout");

__device__ __forceinline__ float2 to_f2(double2 a) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ float2 to_f2(float2 a) { return a; }

// Node counts of a job's tournament: level 0 has ceil(m / leaf) nodes, each level above merges
// kPivFanIn of them.
__device__ __forceinline__ int nodes_at(int m, int level) {
  int nodes = (m + kPivLeafRows - 1) / kPivLeafRows;
  for (int l = 0; l < level; ++l) nodes = (nodes + kPivFanIn - 1) / kPivFanIn;
  return nodes;
}

// One tournament node: candidates (one per thread), GEPP on their panel rows in shared memory,
// the kb nominees in pivot order.  The root also writes the step's row moves and applies them to
// the job's permutation.
template <typename T>
__global__ void __launch_bounds__(kSelThreads) panel_select_kernel(const JobDev *__restrict__ jobs, int k,
                                                                   int level) {
  const JobDev &J = jobs[blockIdx.y];
  if (J.inactive || J.piv == nullptr || k >= J.n) return;
  const int kb = min(kNb, J.n - k);
  const int m = J.n - k;  // candidate rows [k, n)
  const int nodes = nodes_at(m, level);
  if (level > 0 && nodes_at(m, level - 1) <= 1) return;  // this job's root was at a lower level
  const int node = blockIdx.x;
  if (node >= nodes) return;
  const bool root = nodes == 1;
  const int ld = J.ld;
  int *__restrict__ piv = J.piv;
  const int *__restrict__ sets_in = piv + pivot_sets_offset(ld, (level + 1) & 1);
  int *__restrict__ sets_out = piv + pivot_sets_offset(ld, level & 1);

  extern __shared__ __align__(16) unsigned char sel_smem[];
  float2(*A)[kPivLeafRows] = reinterpret_cast<float2(*)[kPivLeafRows]>(sel_smem);  // A[col][cand]
  __shared__ int s_cand[kPivLeafRows];
  __shared__ int s_out[kNb];
  __shared__ float s_wv[2][kSelThreads / 32];
  __shared__ int s_wi[2][kSelThreads / 32];

  const int r = threadIdx.x, lane = r & 31, warp = r >> 5;
  int cand = -1;
  if (level == 0) {
    const int row = k + node * kPivLeafRows + r;
    if (row < J.n) cand = row;
  } else {
    const int prev = nodes_at(m, level - 1);
    const int set = node * kPivFanIn + r / kNb;
    if (set < prev) cand = sets_in[set * kNb + r % kNb];
  }
  s_cand[r] = cand;
  const int R = __syncthreads_count(cand >= 0);

  if (R <= kb) {  // every candidate is a nominee (the last steps, or sparse merges)
    if (r == 0) {
      int c = 0;
      for (int i = 0; i < kPivLeafRows; ++i)
        if (s_cand[i] >= 0) s_out[c++] = s_cand[i];
      for (; c < kNb; ++c) s_out[c] = -1;
    }
    __syncthreads();
  } else {
    const T *__restrict__ F = static_cast<const T *>(J.F);
    // panel rows into shared memory; at the leaves consecutive threads read consecutive rows
    for (int j = 0; j < kb; ++j)
      A[j][r] = cand >= 0 ? to_f2(F[(size_t)cand + (size_t)(k + j) * ld]) : make_float2(0.f, 0.f);
    __syncthreads();
    bool taken = false;
    for (int p = 0; p < kb; ++p) {
      const int par = p & 1;
      float v = -1.f;
      if (cand >= 0 && !taken) {
        const float2 a = A[p][r];
        v = fabsf(a.x) + fabsf(a.y);
        if (!(v == v)) v = 0.f;  // a NaN ranks as zero, so a row in range is still chosen
      }
      int idx = r;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {  // warp arg-max, ties to the lower candidate
        const float ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi < idx)) {
          v = ov;
          idx = oi;
        }
      }
      if (lane == 0) {
        s_wv[par][warp] = v;
        s_wi[par][warp] = idx;
      }
      __syncthreads();
      float bv = s_wv[par][0];
      int bi = s_wi[par][0];
#pragma unroll
      for (int w = 1; w < kSelThreads / 32; ++w) {
        const float ov = s_wv[par][w];
        const int oi = s_wi[par][w];
        if (ov > bv || (ov == bv && oi < bi)) {
          bv = ov;
          bi = oi;
        }
      }
      // R > kb > p candidates remain untaken, each ranked >= 0: bi is one of them
      if (r == bi) taken = true;
      if (r == 0) s_out[p] = s_cand[bi];
      if (cand >= 0 && !taken && p + 1 < kb) {
        const float2 d = A[p][bi];
        const float dd = d.x * d.x + d.y * d.y;
        float2 f = make_float2(0.f, 0.f);
        if (dd > 0.f) {
          const float2 a = A[p][r];
          f = make_float2((a.x * d.x + a.y * d.y) / dd, (a.y * d.x - a.x * d.y) / dd);
        }
        for (int j = p + 1; j < kb; ++j) {
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
  if (!root) {
    if (r < kNb) sets_out[node * kNb + r] = s_out[r];
    return;
  }
  if (r != 0) return;
  // the root: moves that bring the nominees to k..k+kb-1 (pivot order) and the displaced rows to
  // the vacated positions; a permutation of at most 2 kb positions, also applied to perm
  int *mv = piv + pivot_moves_offset(ld);
  int *dst = mv + 1, *src = mv + 1 + 2 * kNb;
  // kb distinct nominees in [k, n) by construction; anything else leaves the rows in place
  for (int p = 0; p < kb; ++p)
    if (s_out[p] < k || s_out[p] >= J.n) {
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
  const int m = max_n - k;
  if (m <= 0) return cudaSuccess;
  const int smem = kNb * kPivLeafRows * (int)sizeof(float2);
  cudaError_t e = ensure_smem(panel_select_kernel<T>, smem);
  if (e != cudaSuccess) return e;
  int nodes = (m + kPivLeafRows - 1) / kPivLeafRows;
  for (int level = 0;; ++level) {
    panel_select_kernel<T><<<dim3(nodes, njobs), kSelThreads, smem, s>>>(jobs, k, level);
    if (launches) *launches += 1;
    if (nodes == 1) break;
    nodes = (nodes + kPivFanIn - 1) / kPivFanIn;
  }
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
