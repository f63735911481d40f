// Block sweeps of the correction solve Y = F^-1 R, one thread-block cluster of 8 CTAs per job.
//
// F holds the block factors of the elimination (block_lu.cu): D_k = A11_k^-1 in the diagonal
// blocks, A21_k below them, W_k = D_k A12_k to their right, S in the trailing b x b block.
//   forward   for k = 0, 64, ..., < n:  Y_k = D_k R_k;  R[k+kb:N] -= A21_k Y_k
//   backward  for the central block, then k = last, ..., 0:  X_k (+)= Y_k;  Y[0:k] -= W[0:k, k] Y_k
// (the S solve between them is schur_solve_kernel).  This is the same contract as the reference's
// zgetrs on the block LU factors (zblock_lu_cpp.cpp:60-86) applied to the N x b right-hand side.
//
// One launch covers the whole sweep: the 8 CTAs of a cluster split the trailing 64-row tiles
// (tile t on rank t % 8, so each tile of R or Y always has the same writer) and meet at a cluster
// barrier (release / acquire) after each block step; cross-CTA reads go through L2 (__ldcg).
// Each CTA recomputes the small Y_k = D_k R_k itself rather than waiting for another CTA's copy.

#include <cuda_runtime.h>

#include "common.cuh"
#include "cplx.cuh"

namespace b200 {
namespace {

using namespace cx;

constexpr int kClus = 8;

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// Every thread of every CTA of the cluster; orders the global writes made before it.
__device__ __forceinline__ void cluster_sync() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::
          : "memory");
}

template <typename T>
constexpr int forward_smem_bytes() {
  return (int)(sizeof(T) * kNb * kNb + 2 * sizeof(double2) * kNb * kMaxB);
}

// Grid (8, njobs), cluster (8, 1, 1).  mode is 1 (refinement rounds only: the initial solve has
// B = 0 above the central block, so its forward sweep is the identity).
template <typename T>
__global__ void __cluster_dims__(kClus, 1, 1) __launch_bounds__(256)
    forward_sweep_kernel(const JobDev *__restrict__ jobs) {
  const JobDev &J = jobs[blockIdx.y];
  if (converged(J.conv)) return;  // the flag changes only between launches: uniform per cluster
  const int rank = (int)cluster_rank();
  const int n = J.n, N = J.N, ld = J.ld, b = J.b;
  const T *__restrict__ F = static_cast<const T *>(J.F);
  extern __shared__ __align__(16) unsigned char fsm[];
  T *Ds = reinterpret_cast<T *>(fsm);                                            // Ds[j * 64 + r]
  double2 *Rs = reinterpret_cast<double2 *>(fsm + sizeof(T) * kNb * kNb);        // Rs[c * 64 + r]
  double2(*Ys)[kMaxB] = reinterpret_cast<double2(*)[kMaxB]>(fsm + sizeof(T) * kNb * kNb +
                                                              sizeof(double2) * kNb * kMaxB);
  const int tid = threadIdx.x;
  const int tr = tid & 63, tc = tid >> 6;
  for (int k = 0; k < n; k += kNb) {
    const int kb = min(kNb, n - k);
    for (int e = tid; e < kb * kb; e += 256) {
      const int r = e % kb, j = e / kb;
      Ds[j * kNb + r] = F[(size_t)(k + r) + (size_t)(k + j) * ld];
    }
    for (int e = tid; e < kb * b; e += 256) {
      const int r = e % kb, c = e / kb;
      Rs[c * kNb + r] = __ldcg(J.R + (size_t)(k + r) + (size_t)c * ld);
    }
    __syncthreads();
    for (int e = tid; e < kb * b; e += 256) {
      const int r = e % kb, c = e / kb;
      double2 s = make_double2(0.0, 0.0);
#pragma unroll 8
      for (int j = 0; j < kb; ++j) s = cfma(ldc(&Ds[j * kNb + r]), Rs[c * kNb + j], s);
      Ys[r][c] = s;
      if (rank == 0) J.Y[(size_t)(k + r) + (size_t)c * ld] = s;
    }
    __syncthreads();
    // R[k+kb:N] -= A21_k Y_k over absolute 64-row tiles
    for (int t = (k + kb) / 64; t * 64 < N; ++t) {
      if (t % kClus != rank) continue;
      const int gr = t * 64 + tr;
      if (gr < k + kb || gr >= N) continue;
      double2 acc[kMaxB / 4];
#pragma unroll
      for (int j = 0; j < kMaxB / 4; ++j) acc[j] = make_double2(0.0, 0.0);
      const T *lrow = F + (size_t)gr + (size_t)k * ld;
#pragma unroll 8
      for (int jj = 0; jj < kb; ++jj) {
        const double2 a = ldc(lrow + (size_t)jj * ld);
#pragma unroll
        for (int j = 0; j < kMaxB / 4; ++j) {
          const int c = tc + 4 * j;
          if (c < b) acc[j] = cfma(a, Ys[jj][c], acc[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < kMaxB / 4; ++j) {
        const int c = tc + 4 * j;
        if (c >= b) continue;
        double2 *dst = J.R + (size_t)gr + (size_t)c * ld;
        *dst = csub(__ldcg(dst), acc[j]);
      }
    }
    cluster_sync();  // R_(k+64) complete before any CTA stages it; Ds, Rs, Ys free again
  }
}

// Grid (8, njobs), cluster (8, 1, 1).  mode 0 sets X = Y, mode 1 adds X += Y (and skips
// converged jobs).
template <typename T>
__global__ void __cluster_dims__(kClus, 1, 1) __launch_bounds__(256)
    backward_sweep_kernel(const JobDev *__restrict__ jobs, int mode) {
  const JobDev &J = jobs[blockIdx.y];
  if (mode == 1 && converged(J.conv)) return;
  const int rank = (int)cluster_rank();
  const int n = J.n, ld = J.ld, b = J.b;
  const T *__restrict__ F = static_cast<const T *>(J.F);
  __shared__ double2 Ys[kNb][kMaxB];
  const int tid = threadIdx.x;
  const int tr = tid & 63, tc = tid >> 6;
  const int last = n > 0 ? ((n - 1) / kNb) * kNb : 0;
  int k = n, kb = b;  // the central block first
  for (;;) {
    for (int e = tid; e < kb * b; e += 256) {
      const int r = e % kb, c = e / kb;
      const size_t idx = (size_t)(k + r) + (size_t)c * ld;
      const double2 y = __ldcg(J.Y + idx);
      Ys[r][c] = y;
      if (rank == 0) {
        if (mode == 0) {
          J.X[idx] = y;
        } else {
          const double2 x = J.X[idx];
          J.X[idx] = make_double2(x.x + y.x, x.y + y.y);
        }
      }
    }
    __syncthreads();
    // Y[0:k] -= F[0:k, k:k+kb] Y_k over absolute 64-row tiles
    for (int t = rank; t * 64 < k; t += kClus) {
      const int gr = t * 64 + tr;
      if (gr >= k) continue;
      double2 acc[kMaxB / 4];
#pragma unroll
      for (int j = 0; j < kMaxB / 4; ++j) acc[j] = make_double2(0.0, 0.0);
      const T *urow = F + (size_t)gr + (size_t)k * ld;
#pragma unroll 8
      for (int jj = 0; jj < kb; ++jj) {
        const double2 a = ldc(urow + (size_t)jj * ld);
#pragma unroll
        for (int j = 0; j < kMaxB / 4; ++j) {
          const int c = tc + 4 * j;
          if (c < b) acc[j] = cfma(a, Ys[jj][c], acc[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < kMaxB / 4; ++j) {
        const int c = tc + 4 * j;
        if (c >= b) continue;
        double2 *dst = J.Y + (size_t)gr + (size_t)c * ld;
        *dst = csub(__ldcg(dst), acc[j]);
      }
    }
    cluster_sync();  // Y_(next k) complete; Ys free again
    if (k == 0) break;
    k = (k == n) ? last : k - kNb;
    kb = min(kNb, n - k);
  }
}

template <typename T>
cudaError_t sweep_impl(const JobDev *jobs, int njobs, bool forward, int mode, cudaStream_t s) {
  const dim3 grid(kClus, njobs);
  if (forward) {
    const int smem = forward_smem_bytes<T>();
    cudaError_t e = cudaFuncSetAttribute(forward_sweep_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem);
    if (e != cudaSuccess) return e;
    forward_sweep_kernel<T><<<grid, 256, smem, s>>>(jobs);
  } else {
    backward_sweep_kernel<T><<<grid, 256, 0, s>>>(jobs, mode);
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_sweep(FactorKind fk, const JobDev *jobs, int njobs, int b, bool forward, int mode,
                         cudaStream_t s) {
  if (njobs <= 0) return cudaSuccess;
  if (b > kMaxB || (forward && mode != 1)) return cudaErrorInvalidValue;
  return fk == kFactorFP64 ? sweep_impl<double2>(jobs, njobs, forward, mode, s)
                           : sweep_impl<float2>(jobs, njobs, forward, mode, s);
}

}  // namespace b200
