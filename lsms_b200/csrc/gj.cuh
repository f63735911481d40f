// Small dense solves in shared memory shared by the elimination and adjoint kernels.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "cplx.cuh"

namespace b200 {
namespace cx {

// b x b solve by Gauss-Jordan on [A | rhs] in shared memory (FP64, partial pivoting on |re|+|im|,
// first index on ties).  A is kMaxB x (2 kMaxB + 1); on return columns [b, 2b) hold A^-1 rhs.
// Called by every thread of the block.  Returns singular.
__device__ inline bool gj_solve_smem(double2 (*A)[2 * kMaxB + 1], int b, int *s_piv, double2 *s_dinv) {
  const int tid = threadIdx.x;
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
      if (tid == 0) *s_piv = bi;
    }
    __syncthreads();
    const int pv = *s_piv;
    if (pv != p)
      for (int c = tid; c < 2 * b; c += blockDim.x) {
        const double2 t = A[p][c];
        A[p][c] = A[pv][c];
        A[pv][c] = t;
      }
    __syncthreads();
    if (tid == 0) {
      const double2 d = A[p][p];
      *s_dinv = (d.x == 0.0 && d.y == 0.0) ? make_double2(0.0, 0.0) : crecip(d);
    }
    __syncthreads();
    const double2 dinv = *s_dinv;
    if (dinv.x == 0.0 && dinv.y == 0.0) singular = true;
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
  return singular;
}

}  // namespace cx
}  // namespace b200
