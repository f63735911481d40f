// Block sweeps of the correction solve Y = F^-1 R, one thread-block cluster per job.
//
// F holds the block factors of the elimination (block_lu.cu): D_k = A11_k^-1 in the diagonal
// blocks, A21_k below them, W_k = D_k A12_k to their right, S in the trailing b x b block.
//   forward   for k = 0, 64, ..., < n:  Y_k = D_k R_k;  R[k+kb:N] -= A21_k Y_k
//   backward  for the central block, then k = last, ..., 0:  X_k (+)= Y_k;  Y[0:k] -= W[0:k, k] Y_k
// (the S solve between them is schur_solve_kernel).  This is the same contract as the reference's
// zgetrs on the block LU factors (zblock_lu_cpp.cpp:60-86) applied to the N x b right-hand side.
//
// Layout of the work.  The CTAs of a cluster (cluster size cs, chosen per launch so that one
// wave of jobs fills the GPU once) split the 64-row tiles of R or Y: tile t always belongs to
// rank t % cs, so every tile has one writer.  The operand panels (A21_k or W_k rows of a tile,
// 64 rows x 32 columns per unit) are constant during a sweep, so each CTA streams its units
// through a two-stage cp.async ring in shared memory, fetching the next unit while it multiplies
// the current one; the arithmetic is FP64 FMA.  One cluster barrier (release / acquire) per block
// step orders the tile updates; cross-CTA reads of R and Y go through L2 (__ldcg).
// In the forward sweep the owner of the next diagonal block updates that tile first and computes
// Y_(k+1) = D_(k+1) R_(k+1) while the other CTAs finish step k, so the small D multiply is off the
// critical path of all but one CTA.

#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "common.cuh"
#include "cluster.cuh"
#include "cplx.cuh"

namespace b200 {
namespace {

using namespace cx;
using namespace cl;

constexpr int kUnitCols = 32;  // operand columns per pipeline unit
constexpr int kMaxCluster = 8;

// Shared-memory layout of the sweep kernels.
// T: factor storage type; V: arithmetic type of the sweep (double2, or float2 for a correction
// solve in single precision on FP32 factors, as in LAPACK's zcgesv).
template <typename T, typename V>
struct SweepSmem {
  static constexpr int kUnitBytes = kUnitCols * 64 * (int)sizeof(T);
  static constexpr int kLs = 0;                                     // 2 units
  static constexpr int kDs = kLs + 2 * kUnitBytes;                  // D_(k+1), 64 x 64 (forward)
  static constexpr int kYs = kDs + 64 * 64 * (int)sizeof(T);        // Y_k, 64 x kMaxB
  static constexpr int kRs = kYs + 64 * kMaxB * (int)sizeof(V);     // R_(k+1) (forward)
  static constexpr int kForward = kRs + 64 * kMaxB * (int)sizeof(V);
  static constexpr int kBackward = kDs + 64 * kMaxB * (int)sizeof(V);  // Ls + Ys only
};

// The units (64-row tile t, 32-column slice h of block step k) of one CTA in the order it
// consumes them; a second copy runs ahead to issue the prefetches.
struct ForwardUnits {
  int n, N, cs, rank;
  int k, kb, t, h;
  __device__ void begin() {
    k = 0;
    seek();
  }
  __device__ bool done() const { return k >= n; }
  __device__ int ncol() const { return min(kUnitCols, kb - h * kUnitCols); }
  // first own tile of step k (rows from k + kb), or of a later step
  __device__ void seek() {
    for (; k < n; k += 64) {
      kb = min(64, n - k);
      const int tlo = (k + kb) / 64;
      t = tlo + (rank - tlo % cs + cs) % cs;
      if (t * 64 < N) {
        h = 0;
        return;
      }
    }
  }
  __device__ void next() {
    if (++h * kUnitCols < kb) return;
    h = 0;
    t += cs;
    if (t * 64 < N) return;
    k += 64;
    seek();
  }
};

struct BackwardUnits {
  int n, b, cs, rank;
  int k, kb, t, h;
  bool fin;
  __device__ void begin() {
    k = n;
    kb = b;
    fin = false;
    seek();
  }
  __device__ bool done() const { return fin; }
  __device__ int ncol() const { return min(kUnitCols, kb - h * kUnitCols); }
  // own tiles of block k cover rows [0, k); blocks run central, last, last - 64, ..., 0
  __device__ void seek() {
    for (;;) {
      t = rank;
      if (t * 64 < k) {
        h = 0;
        return;
      }
      if (k == 0) {
        fin = true;
        return;
      }
      k = (k == n) ? ((n - 1) / 64) * 64 : k - 64;
      kb = min(64, n - k);
    }
  }
  __device__ void next() {
    if (++h * kUnitCols < kb) return;
    h = 0;
    t += cs;
    if (t * 64 < k) return;
    if (k == 0) {
      fin = true;
      return;
    }
    k = (k == n) ? ((n - 1) / 64) * 64 : k - 64;
    kb = min(64, n - k);
    seek();
  }
};

// acc[j] += sum_kk Lu[kk][r] * Ys[y0 + kk][cg + 4 j] over one unit of ncol columns.
template <typename T, typename V, int NJ>
__device__ __forceinline__ void unit_product(V (&acc)[NJ], const T *__restrict__ Lu,
                                             const V (*__restrict__ Ys)[kMaxB], int y0, int ncol, int r, int cg) {
#pragma unroll 8
  for (int kk = 0; kk < ncol; ++kk) {
    const V a = to_v<V>(Lu[kk * 64 + r]);
#pragma unroll
    for (int j = 0; j < NJ; ++j) acc[j] = cfma(a, Ys[y0 + kk][cg + 4 * j], acc[j]);
  }
}

// Columns [b, bc) of a 64 x kMaxB staging block read as zero.
template <typename V>
__device__ __forceinline__ void zero_pad_columns(V (*Ys)[kMaxB], int b, int bc) {
  for (int e = threadIdx.x; e < 64 * (bc - b); e += blockDim.x) Ys[e % 64][b + e / 64] = vzero<V>();
}

// Grid (cs, njobs), cluster (cs, 1, 1), 256 threads.  Refinement rounds only: the initial solve
// has B = 0 above the central block, so its forward sweep is the identity.  BC is 16 or 32,
// the padded column count of the right-hand side (b <= BC).
template <typename T, typename V, int BC>
__global__ void __launch_bounds__(256) forward_sweep_kernel(const JobDev *__restrict__ jobs) {
  constexpr int NJ = BC / 4;
  using L = SweepSmem<T, V>;
  const JobDev &J = jobs[blockIdx.y];
  // uniform over the cluster: the flag changes only between launches
  if (converged(J.conv) || J.n == 0 || J.inactive) return;
  const int rank = cluster_rank(), cs = cluster_size();
  const int n = J.n, N = J.N, ld = J.ld, b = J.b;
  const T *__restrict__ F = static_cast<const T *>(J.F);
  extern __shared__ __align__(128) unsigned char sm[];
  T *Ls = reinterpret_cast<T *>(sm + L::kLs);
  T *Ds = reinterpret_cast<T *>(sm + L::kDs);
  V(*Ys)[kMaxB] = reinterpret_cast<V(*)[kMaxB]>(sm + L::kYs);
  V(*Rs)[kMaxB] = reinterpret_cast<V(*)[kMaxB]>(sm + L::kRs);
  const int tid = threadIdx.x, r = tid & 63, cg = tid >> 6;
  zero_pad_columns(Ys, b, BC);
  zero_pad_columns(Rs, b, BC);

  // Y_k = D_k R_k (D_k in Ds, R_k in Rs) into J.Y rows [k, k + kb)
  auto diag_apply = [&](int k, int kb) {
    if (r >= kb) return;
    V acc[NJ];
#pragma unroll
    for (int j = 0; j < NJ; ++j) acc[j] = vzero<V>();
    unit_product<T, V, NJ>(acc, Ds, Rs, 0, kb, r, cg);
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const int c = cg + 4 * j;
      if (c < b) J.Y[(size_t)(k + r) + (size_t)c * ld] = to_d(acc[j]);
    }
  };

  if (rank == 0) {  // Y_0
    const int kb0 = min(64, n);
    stage_block(Ds, F, ld, 0, 0, kb0);
    cp_async_commit();
    for (int e = tid; e < kb0 * b; e += 256)
      Rs[e % kb0][e / kb0] = to_v<V>(__ldcg(J.R + (size_t)(e % kb0) + (size_t)(e / kb0) * ld));
    cp_async_wait<0>();
    __syncthreads();
    diag_apply(0, kb0);
  }
  cluster_sync();

  constexpr int kUnitElems = kUnitCols * 64;
  ForwardUnits it{n, N, cs, rank};
  it.begin();
  ForwardUnits pf = it;
  for (int s = 0; s < 2; ++s) {
    if (!pf.done()) {
      stage_block(Ls + s * kUnitElems, F, ld, pf.t * 64, pf.k + pf.h * kUnitCols, pf.ncol());
      pf.next();
    }
    cp_async_commit();
  }
  int stage = 0;
  for (int k = 0; k < n; k += 64) {
    const int kb = min(64, n - k);
    const int tnext = (k + 64) / 64;  // tile of the next diagonal block
    const bool owner = k + 64 < n && tnext % cs == rank;
    if (owner) {
      stage_block(Ds, F, ld, k + 64, k + 64, min(64, n - k - 64));
      cp_async_commit();
    }
    for (int e = tid; e < kb * b; e += 256) {
      const int rr = e % kb, c = e / kb;
      Ys[rr][c] = to_v<V>(__ldcg(J.Y + (size_t)(k + rr) + (size_t)c * ld));
    }
    while (!it.done() && it.k == k) {
      const int t = it.t;
      V acc[NJ];
#pragma unroll
      for (int j = 0; j < NJ; ++j) acc[j] = vzero<V>();
      do {
        cp_async_wait<1>();
        __syncthreads();  // this unit has landed for every thread; Ys is complete
        unit_product<T, V, NJ>(acc, Ls + stage * kUnitElems, Ys, it.h * kUnitCols, it.ncol(), r, cg);
        __syncthreads();  // every thread is done with the stage before it is refilled
        if (!pf.done()) {
          stage_block(Ls + stage * kUnitElems, F, ld, pf.t * 64, pf.k + pf.h * kUnitCols, pf.ncol());
          pf.next();
        }
        cp_async_commit();
        stage ^= 1;
        it.next();
      } while (!it.done() && it.k == k && it.t == t && it.h != 0);
      // R[tile] -= A21_k Y_k for the rows below the block
      const int gr = t * 64 + r;
      if (gr >= k + kb && gr < N) {
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          const int c = cg + 4 * j;
          if (c >= b) continue;
          double2 *dst = J.R + (size_t)gr + (size_t)c * ld;
          const V v = csub(to_v<V>(__ldcg(dst)), acc[j]);
          *dst = to_d(v);
          if (owner && t == tnext) Rs[r][c] = v;
        }
      }
      if (owner && t == tnext) {  // Y_(k+1) for every CTA of the next step
        cp_async_wait<0>();
        __syncthreads();
        diag_apply(k + 64, min(64, n - k - 64));
      }
    }
    cluster_sync();  // R and Y of this step are final; Ys, Rs and Ds are free again
  }
  cp_async_wait<0>();
}

// Grid (cs, njobs), cluster (cs, 1, 1), 256 threads.  mode 0 sets X = Y, mode 1 adds X += Y
// (and skips converged jobs).
template <typename T, typename V, int BC>
__global__ void __launch_bounds__(256) backward_sweep_kernel(const JobDev *__restrict__ jobs, int mode) {
  constexpr int NJ = BC / 4;
  using L = SweepSmem<T, V>;
  const JobDev &J = jobs[blockIdx.y];
  if ((mode == 1 && converged(J.conv)) || J.inactive) return;
  const int rank = cluster_rank(), cs = cluster_size();
  const int n = J.n, ld = J.ld, b = J.b;
  const T *__restrict__ F = static_cast<const T *>(J.F);
  extern __shared__ __align__(128) unsigned char sm[];
  T *Ls = reinterpret_cast<T *>(sm + L::kLs);
  V(*Ys)[kMaxB] = reinterpret_cast<V(*)[kMaxB]>(sm + L::kDs);
  const int tid = threadIdx.x, r = tid & 63, cg = tid >> 6;
  zero_pad_columns(Ys, b, BC);

  constexpr int kUnitElems = kUnitCols * 64;
  BackwardUnits it{n, b, cs, rank};
  it.begin();
  BackwardUnits pf = it;
  for (int s = 0; s < 2; ++s) {
    if (!pf.done()) {
      stage_block(Ls + s * kUnitElems, F, ld, pf.t * 64, pf.k + pf.h * kUnitCols, pf.ncol());
      pf.next();
    }
    cp_async_commit();
  }
  int stage = 0;
  int k = n, kb = b;  // the central block first
  for (;;) {
    for (int e = tid; e < kb * b; e += 256) {
      const int rr = e % kb, c = e / kb;
      const size_t idx = (size_t)(k + rr) + (size_t)c * ld;
      const double2 y = __ldcg(J.Y + idx);
      Ys[rr][c] = to_v<V>(y);
      if (rank == 0) {
        if (mode == 0) {
          J.X[idx] = y;
        } else {
          const double2 x = J.X[idx];
          J.X[idx] = make_double2(x.x + y.x, x.y + y.y);
        }
      }
    }
    while (!it.done() && it.k == k) {
      const int t = it.t;
      V acc[NJ];
#pragma unroll
      for (int j = 0; j < NJ; ++j) acc[j] = vzero<V>();
      do {
        cp_async_wait<1>();
        __syncthreads();
        unit_product<T, V, NJ>(acc, Ls + stage * kUnitElems, Ys, it.h * kUnitCols, it.ncol(), r, cg);
        __syncthreads();
        if (!pf.done()) {
          stage_block(Ls + stage * kUnitElems, F, ld, pf.t * 64, pf.k + pf.h * kUnitCols, pf.ncol());
          pf.next();
        }
        cp_async_commit();
        stage ^= 1;
        it.next();
      } while (!it.done() && it.k == k && it.t == t && it.h != 0);
      // Y[tile] -= W[tile, k:k+kb] Y_k for the rows above the block
      const int gr = t * 64 + r;
      if (gr < k) {
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          const int c = cg + 4 * j;
          if (c >= b) continue;
          double2 *dst = J.Y + (size_t)gr + (size_t)c * ld;
          *dst = to_d(csub(to_v<V>(__ldcg(dst)), acc[j]));
        }
      }
    }
    cluster_sync();  // Y of the next block is final; Ys is free again
    if (k == 0) break;
    k = (k == n) ? ((n - 1) / 64) * 64 : k - 64;
    kb = min(64, n - k);
  }
  cp_async_wait<0>();
}

// Clusters of `kern` (cs CTAs of 256 threads, smem bytes each) resident at once, cached per
// (kernel, cs, smem); 0 when the query fails.
int resident_clusters(const void *kern, int cs, int smem) {
  struct Entry {
    const void *kern;
    int cs, smem, dev, v;
  };
  static std::mutex mu;
  static std::vector<Entry> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> lock(mu);
  for (const Entry &c : cache)
    if (c.kern == kern && c.cs == cs && c.smem == smem && c.dev == dev) return c.v;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs, 1, 1);
  cfg.blockDim = dim3(256, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int v = 0;
  if (cudaOccupancyMaxActiveClusters(&v, kern, &cfg) != cudaSuccess) {
    cudaGetLastError();
    v = 0;
  }
  cache.push_back({kern, cs, smem, dev, v});
  return v;
}

// The largest power-of-two cluster (up to 8 CTAs) whose clusters for `want` jobs are resident at
// once, at the kernel's real occupancy (several CTAs per SM where the shared memory allows): the
// per-step latency chain of a job shrinks with its cluster, so one full wave of the largest
// clusters is the fastest.  `want` is the number of jobs expected to work (converged jobs' clusters
// leave at once), so late refinement rounds with few jobs left take larger clusters.
template <typename K>
int cluster_for(K *kern, int smem, int njobs) {
  for (int cs = kMaxCluster; cs > 1; cs >>= 1)
    if (resident_clusters(reinterpret_cast<const void *>(kern), cs, smem) >= njobs) return cs;
  return 1;
}

template <typename T, typename V, int BC>
cudaError_t sweep_impl(const JobDev *jobs, int njobs, bool forward, int mode, cudaStream_t s, int want) {
  cudaError_t e;
  if (forward) {
    const int smem = SweepSmem<T, V>::kForward;
    if ((e = ensure_smem(forward_sweep_kernel<T, V, BC>, smem)) != cudaSuccess)
      return e;
    const int cs = cluster_for(forward_sweep_kernel<T, V, BC>, smem, want);
    return launch_cluster(forward_sweep_kernel<T, V, BC>, cs, njobs, 256, smem, s, jobs);
  }
  const int smem = SweepSmem<T, V>::kBackward;
  if ((e = ensure_smem(backward_sweep_kernel<T, V, BC>, smem)) != cudaSuccess)
    return e;
  const int cs = cluster_for(backward_sweep_kernel<T, V, BC>, smem, want);
  return launch_cluster(backward_sweep_kernel<T, V, BC>, cs, njobs, 256, smem, s, jobs, mode);
}

template <typename T, typename V>
cudaError_t sweep_b(const JobDev *jobs, int njobs, int b, bool forward, int mode, cudaStream_t s,
                    int active_hint = 0) {
  const int want = active_hint > 0 && active_hint < njobs ? active_hint : njobs;
  return b <= 16 ? sweep_impl<T, V, 16>(jobs, njobs, forward, mode, s, want)
                 : sweep_impl<T, V, 32>(jobs, njobs, forward, mode, s, want);
}

}  // namespace


cudaError_t launch_sweep(FactorKind fk, const JobDev *jobs, int njobs, int b, int max_N, bool forward, int mode,
                         bool fp32_arith, const CUtensorMap *fmap, cudaStream_t s, int active_hint) {
  if (njobs <= 0) return cudaSuccess;
  if (b < 1 || b > kMaxB || (forward && mode != 1)) return cudaErrorInvalidValue;
  if (fk == kFactorFP64) return sweep_b<double2, double2>(jobs, njobs, b, forward, mode, s, active_hint);
  if (fp32_arith) {
    bool done = false;
    const cudaError_t e = launch_flow_sweep(jobs, njobs, b, max_N, forward, mode, fmap, s, &done, active_hint);
    if (e != cudaSuccess || done) return e;
    return sweep_b<float2, float2>(jobs, njobs, b, forward, mode, s, active_hint);
  }
  return sweep_b<float2, double2>(jobs, njobs, b, forward, mode, s, active_hint);
}

}  // namespace b200
