// Thread-block-cluster, cp.async and mbarrier helpers of the sweep kernels (sweep.cu,
// sweep_flow.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

namespace b200 {
namespace cl {

__device__ __forceinline__ int cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return (int)r;
}
__device__ __forceinline__ int cluster_size() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return (int)r;
}
// Every thread of every CTA of the cluster; orders the memory operations made before it.
__device__ __forceinline__ void cluster_sync() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::
          : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Copies the 64 x ncol block of F at (row0, col0) into shared memory, column-major with 64 rows
// per column (dst[c * 64 + r]).  The rows past N up to the leading dimension are inside the
// allocation (ld >= N rounded up to 64) and are never used by the arithmetic.
template <typename T>
__device__ __forceinline__ void stage_block(T *dst, const T *F, int ld, int row0, int col0, int ncol) {
  constexpr int kPer = 16 / (int)sizeof(T);  // elements per 16-byte copy
  constexpr int kCpc = 64 / kPer;            // copies per column
  for (int e = threadIdx.x; e < ncol * kCpc; e += blockDim.x) {
    const int c = e / kCpc, part = e - c * kCpc;
    cp_async16(dst + c * 64 + part * kPer, F + (size_t)row0 + part * kPer + (size_t)(col0 + c) * ld);
  }
}

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// The address of the same shared-memory location in CTA `cta` of the cluster.
__device__ __forceinline__ unsigned remote_u32(const void *p, int cta) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(cta));
  return r;
}
__device__ __forceinline__ void st_remote(unsigned addr, float4 v) {
  asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(v.x), "f"(v.y), "f"(v.z),
               "f"(v.w)
               : "memory");
}
__device__ __forceinline__ void st_remote_f32(unsigned addr, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}

__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
// Makes the initialised barriers visible to the other CTAs of the cluster.
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Arrival (release at cluster scope) on the barrier at the same offset in CTA `cta`.
__device__ __forceinline__ void mbar_arrive_cluster(unsigned long long *b, int cta) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(remote_u32(b, cta))
               : "memory");
}
// `count` arrivals on a barrier of this CTA.
__device__ __forceinline__ void mbar_arrive_local(unsigned long long *b, unsigned count) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
// One test of the phase with the given parity; acquire at cluster scope, so the memory
// operations that the (possibly remote) arrivals released are visible once it succeeds.
__device__ __forceinline__ bool mbar_try_cluster(unsigned long long *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// The same with acquire at CTA scope, for barriers that only this CTA's threads, TMA loads or
// tensor-core commits complete.
__device__ __forceinline__ bool mbar_try_cta(unsigned long long *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Local barrier: one arrival that also expects `bytes` of asynchronous (TMA) transfers.
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
// Orders this thread's earlier generic-proxy shared-memory accesses before its later async-proxy
// (TMA) ones.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Tiled TMA load of the box at (x, y, z) of a 3-D tensor map into shared memory, completing on
// barrier `bar`.  x times the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Grid (cs, njobs) of `threads`-thread CTAs in clusters of (cs, 1, 1): one cluster per job.
template <typename Kern, typename... Args>
cudaError_t launch_cluster(Kern kern, int cs, int njobs, int threads, int smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs, njobs, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

}  // namespace cl
}  // namespace b200
