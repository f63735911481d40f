// Mixed-precision trailing update on the 5th-generation tensor cores (sm_100a, tcgen05).
//
// The block elimination's O(N^3) step A22 -= A21 W (block_lu.cu; reference: the zgemm calls of
// zblock_lu_cpp.cpp:72-75 and the cublasZgemm updates of zblock_lu_cuda_c.cu:278-331) runs here
// in complex FP32 storage with TF32 tensor-core products split hi/lo (3 passes: hi*hi + hi*lo +
// lo*hi, FP32 accumulation in TMEM), which keeps the product at about FP32 accuracy; the FP64
// refinement against the unmodified KKR matrix (block_lu.cu) restores FP64 accuracy of tau00.
//
// Complex arithmetic as one real GEMM.  With F stored column-major as interleaved (re, im) floats,
// a column-major complex C (m x n) is the real matrix Chat (2m x n) with rows (2r, 2r+1) = (re, im).
// Then Chat = Atil * Bhat where
//   Bhat (2K x n) is W's own storage: column c = (Wr[0,c], Wi[0,c], Wr[1,c], Wi[1,c], ...)
//   Atil (2m x 2K) expands every complex a of A21 into [[ar, -ai], [ai, ar]],
// i.e. one real GEMM with M = 2m, N = n, K = 2 kb and 8 m n kb real FLOPs, the complex FLOP count.
// tc_pack_kernel writes Atil and Bhat K-major (128 floats per row, hi and lo parts) once per
// step; tc_update_kernel loads 128 x 32 / 256 x 32 float boxes of them with TMA (128-byte
// swizzle) into a 2-stage shared-memory ring and issues tcgen05.mma kind::tf32 (M = 128,
// N = 256, K = 8) from one thread; the 128 x 256 FP32 accumulator lives in TMEM (256 columns);
// four epilogue warps move it out with tcgen05.ld into shared memory and TMA reduce-add it (negated)
// onto F, so the C tile's read-modify-write is done by L2 asynchronously to the SM.
//
// Warp roles (192 threads): warp 0 = TMA producer, warp 1 = TMEM owner + MMA issuer,
// warps 2..5 = epilogue (TMEM lane quarters 2, 3, 0, 1).  Every mbarrier wait is bounded; on
// expiry the CTA records an error flag, drains what it issued, frees TMEM and returns.

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace b200 {
namespace {

constexpr int kTM = 128;          // real rows per tile (64 complex rows)
constexpr int kTN = kTcTileCols;  // columns per tile
constexpr int kTK = kTcChunk;     // floats per K chunk (128 bytes: one 128-byte swizzle span)
constexpr int kKReal = 2 * kNb;   // 128 real K per step
constexpr int kChunks = kKReal / kTK;
// Two 96 KB stages.  A box row is one TMA request, so 128-byte rows move twice the bytes per
// request of 64-byte ones; the TMA request rate, not L2 bandwidth, bounds the operand stream.
constexpr int kStages = 2;
constexpr int kABytes = kTM * kTK * 4;  // 16 KB
constexpr int kBBytes = kTN * kTK * 4;  // 32 KB
constexpr int kStageBytes = 2 * kABytes + 2 * kBBytes;
constexpr int kPieceCols = kTcPieceCols;  // epilogue: columns per TMA reduce-add
constexpr int kAccCols = kTN;           // TMEM columns per accumulator (two of them)
constexpr long kWaitBound = 1L << 22;

struct __align__(1024) TcSmem {
  float a_hi[kStages][kTM * kTK];
  float a_lo[kStages][kTM * kTK];
  float b_hi[kStages][kTN * kTK];
  float b_lo[kStages][kTN * kTK];
  float ep[2][kPieceCols * kTM];  // epilogue staging, [column][128 real rows]
  unsigned long long full[kStages];
  unsigned long long empty[kStages];
  unsigned long long acc_full[2];
  unsigned long long acc_empty[2];
  unsigned long long drain;
  unsigned tmem_base;
  volatile int abort;
  volatile int ep_ok;  // the epilogue issuer's last accumulator wait succeeded
};

__device__ __forceinline__ unsigned su32(const void *p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false if the bound expired.
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity) {
  for (long i = 0; i < kWaitBound; ++i)
    if (mbar_try(b, parity)) return true;
  return false;
}
// The wait for work already in flight after a wait ran out: the far longer drain bound.
__device__ __forceinline__ void mbar_drain(unsigned long long *b, unsigned parity) {
  for (long i = 0; i < kDrainPolls; ++i)
    if (mbar_try(b, parity)) return;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(su32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(su32(bar))
      : "memory");
}

// K-major, 128-byte-swizzled operand: rows 128 B apart, 8-row groups 1024 B apart (SBO),
// LBO unused (1), descriptor version 1 (sm_100), layout type 2 = SWIZZLE_128B.
__device__ __forceinline__ uint64_t smem_desc(const void *p) {
  const uint64_t addr = su32(p);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;
  d |= (uint64_t)1 << 16;              // LBO (ignored for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;    // SBO
  d |= (uint64_t)1 << 46;              // version
  d |= (uint64_t)2 << 61;              // SWIZZLE_128B
  return d;
}

// kind::tf32, D = F32, A = B = TF32, both K-major, N = 256, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTN >> 3) << 17) |
                            ((uint32_t)(kTM >> 4) << 24);

__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{ .reg .pred p; setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p; }" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}

__device__ __forceinline__ float tf32_hi(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Tiles of one launch, sized for the largest trailing block of the wave: per job, part 0 covers
// every tile (tm, tn) in the order ((z * tiles_m) + tm) * tiles_n + tn (tn fastest, so consecutive
// CTAs share the A row block); part 1 only tile (0, 0), which holds the next step's diagonal
// block; part 2 all the others, in the same order.  Tiles outside a job's own trailing block are
// skipped identically by every role.
struct TileSpace {
  int tiles_m, tiles_n, per_job, total, part;
};
__device__ __forceinline__ bool tile_of(const JobDev *jobs, const TileSpace &ts, int k, int t, int &z, int &row0,
                                        int &col0, int &kb) {
  z = t / ts.per_job;
  const int i = t - z * ts.per_job;
  int tm, tn;
  if (ts.part == 0) {
    tm = i / ts.tiles_n;
    tn = i - tm * ts.tiles_n;
  } else if (ts.part == 1) {
    tm = 0;
    tn = 0;
  } else if (ts.part == 2) {
    tm = (i + 1) / ts.tiles_n;
    tn = i + 1 - tm * ts.tiles_n;
  } else if (ts.part == 3) {
    tm = i;
    tn = 0;
  } else {
    tm = i / (ts.tiles_n - 1);
    tn = 1 + i - tm * (ts.tiles_n - 1);
  }
  const JobDev &J = jobs[z];
  if (k >= J.n) return false;
  kb = min(kNb, J.n - k);
  const int rest = J.N - k - kb;
  row0 = tm * kTM;
  col0 = tn * kTN;
  return row0 < 2 * rest && col0 < rest;
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}

// Persistent: one CTA per SM loops over the launch's tiles.  Warp 0 (one thread) streams the
// operand chunks through a 2-stage ring; warp 1 owns TMEM (2 x 256 columns) and issues the MMAs
// of tile i into accumulator i % 2; warps 2..5 drain the other accumulator meanwhile (tcgen05.ld ->
// negated -> shared-memory staging -> TMA reduce-add onto F), so one tile's epilogue overlaps
// the next tile's MMAs.
__global__ void __launch_bounds__(192, 1)
    tc_update_kernel(const __grid_constant__ CUtensorMap tA_hi, const __grid_constant__ CUtensorMap tA_lo,
                     const __grid_constant__ CUtensorMap tB_hi, const __grid_constant__ CUtensorMap tB_lo,
                     const __grid_constant__ CUtensorMap tF, const JobDev *__restrict__ jobs, int k, TileSpace ts,
                     int *err) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  // the dynamic window is 1024-aligned by the launch (extra 1 KB requested)
  TcSmem &sm = *reinterpret_cast<TcSmem *>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&sm.acc_full[a], 1);
      mbar_init(&sm.acc_empty[a], 4);  // one arrival per epilogue warp
    }
    mbar_init(&sm.drain, 1);
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&sm.tmem_base)),
                 "r"(2 * kAccCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sm.tmem_base;

  if (warp == 0) {
    if (lane == 0) {
      long g = 0;  // chunks issued
      for (int t = blockIdx.x; t < ts.total && !sm.abort; t += gridDim.x) {
        int z, row0, col0, kb;
        if (!tile_of(jobs, ts, k, t, z, row0, col0, kb)) continue;
        for (int c = 0; c < kChunks; ++c, ++g) {
          const int s = (int)(g % kStages);
          if (g >= kStages && !mbar_wait(&sm.empty[s], (unsigned)(((g / kStages) - 1) & 1))) {
            atomicOr(err, kErrUpdateWait);
            sm.abort = 1;
            break;
          }
          mbar_expect_tx(&sm.full[s], kStageBytes);
          tma_load_3d(sm.a_hi[s], &tA_hi, c * kTK, row0, z, &sm.full[s]);
          tma_load_3d(sm.a_lo[s], &tA_lo, c * kTK, row0, z, &sm.full[s]);
          tma_load_3d(sm.b_hi[s], &tB_hi, c * kTK, col0, z, &sm.full[s]);
          tma_load_3d(sm.b_lo[s], &tB_lo, c * kTK, col0, z, &sm.full[s]);
        }
      }
      // every issued load has landed before the CTA can exit (normally already true); a wait that
      // runs out is recorded and the wait goes on, far longer, so that no load can still be
      // writing into this CTA's shared memory when it exits
      for (long q = g > kStages ? g - kStages : 0; q < g; ++q)
        if (!mbar_wait(&sm.full[q % kStages], (unsigned)((q / kStages) & 1))) {
          atomicOr(err, kErrUpdateWait);
          mbar_drain(&sm.full[q % kStages], (unsigned)((q / kStages) & 1));
        }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      long g = 0;
      int li = 0;
      for (int t = blockIdx.x; t < ts.total && !sm.abort; t += gridDim.x) {
        int z, row0, col0, kb;
        if (!tile_of(jobs, ts, k, t, z, row0, col0, kb)) continue;
        const int a = li & 1;
        if (li >= 2 && !mbar_wait(&sm.acc_empty[a], (unsigned)(((li >> 1) - 1) & 1))) {
          atomicOr(err, kErrUpdateWait);
          sm.abort = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(a * kAccCols);
        bool ok = true;
        for (int c = 0; c < kChunks; ++c, ++g) {
          const int s = (int)(g % kStages);
          if (!mbar_wait(&sm.full[s], (unsigned)((g / kStages) & 1))) {
            atomicOr(err, kErrUpdateWait);
            sm.abort = 1;
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint64_t dah = smem_desc(sm.a_hi[s]), dal = smem_desc(sm.a_lo[s]);
          const uint64_t dbh = smem_desc(sm.b_hi[s]), dbl = smem_desc(sm.b_lo[s]);
#pragma unroll
          for (int kk = 0; kk < kTK / 8; ++kk) {
            const uint64_t off = (uint64_t)((kk * 32) >> 4);  // 8 tf32 = 32 bytes along K
            const uint32_t acc0 = (c > 0 || kk > 0) ? 1u : 0u;
            umma_tf32(d, dal + off, dbh + off, acc0);
            umma_tf32(d, dah + off, dbl + off, 1u);
            umma_tf32(d, dah + off, dbh + off, 1u);
          }
          umma_commit(&sm.empty[s]);
        }
        if (!ok) break;
        umma_commit(&sm.acc_full[a]);
        ++li;
      }
      // the MMAs issued are complete before TMEM is released (the same keep-waiting rule)
      umma_commit(&sm.drain);
      if (!mbar_wait(&sm.drain, 0)) {
        atomicOr(err, kErrUpdateWait);
        mbar_drain(&sm.drain, 0);
      }
    }
  } else {
    // Epilogue, warps 2..5 -> TMEM lane quarter (warp % 4), 32 real rows each.  Each 32-column
    // piece of the accumulator is negated into a staging buffer (two, alternating) and added onto
    // F by one TMA reduce-add (cp.reduce.async.bulk.tensor .add.f32): the read-modify-write of the
    // C tile happens in L2, asynchronously to the SM.  Rows/columns of a tile beyond the trailing
    // block land in F's padding (rows/columns N..ld-1, never read) or are clipped at the tensor
    // bounds.
    const int q = warp & 3;
    const int rl = q * 32 + lane;  // real row within the tile
    const bool issuer = (warp == 2 && lane == 0);
    int li = 0, pcount = 0;
    // The four warps must take the same path through the named barriers below, so the loop runs
    // over the same tiles for all of them and the one wait is taken by the issuer, whose outcome
    // the others read after a barrier.
    for (int t = blockIdx.x; t < ts.total; t += gridDim.x) {
      int z, row0, col0, kb;
      if (!tile_of(jobs, ts, k, t, z, row0, col0, kb)) continue;
      const int a = li & 1;
      if (issuer) {
        const bool ok = mbar_wait(&sm.acc_full[a], (unsigned)((li >> 1) & 1));
        sm.ep_ok = ok ? 1 : 0;
        if (!ok) {
          atomicOr(err, kErrUpdateWait);
          sm.abort = 1;
        }
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
      if (!sm.ep_ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int fx = 2 * (k + kb) + row0;  // float row coordinate in F (multiple of 4)
      const int fy = k + kb + col0;        // column coordinate in F
      for (int piece = 0; piece < kTN / kPieceCols; ++piece, ++pcount) {
        float *ps = sm.ep[pcount & 1];
        if (issuer) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");  // ps is free again
        asm volatile("bar.sync 1, 128;" ::: "memory");
#pragma unroll
        for (int c16 = 0; c16 < kPieceCols; c16 += 16) {
          uint32_t v[16];
          const uint32_t taddr =
              tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * kAccCols + piece * kPieceCols + c16);
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
              "[%16];"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                "=r"(v[15])
              : "r"(taddr)
              : "memory");
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int j = 0; j < 16; ++j) ps[(c16 + j) * kTM + rl] = -__uint_as_float(v[j]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("bar.sync 1, 128;" ::: "memory");
        if (issuer) {
          asm volatile(
              "cp.reduce.async.bulk.tensor.3d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                  &tF),
              "r"(fx), "r"(fy + piece * kPieceCols), "r"(z), "r"(su32(ps))
              : "memory");
          asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
      }
      // this accumulator has been read out: the MMA warp may reuse it
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.acc_empty[a]);
      ++li;
    }
    if (issuer) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kAccCols) : "memory");
  }
}

// Pack the step's operands K-major with hi/lo TF32 split:
//   A (blocks [0, nA)): Atil rows 2r, 2r+1 for complex rows r of A21 = F[k+kb+r, k:k+kb]
//   B (blocks [nA, ..)): Bhat row c = W column F[k:k+kb, k+kb+c]
// Entries with K index >= 2 kb are zero (short last step).
__global__ void __launch_bounds__(256) tc_pack_kernel(const JobDev *__restrict__ jobs, int k, int nA,
                                                      float *__restrict__ a_hi, float *__restrict__ a_lo,
                                                      float *__restrict__ b_hi, float *__restrict__ b_lo,
                                                      size_t a_slot, size_t b_slot) {
  const JobDev &J = jobs[blockIdx.y];
  if (k >= J.n) return;
  const int kb = min(kNb, J.n - k);
  const int rest = J.N - k - kb;
  const float2 *F = static_cast<const float2 *>(J.F);
  const int ld = J.ld;
  const int tid = threadIdx.x;
  if ((int)blockIdx.x < nA) {
    // 4 complex rows per block, 64 threads (one per complex K index) per row
    const int r = blockIdx.x * 4 + (tid >> 6);
    const int p = tid & 63;
    if (r >= rest) return;
    float2 a = make_float2(0.f, 0.f);
    if (p < kb) a = F[(size_t)(k + kb + r) + (size_t)(k + p) * ld];
    const float hr = tf32_hi(a.x), hi_ = tf32_hi(a.y);
    const float lr = a.x - hr, li = a.y - hi_;
    float *h0 = a_hi + blockIdx.y * a_slot + (size_t)(2 * r) * kKReal;
    float *l0 = a_lo + blockIdx.y * a_slot + (size_t)(2 * r) * kKReal;
    // row 2r: (ar, -ai); row 2r+1: (ai, ar)
    reinterpret_cast<float2 *>(h0)[p] = make_float2(hr, -hi_);
    reinterpret_cast<float2 *>(l0)[p] = make_float2(lr, -li);
    reinterpret_cast<float2 *>(h0 + kKReal)[p] = make_float2(hi_, hr);
    reinterpret_cast<float2 *>(l0 + kKReal)[p] = make_float2(li, lr);
  } else {
    const int c = (blockIdx.x - nA) * 4 + (tid >> 6);
    const int p = tid & 63;
    if (c >= rest) return;
    float2 w = make_float2(0.f, 0.f);
    if (p < kb) w = F[(size_t)(k + p) + (size_t)(k + kb + c) * ld];
    const float hr = tf32_hi(w.x), hi_ = tf32_hi(w.y);
    reinterpret_cast<float2 *>(b_hi + blockIdx.y * b_slot + (size_t)c * kKReal)[p] = make_float2(hr, hi_);
    reinterpret_cast<float2 *>(b_lo + blockIdx.y * b_slot + (size_t)c * kKReal)[p] = make_float2(w.x - hr, w.y - hi_);
  }
}

}  // namespace

static_assert(sizeof(TcSmem) + 1024 <= 232448, "tc_update shared memory above the per-block limit");

size_t tc_smem_bytes() { return sizeof(TcSmem) + 1024; }

int tc_num_sms() {
  static int n = 0;
  if (n == 0) {
    int dev = 0, v = 0;
    n = (cudaGetDevice(&dev) == cudaSuccess &&
         cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
            ? v
            : 148;
  }
  return n;
}

cudaError_t launch_tc_pack(const TcMaps &maps, const JobDev *jobs, int njobs, int k, int max_N, cudaStream_t s,
                           bool pack_b) {
  const int rest = max_N - k - 1;  // upper bound of the trailing size over the wave
  if (rest <= 0) return cudaSuccess;
  const int nA = (rest + 3) / 4, nB = pack_b ? (rest + 3) / 4 : 0;
  tc_pack_kernel<<<dim3(nA + nB, njobs), 256, 0, s>>>(jobs, k, nA, maps.a_hi, maps.a_lo, maps.b_hi, maps.b_lo,
                                                      maps.a_slot, maps.b_slot);
  return cudaGetLastError();
}

cudaError_t launch_tc_update(const TcMaps &maps, const JobDev *jobs, int njobs, int k, int max_N, int *err,
                             cudaStream_t s, int part, int max_grid) {
  const int rest = max_N - k - 1;
  if (rest <= 0) return cudaSuccess;
  TileSpace ts;
  ts.tiles_n = (rest + kTN - 1) / kTN;
  ts.tiles_m = (2 * rest + kTM - 1) / kTM;
  ts.part = part;
  ts.per_job = part == 0   ? ts.tiles_m * ts.tiles_n
               : part == 1 ? 1
               : part == 2 ? ts.tiles_m * ts.tiles_n - 1
               : part == 3 ? ts.tiles_m
                           : ts.tiles_m * (ts.tiles_n - 1);
  ts.total = ts.per_job * njobs;
  if (ts.total <= 0) return cudaSuccess;
  int grid = ts.total < tc_num_sms() ? ts.total : tc_num_sms();
  if (max_grid > 0 && grid > max_grid) grid = max_grid;
  tc_update_kernel<<<grid, 192, tc_smem_bytes(), s>>>(maps.tA_hi, maps.tA_lo, maps.tB_hi, maps.tB_lo, maps.tF, jobs,
                                                      k, ts, err);
  return cudaGetLastError();
}

cudaError_t launch_tc_step(const TcMaps &maps, const JobDev *jobs, int njobs, int k, int max_N, int *err,
                           cudaStream_t s) {
  cudaError_t e = launch_tc_pack(maps, jobs, njobs, k, max_N, s, true);
  if (e != cudaSuccess) return e;
  return launch_tc_update(maps, jobs, njobs, k, max_N, err, s, 0, 0);
}

cudaError_t tc_prepare() {
  return ensure_smem(tc_update_kernel, (int)tc_smem_bytes());
}

}  // namespace b200
