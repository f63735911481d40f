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

#include <algorithm>
#include <cstdint>

#include "common.cuh"

namespace b200 {
namespace {

constexpr int kTM = 128;          // real rows per tile (64 complex rows)
constexpr int kTN = kTcTileCols;  // columns per tile
constexpr int kTK = kTcChunk;     // floats per K chunk (128 bytes: one 128-byte swizzle span)
constexpr int kStepChunks = 2 * kNb / kTK;  // K chunks of one 64-column step (128 real K)
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
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity, long bound = kWaitBound) {
  for (long i = 0; i < bound; ++i)
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
// CTAs share the A row block); part 1 tiles (0, 0) and (1, 0), the first 256-row tile of the pair
// kernel below, which holds the next step's diagonal block; part 2 all the others; part 3 the first
// tile column, part 4 the others.  Tiles outside a job's own trailing block are skipped
// identically by every role.  This kernel runs parts 1 and 3; the pair kernel parts 0, 2 and 4.
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
    tm = i;
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
                     int nch, int *err) {
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
        for (int c = 0; c < nch; ++c, ++g) {
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
        for (int c = 0; c < nch; ++c, ++g) {
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


// ---------------------------------------------------------------------------------------------
// The trailing update on CTA pairs (tcgen05 cta_group::2): one MMA of M = 256 x N = 256 x K = 8
// spans the two SMs of a pair, each CTA holding 128 rows of A and 128 columns of B in its shared
// memory and 128 rows of the accumulator in its TMEM.  Per SM this halves the B operand stream
// (64 KB instead of 96 KB per 32-float K chunk for the same MMA work), so three stages fit.
// Tiles are 256 real rows x 256 columns, handed out dynamically: the leader CTA (rank 0) takes
// the next tile from a per-launch counter and passes it through a ring in shared memory to its
// MMA and epilogue warps and to the peer's producer and epilogue warps; a pair that starts late
// (its SMs still held by the concurrent diagonal inverses) takes fewer tiles.
// Barriers: both CTAs' TMA loads complete on the leader's full[s] (the leader expects both
// halves); the leader's MMA commits arrive on empty[s], acc_full[a] and drain in both CTAs
// (multicast commit); both CTAs' epilogue warps arrive on the leader's acc_empty[a].  No load
// uses cluster multicast.  Every wait is bounded as in the single-CTA kernel.
// ---------------------------------------------------------------------------------------------
constexpr int kHalf = 128;            // A rows and B columns per CTA of a pair
constexpr int kPM = 2 * kHalf;        // real rows per pair tile
constexpr int kStages2 = 3;
constexpr int kBox2 = kHalf * kTK * 4;  // 16 KB
constexpr int kStageBytes2 = 4 * kBox2;  // one CTA's A hi/lo and B hi/lo boxes of a K chunk
constexpr int kTQ = 8;                 // tile ring depth

struct __align__(1024) Tc2Smem {
  float a_hi[kStages2][kHalf * kTK];
  float a_lo[kStages2][kHalf * kTK];
  float b_hi[kStages2][kHalf * kTK];
  float b_lo[kStages2][kHalf * kTK];
  float epw[4][2][kPieceCols * 32];  // per epilogue warp: two 32-column x 32-row staging buffers
  unsigned long long full[kStages2];
  unsigned long long empty[kStages2];
  unsigned long long acc_full[2];
  unsigned long long acc_empty[2];
  unsigned long long drain;
  unsigned long long tfull[kTQ];
  unsigned long long tempty[kTQ];
  int tq[kTQ];
  unsigned tmem_base;
  volatile int abort;
};
static_assert(sizeof(Tc2Smem) + 1024 <= 232448, "pair update shared memory above the per-block limit");
// readers of each tile-ring entry: the leader's MMA warp, both CTAs' four epilogue warps, the peer's producer
constexpr int kTileReaders = 1 + 4 + 1 + 4;

// kind::tf32, D = F32, A = B = TF32, both K-major, N = 256, M = 256 (the pair)
constexpr uint32_t kIdesc2 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTN >> 3) << 17) |
                             ((uint32_t)(kPM >> 4) << 24);

__device__ __forceinline__ unsigned cta_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// The shared::cluster address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ unsigned mapa(unsigned addr, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(unsigned cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ bool mbar_try_cluster(unsigned long long *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on a local barrier that the other CTA of the pair also arrives on.
__device__ __forceinline__ bool mbar_wait_cluster(unsigned long long *b, unsigned parity, long bound = kWaitBound) {
  for (long i = 0; i < bound; ++i)
    if (mbar_try_cluster(b, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_3d_pair(void *dst, const CUtensorMap *map, int x, int y, int z,
                                                 unsigned mbar_cluster) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
      "%4}], [%5];" ::"r"(su32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(mbar_cluster)
      : "memory");
}
__device__ __forceinline__ void umma_tf32_pair(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{ .reg .pred p; setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p; }" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc2), "r"(accumulate)
      : "memory");
}
// Arrives on `bar` in both CTAs of the pair once the MMAs issued so far have completed.
__device__ __forceinline__ void umma_commit_pair(unsigned long long *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          su32(bar)),
      "h"((unsigned short)3)
      : "memory");
}

struct TileSpace2 {
  int tiles_m, tiles_n, per_job, total, part;
};
// Pair tiles: part 0 all, part 2 all but (0, 0), part 4 those with tn >= 1; tn fastest.
__device__ __forceinline__ bool tile_of2(const JobDev *jobs, const TileSpace2 &ts, int k, int t, int &z, int &row0,
                                         int &col0, int &kb) {
  z = t / ts.per_job;
  const int i = t - z * ts.per_job;
  int tm, tn;
  if (ts.part == 0) {
    tm = i / ts.tiles_n;
    tn = i - tm * ts.tiles_n;
  } else if (ts.part == 2) {
    tm = (i + 1) / ts.tiles_n;
    tn = i + 1 - tm * ts.tiles_n;
  } else {
    tm = i / (ts.tiles_n - 1);
    tn = 1 + i - tm * (ts.tiles_n - 1);
  }
  const JobDev &J = jobs[z];
  if (k >= J.n) return false;
  kb = min(kNb, J.n - k);
  const int rest = J.N - k - kb;
  row0 = tm * kPM;
  col0 = tn * kTN;
  return row0 < 2 * rest && col0 < rest;
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(192, 1)
    tc_update2_kernel(const __grid_constant__ CUtensorMap tA_hi, const __grid_constant__ CUtensorMap tA_lo,
                      const __grid_constant__ CUtensorMap tB_hi, const __grid_constant__ CUtensorMap tB_lo,
                      const __grid_constant__ CUtensorMap tFw, const JobDev *__restrict__ jobs, int k, TileSpace2 ts,
                      int nch, int *counter, int *err) {
  extern __shared__ __align__(1024) unsigned char tc2_raw[];
  Tc2Smem &sm = *reinterpret_cast<Tc2Smem *>((reinterpret_cast<uintptr_t>(tc2_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned rank = cta_rank();

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages2; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&sm.acc_full[a], 1);
      mbar_init(&sm.acc_empty[a], 8);  // the four epilogue warps of each CTA
    }
    mbar_init(&sm.drain, 1);
    for (int q = 0; q < kTQ; ++q) {
      mbar_init(&sm.tfull[q], 1);
      mbar_init(&sm.tempty[q], kTileReaders);
    }
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&sm.tmem_base)),
                 "r"(2 * kAccCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  cluster_sync();  // the peer's barriers exist before any remote arrive or load signal
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sm.tmem_base;

  if (warp == 0) {
    if (lane == 0) {
      long g = 0;
      // this CTA's share of a pair tile's K chunks: A rows and B columns [128 rank, +128)
      auto load_tile = [&](int t) -> bool {
        int z, row0, col0, kb;
        tile_of2(jobs, ts, k, t, z, row0, col0, kb);
        const int ra = row0 + (int)rank * kHalf, cb = col0 + (int)rank * kHalf;
        for (int c = 0; c < nch; ++c, ++g) {
          const int s = (int)(g % kStages2);
          if (g >= kStages2 && !mbar_wait(&sm.empty[s], (unsigned)(((g / kStages2) - 1) & 1))) {
            atomicOr(err, kErrUpdateWait);
            sm.abort = 1;
            return false;
          }
          if (rank == 0) mbar_expect_tx(&sm.full[s], 2 * kStageBytes2);
          const unsigned fb = mapa(su32(&sm.full[s]), 0);
          tma_load_3d_pair(sm.a_hi[s], &tA_hi, c * kTK, ra, z, fb);
          tma_load_3d_pair(sm.a_lo[s], &tA_lo, c * kTK, ra, z, fb);
          tma_load_3d_pair(sm.b_hi[s], &tB_hi, c * kTK, cb, z, fb);
          tma_load_3d_pair(sm.b_lo[s], &tB_lo, c * kTK, cb, z, fb);
        }
        return true;
      };
      if (rank == 0) {
        // The leader hands out tiles two ahead of its own loads: the counter's round trip for the
        // tile after next overlaps the current tile's loads, and the peer knows its next tile
        // before it needs it.  Published: the tiles in order, then -1.
        int pub = 0;
        auto publish = [&](int t) -> bool {
          const int q = pub % kTQ;
          if (pub >= kTQ && !mbar_wait_cluster(&sm.tempty[q], (unsigned)(((pub / kTQ) - 1) & 1))) {
            atomicOr(err, kErrUpdateWait);
            sm.abort = 1;
            return false;
          }
          sm.tq[q] = t;
          asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(mapa(su32(&sm.tq[q]), 1)), "r"(t) : "memory");
          mbar_arrive(&sm.tfull[q]);
          mbar_arrive_cluster(mapa(su32(&sm.tfull[q]), 1));
          ++pub;
          return true;
        };
        auto resolve = [&](int c) -> int {  // the first tile at or after counter value c that has work
          int z, row0, col0, kb;
          while (c < ts.total && !tile_of2(jobs, ts, k, c, z, row0, col0, kb)) c = atomicAdd(counter, 1);
          return c < ts.total ? c : -1;
        };
        int cur = resolve(atomicAdd(counter, 1));
        bool ok = publish(cur);
        int nxt = -1;
        if (ok && cur >= 0) {
          nxt = resolve(atomicAdd(counter, 1));
          ok = publish(nxt);
        }
        while (ok && cur >= 0 && !sm.abort) {
          const int raw = nxt >= 0 ? atomicAdd(counter, 1) : ts.total;  // in flight during the loads
          if (!load_tile(cur)) break;
          int nn = -1;
          if (nxt >= 0) {
            nn = resolve(raw);
            if (!publish(nn)) break;
          }
          cur = nxt;
          nxt = nn;
        }
      } else {
        for (int it = 0;; ++it) {
          const int q = it % kTQ;
          if (!mbar_wait_cluster(&sm.tfull[q], (unsigned)((it / kTQ) & 1))) {
            atomicOr(err, kErrUpdateWait);
            sm.abort = 1;
            break;
          }
          const int t = sm.tq[q];
          mbar_arrive_cluster(mapa(su32(&sm.tempty[q]), 0));
          if (t < 0 || !load_tile(t)) break;
        }
      }
      // the leader's full barriers complete only with both CTAs' bytes: every issued load of the
      // pair has landed once the last stages are complete (the peer stays resident until then
      // through the final cluster barrier)
      if (rank == 0)
        for (long q = g > kStages2 ? g - kStages2 : 0; q < g; ++q)
          if (!mbar_wait(&sm.full[q % kStages2], (unsigned)((q / kStages2) & 1))) {
            atomicOr(err, kErrUpdateWait);
            mbar_drain(&sm.full[q % kStages2], (unsigned)((q / kStages2) & 1));
          }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      if (rank == 0) {
        long g = 0;
        int li = 0, it = 0;
        for (;;) {
          const int q = it % kTQ;
          if (!mbar_wait_cluster(&sm.tfull[q], (unsigned)((it / kTQ) & 1))) {
            atomicOr(err, kErrUpdateWait);
            sm.abort = 1;
            break;
          }
          const int t = sm.tq[q];
          mbar_arrive(&sm.tempty[q]);
          ++it;
          if (t < 0) break;
          const int a = li & 1;
          if (li >= 2 && !mbar_wait_cluster(&sm.acc_empty[a], (unsigned)(((li >> 1) - 1) & 1))) {
            atomicOr(err, kErrUpdateWait);
            sm.abort = 1;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t d = tmem + (uint32_t)(a * kAccCols);
          bool ok = true;
          for (int c = 0; c < nch; ++c, ++g) {
            const int s = (int)(g % kStages2);
            if (!mbar_wait(&sm.full[s], (unsigned)((g / kStages2) & 1))) {
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
              const uint64_t off = (uint64_t)((kk * 32) >> 4);
              const uint32_t acc0 = (c > 0 || kk > 0) ? 1u : 0u;
              umma_tf32_pair(d, dal + off, dbh + off, acc0);
              umma_tf32_pair(d, dah + off, dbl + off, 1u);
              umma_tf32_pair(d, dah + off, dbh + off, 1u);
            }
            umma_commit_pair(&sm.empty[s]);
          }
          if (!ok) break;
          umma_commit_pair(&sm.acc_full[a]);
          ++li;
        }
        umma_commit_pair(&sm.drain);
      }
      // both CTAs: the pair's MMAs are complete before TMEM is released
      if (!mbar_wait(&sm.drain, 0, kDrainPolls)) atomicOr(err, kErrUpdateWait);
    }
  } else {
    // Epilogue, warps 2..5 of each CTA, each on its own: warp w reads TMEM lanes 32 (w % 4) .. +31
    // (its 32 of the CTA's 128 rows), 32 columns at a time, negates them into one of its two
    // staging buffers and adds them onto F with its own TMA reduce-add (a 32 x 32 box).  No
    // barriers between the warps: each reads the tile ring and the accumulator barrier itself and
    // tells the leader's MMA warp when its rows of an accumulator are read out.
    const int q4 = warp & 3;
    float(*wbuf)[kPieceCols * 32] = sm.epw[q4];
    const bool lead = lane == 0;
    int li = 0, pcount = 0;
    for (int it = 0;; ++it) {
      int t = -1;
      if (lead) {
        const int q = it % kTQ;
        if (mbar_wait_cluster(&sm.tfull[q], (unsigned)((it / kTQ) & 1))) {
          t = sm.tq[q];
          if (rank == 0) mbar_arrive(&sm.tempty[q]);
          else mbar_arrive_cluster(mapa(su32(&sm.tempty[q]), 0));
          if (t >= 0 && !mbar_wait(&sm.acc_full[li & 1], (unsigned)((li >> 1) & 1))) {
            atomicOr(err, kErrUpdateWait);
            sm.abort = 1;
            t = -1;
          }
        } else {
          atomicOr(err, kErrUpdateWait);
          sm.abort = 1;
        }
      }
      t = __shfl_sync(0xffffffffu, t, 0);
      if (t < 0) break;
      int z, row0, col0, kb;
      tile_of2(jobs, ts, k, t, z, row0, col0, kb);
      const int rest = jobs[z].N - k - kb;
      const int a = li & 1;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int wr0 = row0 + (int)rank * kHalf + q4 * 32;  // this warp's first real row of the tile
      const bool rows_in = wr0 < 2 * rest;
      const int fx = 2 * (k + kb) + wr0;
      const int fy = k + kb + col0;
      for (int piece = 0; piece < kTN / kPieceCols; ++piece, ++pcount) {
        float *ps = wbuf[pcount & 1];
        if (lead) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");  // ps is free again
        __syncwarp();
        uint32_t v[32];
        const uint32_t taddr = tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(a * kAccCols + piece * kPieceCols);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
            "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
              "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
              "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
              "=r"(v[30]), "=r"(v[31])
            : "r"(taddr)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < 32; ++j) ps[j * 32 + lane] = -__uint_as_float(v[j]);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        // pieces wholly outside the trailing block (this warp's rows past it, or columns past it)
        // are not written; their group is committed empty, so that the wait above always covers
        // the reduce that last read the staging buffer
        if (lead) {
          if (rows_in && col0 + piece * kPieceCols < rest)
            asm volatile(
                "cp.reduce.async.bulk.tensor.3d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                    &tFw),
                "r"(fx), "r"(fy + piece * kPieceCols), "r"(z), "r"(su32(ps))
                : "memory");
          asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
      }
      // this warp's rows of the accumulator are read out: tell the leader's MMA warp
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lead) {
        if (rank == 0) mbar_arrive(&sm.acc_empty[a]);
        else mbar_arrive_cluster(mapa(su32(&sm.acc_empty[a]), 0));
      }
      ++li;
    }
    if (lead) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  cluster_sync();  // neither CTA frees TMEM or exits while the other may still use its memory
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kAccCols) : "memory");
  }
}

// Pack the operands K-major with hi/lo TF32 split, for the update of the trailing block of step
// k_last (rows and columns from R0 = k_last + kb_last) by nblk consecutive steps kA, kA + 64, ...:
//   A (blocks [0, nA)): Atil rows 2r, 2r+1 for complex rows r of [A21_kA | A21_kA+64 | ...],
//                       A21_q = F[R0 + r, q : q + kb_q]
//   B (blocks [nA, ..)): Bhat row c = [W_kA ; W_kA+64 ; ...] column R0 + c (W stored in F's rows)
// K index 2 (64 q + p) + {0, 1} holds step q's column p; entries with p >= kb_q are zero.  Rows are
// kTcKMax floats; the update reads the first nblk * 128 of them.
__global__ void __launch_bounds__(256) tc_pack_kernel(const JobDev *__restrict__ jobs, int kA, int nblk, int k_last,
                                                      int nA, float *__restrict__ a_hi, float *__restrict__ a_lo,
                                                      float *__restrict__ b_hi, float *__restrict__ b_lo,
                                                      size_t a_slot, size_t b_slot) {
  const JobDev &J = jobs[blockIdx.y];
  if (k_last >= J.n) return;
  const int R0 = k_last + min(kNb, J.n - k_last);
  const int rest = J.N - R0;
  const float2 *F = static_cast<const float2 *>(J.F);
  const int ld = J.ld;
  const int tid = threadIdx.x;
  const int kw = kNb * nblk;  // complex K of the update
  if ((int)blockIdx.x < nA) {
    // 4 complex rows per block, 64 threads per row, each over the row's K in steps of 64
    const int r = blockIdx.x * 4 + (tid >> 6);
    if (r >= rest) return;
    float *h0 = a_hi + blockIdx.y * a_slot + (size_t)(2 * r) * kTcKMax;
    float *l0 = a_lo + blockIdx.y * a_slot + (size_t)(2 * r) * kTcKMax;
    for (int p = tid & 63; p < kw; p += 64) {
      const int kq = kA + p;  // column of F
      float2 a = make_float2(0.f, 0.f);
      if (kq < J.n) a = F[(size_t)(R0 + r) + (size_t)kq * ld];
      const float hr = tf32_hi(a.x), hi_ = tf32_hi(a.y);
      const float lr = a.x - hr, li = a.y - hi_;
      // row 2r: (ar, -ai); row 2r+1: (ai, ar)
      reinterpret_cast<float2 *>(h0)[p] = make_float2(hr, -hi_);
      reinterpret_cast<float2 *>(l0)[p] = make_float2(lr, -li);
      reinterpret_cast<float2 *>(h0 + kTcKMax)[p] = make_float2(hi_, hr);
      reinterpret_cast<float2 *>(l0 + kTcKMax)[p] = make_float2(li, lr);
    }
  } else {
    const int c = (blockIdx.x - nA) * 4 + (tid >> 6);
    if (c >= rest) return;
    for (int p = tid & 63; p < kw; p += 64) {
      const int kq = kA + p;  // row of F
      float2 w = make_float2(0.f, 0.f);
      if (kq < J.n) w = F[(size_t)kq + (size_t)(R0 + c) * ld];
      const float hr = tf32_hi(w.x), hi_ = tf32_hi(w.y);
      reinterpret_cast<float2 *>(b_hi + blockIdx.y * b_slot + (size_t)c * kTcKMax)[p] = make_float2(hr, hi_);
      reinterpret_cast<float2 *>(b_lo + blockIdx.y * b_slot + (size_t)c * kTcKMax)[p] = make_float2(w.x - hr, w.y - hi_);
    }
  }
}

}  // namespace

static_assert(sizeof(TcSmem) + 1024 <= 232448, "tc_update shared memory above the per-block limit");

size_t tc_smem_bytes() { return sizeof(TcSmem) + 1024; }
size_t tc2_smem_bytes() { return sizeof(Tc2Smem) + 1024; }

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

cudaError_t launch_tc_pack(const TcMaps &maps, const JobDev *jobs, int njobs, int kA, int nblk, int k_last,
                           int max_N, cudaStream_t s, bool pack_b) {
  const int rest = max_N - k_last - 1;  // upper bound of the trailing size over the wave
  if (rest <= 0) return cudaSuccess;
  const int nA = (rest + 3) / 4, nB = pack_b ? (rest + 3) / 4 : 0;
  tc_pack_kernel<<<dim3(nA + nB, njobs), 256, 0, s>>>(jobs, kA, nblk, k_last, nA, maps.a_hi, maps.a_lo, maps.b_hi,
                                                      maps.b_lo, maps.a_slot, maps.b_slot);
  return cudaGetLastError();
}

cudaError_t launch_tc_update(const TcMaps &maps, const JobDev *jobs, int njobs, int k, int max_N, int *err,
                             cudaStream_t s, int part, int max_grid, int nblk) {
  const int rest = max_N - k - 1;
  if (rest <= 0) return cudaSuccess;
  if (nblk < 1 || nblk * 2 * kNb > kTcKMax) return cudaErrorInvalidValue;
  const int nch = nblk * kStepChunks;
  const int sms = max_grid > 0 ? std::min(max_grid, tc_num_sms()) : tc_num_sms();
  if (part == 0 || part == 2 || part == 4) {
    // the interior on CTA pairs, tiles handed out from the launch's counter
    TileSpace2 ts;
    ts.tiles_n = (rest + kTN - 1) / kTN;
    ts.tiles_m = (2 * rest + kPM - 1) / kPM;
    ts.part = part;
    ts.per_job = part == 0 ? ts.tiles_m * ts.tiles_n
                 : part == 2 ? ts.tiles_m * ts.tiles_n - 1
                             : ts.tiles_m * (ts.tiles_n - 1);
    ts.total = ts.per_job * njobs;
    if (ts.per_job <= 0 || ts.total <= 0) return cudaSuccess;
    const int slot = (k / kNb) * kTcCountersPerStep + part;
    if (maps.counters == nullptr || slot >= maps.counter_slots) return cudaErrorInvalidValue;
    const int pairs = std::max(1, std::min(ts.total, sms / 2));
    tc_update2_kernel<<<2 * pairs, 192, tc2_smem_bytes(), s>>>(maps.tA_hi, maps.tA_lo, maps.tB2_hi, maps.tB2_lo,
                                                               maps.tFw, jobs, k, ts, nch, maps.counters + slot, err);
    return cudaGetLastError();
  }
  TileSpace ts;
  ts.tiles_n = (rest + kTN - 1) / kTN;
  ts.tiles_m = (2 * rest + kTM - 1) / kTM;
  ts.part = part;
  ts.per_job = part == 1 ? 2 : ts.tiles_m;
  ts.total = ts.per_job * njobs;
  if (ts.total <= 0) return cudaSuccess;
  const int grid = std::min(ts.total, sms);
  tc_update_kernel<<<grid, 192, tc_smem_bytes(), s>>>(maps.tA_hi, maps.tA_lo, maps.tB_hi, maps.tB_lo, maps.tF, jobs,
                                                      k, ts, nch, err);
  return cudaGetLastError();
}

cudaError_t launch_tc_step(const TcMaps &maps, const JobDev *jobs, int njobs, int k, int max_N, int *err,
                           cudaStream_t s) {
  cudaError_t e = launch_tc_pack(maps, jobs, njobs, k, 1, k, max_N, s, true);
  if (e != cudaSuccess) return e;
  return launch_tc_update(maps, jobs, njobs, k, max_N, err, s, 0, 0);
}

cudaError_t launch_tc_counters_reset(const TcMaps &maps, cudaStream_t s) {
  if (maps.counters == nullptr) return cudaSuccess;
  return cudaMemsetAsync(maps.counters, 0, sizeof(int) * (size_t)maps.counter_slots, s);
}

cudaError_t tc_prepare() {
  const cudaError_t e = ensure_smem(tc_update_kernel, (int)tc_smem_bytes());
  if (e != cudaSuccess) return e;
  return ensure_smem(tc_update2_kernel, (int)tc2_smem_bytes());
}

}  // namespace b200
