// Dataflow block sweeps of the correction solve: FP32 factors, FP32 arithmetic, b <= 16.
//
// Same contract as the step-synchronous sweeps of sweep.cu (forward: Y_k = D_k R_k,
// R[k+kb:N] -= A21_k Y_k; backward: X_k (+)= Y_k, Y[0:k] -= W[0:k, k] Y_k, i.e. zgetrs on the
// block LU factors, zblock_lu_cpp.cpp:60-86), organised so that no CTA waits for the others to
// finish a step:
//
//  * One cluster of cs CTAs per job; the 64-row tile t of the right-hand side belongs to rank
//    t % cs for the whole sweep and stays in that CTA's shared memory (FP32, column-major),
//    so tile updates never leave the SM.
//  * The only value that crosses CTAs is the 64 x 16 block of the step (Y_k forward, the final
//    rows of block k backward).  The CTA owning the next block's tile updates that tile first,
//    produces the block and stores it into a ring slot of every CTA of the cluster (distributed
//    shared memory), then arrives on each CTA's `full` barrier of the slot.  A CTA starts step j
//    as soon as its slot is full; when it is done with the slot it arrives on the slot's `empty`
//    barrier in the CTA that produces the slot's next use.  Slot s of an ns-deep ring is always
//    produced by the same rank (cs divides ns), so both barriers count plain phases.
//  * Operand panels (A21, D or W; 64 rows x 32 columns per unit) stream through a ring of
//    shared-memory stages several units ahead, one TMA load per unit issued by one thread.  The D_(j+1) multiply of the forward sweep is just two more units in
//    the producing CTA's stream.
//  * Each unit's 32 columns are split over four groups of 64 threads; a thread holds a 4 x 4
//    register tile of the 64 x 16 product (6 shared-memory loads per 64 FMAs), and the four
//    partial sums meet in shared memory at the end of a tile.
//
// Every barrier wait is bounded.  A wait that runs out marks the job diverged (JobDev::conv),
// which also ends the other CTAs' waits, and the refinement re-solves that job in FP64.

#include <cuda_runtime.h>

#include "cluster.cuh"
#include "common.cuh"
#include "cplx.cuh"

namespace b200 {
namespace {

using namespace cx;
using namespace cl;

constexpr int kThreads = 256;             // compute threads (8 warps)
constexpr int kBlock = kThreads + 32;     // and the producer warp
constexpr int kWarps = kThreads / 32;
constexpr int kCols = 16;                  // right-hand-side columns held (b <= 16)
constexpr int kUnit = 32;                  // factor columns per pipeline unit
constexpr int kUnitElems = 64 * kUnit;
constexpr unsigned kUnitBytes = kUnitElems * 8;  // one TMA box: 128 floats x 32 columns
constexpr int kStages = 4;                 // operand ring depth (units)
constexpr int kLgStages = 2;
constexpr int kGroups = 4;                 // column groups of a unit (8 columns each)
constexpr int kTileElems = 64 * kCols;     // one 64-row tile of the right-hand side
constexpr int kMaxSmem = 227 * 1024;
constexpr long kFlowWaitBound = 1L << 22;  // barrier polls before a wait gives up

// Shared-memory layout (byte offsets) for cluster size cs and `own` resident tiles per CTA.
struct FlowLayout {
  int ns, own;
  int ring, part, slots, tiles, bars, total;  // bars: full[ns], empty[ns], ring_full/empty[kStages]
};
__host__ __device__ inline FlowLayout flow_layout(int cs, int own) {
  FlowLayout L;
  L.ns = cs > 4 ? cs : 4;
  L.own = own;
  L.ring = 0;
  L.part = L.ring + kStages * kUnitElems * 8;
  L.slots = L.part + kGroups * kTileElems * 8;
  L.tiles = L.slots + L.ns * kTileElems * 8;
  L.bars = L.tiles + own * kTileElems * 8;
  L.total = L.bars + (2 * L.ns + 2 * kStages) * 8;
  return L;
}

// Register tile of a thread: rows rq + 16 i (i < 4) and columns 4 cq + m (m < 4) of the 64 x 16
// product, over its group's columns kk of each unit.  Per column kk a warp loads 4 operand values
// and 2 x 4 right-hand-side values per lane for 64 FMAs, which balances the shared-memory pipe
// (128 B of register payload per clock, broadcasts included) against the FMA pipe.
struct Frag {
  float2 v[4][4];  // [i][m]
};

// acc += A[kk][row] * Y[y0 + kk][col] over kk in [k0, k1) of unit A, with the right-hand side
// row-major (a ring slot).
__device__ __forceinline__ void row_step(Frag &acc, const float2 *__restrict__ A, const float2 *__restrict__ Y,
                                         int y0, int kk, int rq, int cq) {
  float2 a[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) a[i] = A[kk * 64 + rq + 16 * i];
  const float4 *y = reinterpret_cast<const float4 *>(Y + (y0 + kk) * kCols + 4 * cq);
  const float4 y01 = y[0], y23 = y[1];
  const float2 yv[4] = {make_float2(y01.x, y01.y), make_float2(y01.z, y01.w), make_float2(y23.x, y23.y),
                        make_float2(y23.z, y23.w)};
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int m = 0; m < 4; ++m) acc.v[i][m] = cfma(a[i], yv[m], acc.v[i][m]);
}
__device__ __forceinline__ void product_rows(Frag &acc, const float2 *__restrict__ A, const float2 *__restrict__ Y,
                                             int y0, int k0, int k1, int rq, int cq) {
  if (k1 - k0 == kUnit / kGroups) {
#pragma unroll
    for (int i = 0; i < kUnit / kGroups; ++i) row_step(acc, A, Y, y0, k0 + i, rq, cq);
  } else {
    for (int kk = k0; kk < k1; ++kk) row_step(acc, A, Y, y0, kk, rq, cq);
  }
}
// The same with the right-hand side column-major (a resident tile, Yc[c * 64 + row]).
__device__ __forceinline__ void col_step(Frag &acc, const float2 *__restrict__ A, const float2 *__restrict__ Yc,
                                         int y0, int kk, int rq, int cq) {
  float2 a[4], yv[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) a[i] = A[kk * 64 + rq + 16 * i];
#pragma unroll
  for (int m = 0; m < 4; ++m) yv[m] = Yc[(4 * cq + m) * 64 + y0 + kk];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int m = 0; m < 4; ++m) acc.v[i][m] = cfma(a[i], yv[m], acc.v[i][m]);
}
__device__ __forceinline__ void product_cols(Frag &acc, const float2 *__restrict__ A, const float2 *__restrict__ Yc,
                                             int y0, int k0, int k1, int rq, int cq) {
  if (k1 - k0 == kUnit / kGroups) {
#pragma unroll
    for (int i = 0; i < kUnit / kGroups; ++i) col_step(acc, A, Yc, y0, k0 + i, rq, cq);
  } else {
    for (int kk = k0; kk < k1; ++kk) col_step(acc, A, Yc, y0, kk, rq, cq);
  }
}

__device__ __forceinline__ void zero(Frag &acc) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int m = 0; m < 4; ++m) acc.v[i][m] = make_float2(0.f, 0.f);
}
// Partial sums of group g, column-major per group: part[(g * 16 + col) * 64 + row].
__device__ __forceinline__ void store_partials(float2 *part, const Frag &acc, int g, int rq, int cq) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int m = 0; m < 4; ++m) part[(g * kCols + 4 * cq + m) * 64 + rq + 16 * i] = acc.v[i][m];
}
__device__ __forceinline__ float2 sum_partials(const float2 *part, int c, int row) {
  float2 s = part[c * 64 + row];
#pragma unroll
  for (int g = 1; g < kGroups; ++g) {
    const float2 v = part[(g * kCols + c) * 64 + row];
    s.x += v.x;
    s.y += v.y;
  }
  return s;
}

// The job's abort word: JobDev::conv (null for an initial solve without refinement state).
__device__ __forceinline__ bool job_aborted(const int *conv) {
  return conv != nullptr && *reinterpret_cast<volatile const int *>(conv) == kDiverged;
}
__device__ __forceinline__ void job_abort(int *conv) {
  if (conv != nullptr) atomicExch(conv, kDiverged);
}
// Barrier 1 over the 256 compute threads (the producer warp runs on its own).
__device__ __forceinline__ void compute_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }
// The same barrier with an AND vote: true for every compute thread when p held for all of them.
__device__ __forceinline__ bool compute_and(bool p) {
  unsigned r;
  asm volatile(
      "{ .reg .pred a, b; setp.ne.u32 a, %1, 0; bar.red.and.pred b, 1, 256, a; selp.u32 %0, 1, 0, b; }"
      : "=r"(r)
      : "r"((unsigned)p)
      : "memory");
  return r != 0;
}
// Bounded wait of this thread for the phase of the given parity of a barrier of this CTA; false
// when the bound ran out or the job was aborted.
__device__ __forceinline__ bool wait_phase(unsigned long long *bar, unsigned parity, const int *conv) {
  for (long i = 0; i < kFlowWaitBound; ++i) {
    if (mbar_try_cluster(bar, parity)) return true;
    if ((i & 1023) == 1023 && job_aborted(conv)) return false;
  }
  return false;
}
// The same for every compute thread, with a uniform outcome.
__device__ __forceinline__ bool cta_wait(unsigned long long *bar, unsigned parity, const int *conv) {
  return compute_and(wait_phase(bar, parity, conv));
}

// Producer rank of forward step j (the owner of tile j) and of backward step s (the owner of the
// tile of block s; p0 = last block's tile + 1 so that step 0, the central block, maps like the
// others).  Both are periodic in cs, hence in ns.
// (cs is a power of two; csm = cs - 1.)
__device__ __forceinline__ int fwd_producer(int j, int csm) { return j & csm; }
__device__ __forceinline__ int bwd_producer(int s, int p0, int csm) { return (p0 - s) & csm; }

// Work items of one CTA in the forward sweep, in consumption order: for each step j, the A21
// units of its own tiles at or below the block (ascending, so tile j + 1 comes first), and right
// after tile j + 1, when it owns it, the D units of block j + 1.  Rank 0 starts with the D units
// of block 0 (step -1).
struct FwdItems {
  int n, N, cs, csm, q, nsteps, T;
  int j, t, h, kb;
  bool d, fin;
  __device__ void begin() {
    fin = false;
    if (q == 0) {
      j = -1;
      t = 0;
      h = 0;
      kb = 0;
      d = true;
      return;
    }
    seek(0);
  }
  __device__ int width() const { return d ? min(64, n - 64 * (j + 1)) : kb; }
  __device__ int units() const { return (width() + kUnit - 1) / kUnit; }
  __device__ int ncol() const { return min(kUnit, width() - h * kUnit); }
  __device__ int row0() const { return d ? 64 * (j + 1) : 64 * t; }
  __device__ int col0() const { return (d ? 64 * (j + 1) : 64 * j) + h * kUnit; }
  __device__ void seek(int js) {
    for (j = js; j < nsteps; ++j) {
      kb = min(64, n - 64 * j);
      const int tlo = (64 * j + kb) / 64;  // tile holding the first row below the block
      t = tlo + ((q - tlo) & csm);
      if (t < T) {
        h = 0;
        d = false;
        return;
      }
    }
    fin = true;
  }
  __device__ void advance() {
    t += cs;
    if (t < T) return;
    seek(j + 1);
  }
  __device__ void next() {
    if (++h < units()) return;
    h = 0;
    if (d) {
      if (j < 0) {
        seek(0);
        return;
      }
      d = false;
      advance();
      return;
    }
    if (t == j + 1 && j + 1 < nsteps) {
      d = true;
      return;
    }
    advance();
  }
};

// Work items of one CTA in the backward sweep: step 0 is the central block (k = n, kb = b),
// step s >= 1 the block at k = kstart - 64 (s - 1); the W units of the own tiles above the block,
// descending, so the tile of the next block comes first.
struct BwdItems {
  int n, b, cs, csm, q, kstart, nsteps;
  int s, k, kb, t, h;
  bool fin;
  __device__ int kof(int ss) const { return ss == 0 ? n : kstart - 64 * (ss - 1); }
  __device__ void begin() {
    fin = false;
    seek(0);
  }
  __device__ int units() const { return (kb + kUnit - 1) / kUnit; }
  __device__ int ncol() const { return min(kUnit, kb - h * kUnit); }
  __device__ int row0() const { return 64 * t; }
  __device__ int col0() const { return k + h * kUnit; }
  __device__ void seek(int ss) {
    for (s = ss; s < nsteps; ++s) {
      k = kof(s);
      kb = s == 0 ? b : min(64, n - k);
      if (k == 0) continue;
      const int ttop = (k - 1) / 64;  // highest tile with rows above the block
      t = ttop - ((ttop - q) & csm);
      if (t >= 0) {
        h = 0;
        return;
      }
    }
    fin = true;
  }
  __device__ void next() {
    if (++h < units()) return;
    h = 0;
    t -= cs;
    if (t >= 0) return;
    seek(s + 1);
  }
};

// Shared-memory views of one CTA.
struct FlowSmem {
  float2 *ring, *part, *slots, *tiles;
  unsigned long long *full, *empty, *ring_full, *ring_empty;
  __device__ FlowSmem(unsigned char *sm, const FlowLayout &L)
      : ring(reinterpret_cast<float2 *>(sm + L.ring)),
        part(reinterpret_cast<float2 *>(sm + L.part)),
        slots(reinterpret_cast<float2 *>(sm + L.slots)),
        tiles(reinterpret_cast<float2 *>(sm + L.tiles)),
        full(reinterpret_cast<unsigned long long *>(sm + L.bars)),
        empty(reinterpret_cast<unsigned long long *>(sm + L.bars) + L.ns),
        ring_full(reinterpret_cast<unsigned long long *>(sm + L.bars) + 2 * L.ns),
        ring_empty(reinterpret_cast<unsigned long long *>(sm + L.bars) + 2 * L.ns + kStages) {}
};

// Barriers: full[s] completes a phase when the 8 compute warps of the slot's producer have stored
// the block (or, for a slot filled by the CTA itself, when it arrives 8 times); empty[s] when all
// cs CTAs are done with the slot's current use; ring_full[s] when the TMA load of the operand
// unit in ring stage s has landed; ring_empty[s] when the 8 compute warps are done with it.
__device__ __forceinline__ void init_barriers(const FlowSmem &S, int ns, int cs) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < ns; ++s) {
      mbar_init(S.full + s, kWarps);
      mbar_init(S.empty + s, cs);
    }
    for (int s = 0; s < kStages; ++s) {
      mbar_init(S.ring_full + s, 1);
      mbar_init(S.ring_empty + s, kWarps);
    }
    fence_mbar_init();
  }
}

// The producer warp's lane 0: streams the CTA's units, in consumption order, into ring stage
// v % kStages by one TMA load each (the factor slot's 64 x 32 box), reusing a stage once the 8
// compute warps have released it; then waits for its last loads, so that none lands after the CTA
// has left.
template <class Items>
__device__ void produce_units(Items pf, const FlowSmem &S, const CUtensorMap *map, int slot, int *conv) {
  int issued = 0;
  bool ok = true;
  for (; !pf.fin; pf.next(), ++issued) {
    const int st = issued & (kStages - 1);
    if (issued >= kStages && !wait_phase(S.ring_empty + st, ((issued >> kLgStages) - 1) & 1, conv)) {
      ok = false;
      break;
    }
    mbar_expect_tx(S.ring_full + st, kUnitBytes);
    tma_load_3d(S.ring + st * kUnitElems, map, 2 * pf.row0(), pf.col0(), slot, S.ring_full + st);
  }
  if (!ok) job_abort(conv);
  for (int v = max(0, issued - kStages); v < issued; ++v)
    wait_phase(S.ring_full + (v & (kStages - 1)), (v >> kLgStages) & 1, nullptr);
}

// Compute side of one unit: wait for the load (bounded, per thread), multiply, release the stage.
// A thread whose wait ran out skips the arithmetic; the tile epilogue makes the outcome uniform.
__device__ __forceinline__ const float2 *unit_begin(const FlowSmem &S, int u, bool &okt, const int *conv) {
  okt = okt && wait_phase(S.ring_full + (u & (kStages - 1)), (u >> kLgStages) & 1, conv);
  return S.ring + (u & (kStages - 1)) * kUnitElems;
}
__device__ __forceinline__ void unit_end(const FlowSmem &S, int u) {
  __syncwarp();
  if ((threadIdx.x & 31) == 0) mbar_arrive_local(S.ring_empty + (u & (kStages - 1)), 1);
}

// Stores rows [0, 64) of a 64 x 16 block (thread: row tid / 4, columns 4 (tid % 4) .. + 3, zero
// for rows >= valid) into slot `slot` of every CTA of the cluster, then each compute warp's lane
// 0 arrives (release, cluster scope) on every CTA's full barrier of the slot.
__device__ __forceinline__ void push_block(const FlowSmem &S, int slot, int cs, int row, int c0, const float2 (&y)[4]) {
  float2 *dst = S.slots + slot * kTileElems + row * kCols + c0;
  const float4 v0 = make_float4(y[0].x, y[0].y, y[1].x, y[1].y);
  const float4 v1 = make_float4(y[2].x, y[2].y, y[3].x, y[3].y);
  for (int p = 0; p < cs; ++p) {
    st_remote(remote_u32(dst, p), v0);
    st_remote(remote_u32(dst + 2, p), v1);
  }
  __syncwarp();
  if ((threadIdx.x & 31) == 0)
    for (int p = 0; p < cs; ++p) mbar_arrive_cluster(S.full + slot, p);
}

// Grid (cs, njobs), cluster (cs, 1, 1), 288 threads: 8 compute warps and the producer warp.
// Refinement rounds only (the initial solve has B = 0 above the central block).  own_max:
// resident tiles per CTA (ceil(tiles / cs)).
__global__ void __launch_bounds__(kBlock, 1)
    forward_flow_kernel(const JobDev *__restrict__ jobs, int own_max, const __grid_constant__ CUtensorMap fmap) {
  const JobDev &J = jobs[blockIdx.y];
  // uniform over the cluster: the flag changes only between launches
  if (converged(J.conv) || J.n == 0 || J.inactive) return;
  const int q = cluster_rank(), cs = cluster_size(), csm = cs - 1, lcs = __ffs(cs) - 1;
  const FlowLayout L = flow_layout(cs, own_max);
  extern __shared__ __align__(128) unsigned char sm[];
  const FlowSmem S(sm, L);
  const int n = J.n, N = J.N, ld = J.ld, b = J.b, ns = L.ns, nsm = ns - 1, lns = __ffs(ns) - 1;
  int *conv = J.conv;
  const int tid = threadIdx.x, r = tid & 63, g = (tid >> 6) & 3, rq = tid & 15, cq = (tid >> 4) & 3;
  const int nsteps = (n + 63) / 64, T = (N + 63) / 64;

  init_barriers(S, ns, cs);
  // own tiles of R in FP32, zero past row N and column b
  if (tid < kThreads)
    for (int i = 0; q + i * cs < T; ++i) {
      const int t = q + i * cs;
      for (int e = tid; e < kTileElems; e += kThreads) {
        const int c = e >> 6, rr = e & 63, gr = 64 * t + rr;
        S.tiles[i * kTileElems + e] = (c < b && gr < N) ? to_v<float2>(__ldcg(J.R + (size_t)gr + (size_t)c * ld))
                                                        : make_float2(0.f, 0.f);
      }
    }
  cluster_sync();  // barriers initialised in every CTA before any remote arrival or store

  FwdItems it{n, N, cs, csm, q, nsteps, T};
  it.begin();
  if (tid >= kThreads) {
    if (tid == kThreads) produce_units(it, S, &fmap, J.slot, conv);
    __syncwarp();
  } else {
    int u = 0;  // units consumed
    bool ok = true;
    for (int j = -1; j < nsteps && ok; ++j) {
      if (j >= 0) ok = cta_wait(S.full + (j & nsm), (j >> lns) & 1, conv);  // Y_j is in slot j % ns
      while (ok && !it.fin && it.j == j) {
        const int t = it.t;
        const bool dk = it.d;
        Frag acc;
        zero(acc);
        bool okt = true;
        do {
          const float2 *A = unit_begin(S, u, okt, conv);
          if (okt) {
            const int k0 = 8 * g, k1 = min(k0 + 8, it.ncol());
            if (dk)
              product_cols(acc, A, S.tiles + (t >> lcs) * kTileElems, it.h * kUnit, k0, k1, rq, cq);
            else
              product_rows(acc, A, S.slots + (j & nsm) * kTileElems, it.h * kUnit, k0, k1, rq, cq);
          }
          unit_end(S, u);
          ++u;
          it.next();
        } while (!it.fin && it.j == j && it.t == t && it.d == dk && it.h != 0);
        store_partials(S.part, acc, g, rq, cq);
        ok = compute_and(okt);  // also: every partial sum is stored
        if (!ok) break;
        if (!dk) {
          // R[tile t] -= A21_j Y_j for the rows below the block
          const int k = 64 * j, kb = min(64, n - k), gr = 64 * t + r;
          if (gr >= k + kb && gr < N) {
            float2 *Rt = S.tiles + (t >> lcs) * kTileElems;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
              const int c = 4 * g + m;
              Rt[c * 64 + r] = csub(Rt[c * 64 + r], sum_partials(S.part, c, r));
            }
          }
        } else {
          // Y_(j+1) = D_(j+1) R_(j+1): into J.Y and into slot (j + 1) % ns of every CTA
          const int jd = j + 1, kd = 64 * jd, kbd = min(64, n - kd), slot = jd & nsm;
          if (jd >= ns) ok = cta_wait(S.empty + slot, ((jd >> lns) - 1) & 1, conv);
          if (!ok) break;
          const int row = tid >> 2, c0 = 4 * (tid & 3);
          float2 y[4];
#pragma unroll
          for (int m = 0; m < 4; ++m) y[m] = row < kbd ? sum_partials(S.part, c0 + m, row) : make_float2(0.f, 0.f);
          if (row < kbd) {
#pragma unroll
            for (int m = 0; m < 4; ++m)
              if (c0 + m < b) J.Y[(size_t)(kd + row) + (size_t)(c0 + m) * ld] = to_d(y[m]);
          }
          push_block(S, slot, cs, row, c0, y);
        }
        compute_sync();  // the partial sums are read before the next tile stores its own
      }
      if (ok && j >= 0) {
        compute_sync();  // every warp is done with slot j % ns
        if (tid == 0) mbar_arrive_cluster(S.empty + (j & nsm), fwd_producer(j + ns, csm));
      }
    }
    if (ok) {
      // the central rows of R for the Schur solve
      for (int i = 0; q + i * cs < T; ++i) {
        const int t = q + i * cs;
        if (64 * t + 63 < n) continue;
        for (int e = tid; e < kTileElems; e += kThreads) {
          const int c = e >> 6, gr = 64 * t + (e & 63);
          if (c < b && gr >= n && gr < N) J.R[(size_t)gr + (size_t)c * ld] = to_d(S.tiles[i * kTileElems + e]);
        }
      }
    } else if (tid == 0) {
      job_abort(conv);
    }
  }
  cluster_sync();  // no CTA leaves while another may still store into its shared memory
}

// Grid (cs, njobs), cluster (cs, 1, 1), 288 threads.  mode 0 sets X = Y, mode 1 adds X += Y
// (and skips converged jobs).
__global__ void __launch_bounds__(kBlock, 1)
    backward_flow_kernel(const JobDev *__restrict__ jobs, int own_max, int mode,
                         const __grid_constant__ CUtensorMap fmap) {
  const JobDev &J = jobs[blockIdx.y];
  if ((mode == 1 && converged(J.conv)) || J.inactive) return;
  const int q = cluster_rank(), cs = cluster_size(), csm = cs - 1, lcs = __ffs(cs) - 1;
  const FlowLayout L = flow_layout(cs, own_max);
  extern __shared__ __align__(128) unsigned char sm[];
  const FlowSmem S(sm, L);
  const int n = J.n, ld = J.ld, b = J.b, ns = L.ns, nsm = ns - 1, lns = __ffs(ns) - 1;
  int *conv = J.conv;
  const int tid = threadIdx.x, r = tid & 63, g = (tid >> 6) & 3, rq = tid & 15, cq = (tid >> 4) & 3;
  const int kstart = n > 0 ? ((n - 1) / 64) * 64 : 0;  // last block
  const int nsteps = n > 0 ? kstart / 64 + 2 : 1;       // central block + blocks kstart .. 0
  const int p0 = kstart / 64 + 1;
  const int Tn = (n + 63) / 64;                         // tiles with rows above the central block

  init_barriers(S, ns, cs);
  if (tid < kThreads) {
    // own tiles of Y (rows < n) in FP32
    for (int i = 0; q + i * cs < Tn; ++i) {
      const int t = q + i * cs;
      for (int e = tid; e < kTileElems; e += kThreads) {
        const int c = e >> 6, gr = 64 * t + (e & 63);
        S.tiles[i * kTileElems + e] = (c < b && gr < n) ? to_v<float2>(__ldcg(J.Y + (size_t)gr + (size_t)c * ld))
                                                        : make_float2(0.f, 0.f);
      }
    }
    // step 0, the central block from the Schur solve: every CTA fills its own slot 0
    for (int e = tid; e < kTileElems; e += kThreads) {
      const int row = e / kCols, c = e % kCols;
      S.slots[e] = (row < b && c < b) ? to_v<float2>(__ldcg(J.Y + (size_t)(n + row) + (size_t)c * ld))
                                      : make_float2(0.f, 0.f);
    }
    if (q == 0) {  // X_c (+)= Y_c
      for (int e = tid; e < b * b; e += kThreads) {
        const size_t idx = (size_t)(n + e % b) + (size_t)(e / b) * ld;
        const double2 y = __ldcg(J.Y + idx);
        if (mode == 0) {
          J.X[idx] = y;
        } else {
          const double2 x = J.X[idx];
          J.X[idx] = make_double2(x.x + y.x, x.y + y.y);
        }
      }
    }
  }
  cluster_sync();  // barriers initialised in every CTA before any remote arrival or store
  if (tid == 0) mbar_arrive_local(S.full, kWarps);

  BwdItems it{n, b, cs, csm, q, kstart, nsteps};
  it.begin();
  if (tid >= kThreads) {
    if (tid == kThreads) produce_units(it, S, &fmap, J.slot, conv);
    __syncwarp();
  } else {
    int u = 0;
    bool ok = true;
    for (int s = 0; s < nsteps && ok; ++s) {
      ok = cta_wait(S.full + (s & nsm), (s >> lns) & 1, conv);  // block s is in slot s % ns
      const int ks = s == 0 ? n : kstart - 64 * (s - 1);
      const int tnext = s + 1 < nsteps ? (kstart - 64 * s) / 64 : -1;  // tile of block s + 1
      while (ok && !it.fin && it.s == s) {
        const int t = it.t;
        Frag acc;
        zero(acc);
        bool okt = true;
        do {
          const float2 *A = unit_begin(S, u, okt, conv);
          if (okt) {
            const int k0 = 8 * g, k1 = min(k0 + 8, it.ncol());
            product_rows(acc, A, S.slots + (s & nsm) * kTileElems, it.h * kUnit, k0, k1, rq, cq);
          }
          unit_end(S, u);
          ++u;
          it.next();
        } while (!it.fin && it.s == s && it.t == t && it.h != 0);
        store_partials(S.part, acc, g, rq, cq);
        ok = compute_and(okt);
        if (!ok) break;
        // Y[tile t] -= W[tile t, block s] Y_s for the rows above the block
        float2 *Yt = S.tiles + (t >> lcs) * kTileElems;
        if (64 * t + r < ks) {
#pragma unroll
          for (int m = 0; m < 4; ++m) {
            const int c = 4 * g + m;
            Yt[c * 64 + r] = csub(Yt[c * 64 + r], sum_partials(S.part, c, r));
          }
        }
        if (t == tnext) {
          // the rows of block s + 1 are final: X (+)= Y there, and the block to every CTA
          const int kn = 64 * tnext, kbn = min(64, n - kn), slot = (s + 1) & nsm;
          if (s + 1 >= ns)
            ok = cta_wait(S.empty + slot, (((s + 1) >> lns) - 1) & 1, conv);
          else
            compute_sync();
          if (!ok) break;
          const int row = tid >> 2, c0 = 4 * (tid & 3);
          float2 y[4];
#pragma unroll
          for (int m = 0; m < 4; ++m) y[m] = row < kbn ? Yt[(c0 + m) * 64 + row] : make_float2(0.f, 0.f);
          if (row < kbn) {
#pragma unroll
            for (int m = 0; m < 4; ++m) {
              if (c0 + m >= b) continue;
              const size_t idx = (size_t)(kn + row) + (size_t)(c0 + m) * ld;
              const double2 yd = to_d(y[m]);
              if (mode == 0) {
                J.X[idx] = yd;
              } else {
                const double2 x = J.X[idx];
                J.X[idx] = make_double2(x.x + yd.x, x.y + yd.y);
              }
            }
          }
          push_block(S, slot, cs, row, c0, y);
        }
        compute_sync();  // the partial sums are read before the next tile stores its own
      }
      if (ok) {
        compute_sync();  // every warp is done with slot s % ns
        if (tid == 0) mbar_arrive_cluster(S.empty + (s & nsm), bwd_producer(s + ns, p0, csm));
      }
    }
    if (!ok && tid == 0) job_abort(conv);
  }
  cluster_sync();
}

}  // namespace

namespace {

// Clusters of the kernel resident at once for cluster size cs and `smem` bytes per CTA (cached).
int active_clusters(const void *kern, int cs, int smem) {
  static int cache[2][4] = {};
  static int cache_smem[2][4] = {};
  const int ki = kern == reinterpret_cast<const void *>(forward_flow_kernel) ? 0 : 1;
  const int ci = cs == 1 ? 0 : cs == 2 ? 1 : cs == 4 ? 2 : 3;
  if (cache_smem[ki][ci] == smem) return cache[ki][ci];
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs, 1, 1);
  cfg.blockDim = dim3(kBlock, 1, 1);
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
  cache[ki][ci] = v;
  cache_smem[ki][ci] = smem;
  return v;
}

}  // namespace

// Cluster size: the largest of 8, 4, 2, 1 whose layout fits and whose clusters for all jobs are
// resident at once; else the smallest that fits (the jobs then run in waves).  Not launched
// (*launched false) when no cluster size up to 8 holds the tiles in shared memory.
cudaError_t launch_flow_sweep(const JobDev *jobs, int njobs, int b, int max_N, bool forward, int mode,
                              const CUtensorMap *fmap, cudaStream_t s, bool *launched) {
  *launched = false;
  if (njobs <= 0 || b > kCols || max_N <= 0 || fmap == nullptr) return cudaSuccess;
  const int T = (max_N + 63) / 64;
  const void *kern = forward ? reinterpret_cast<const void *>(forward_flow_kernel)
                             : reinterpret_cast<const void *>(backward_flow_kernel);
  int cs = 0, fallback = 0;
  for (int c = 8; c >= 1; c >>= 1) {
    const FlowLayout L = flow_layout(c, (T + c - 1) / c);
    if (L.total > kMaxSmem) break;
    fallback = c;
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L.total);
    if (e != cudaSuccess) return e;
    if (active_clusters(kern, c, L.total) >= njobs) {
      cs = c;
      break;
    }
  }
  if (cs == 0) cs = fallback;
  if (cs == 0) return cudaSuccess;
  const FlowLayout L = flow_layout(cs, (T + cs - 1) / cs);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L.total);
  if (e != cudaSuccess) return e;
  if (forward)
    e = launch_cluster(forward_flow_kernel, cs, njobs, kBlock, L.total, s, jobs, L.own, *fmap);
  else
    e = launch_cluster(backward_flow_kernel, cs, njobs, kBlock, L.total, s, jobs, L.own, mode, *fmap);
  if (e == cudaSuccess) *launched = true;
  return e;
}

}  // namespace b200
