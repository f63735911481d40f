// Dataflow block sweeps of the correction solve: FP32 factors, b <= 16, the products on the
// tensor cores.
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
//    as soon as its slot is full, turns the block into the step's tensor-core operand and
//    releases the slot on its `empty` barrier in the CTA that produces the slot's next use.
//    Blocks are produced in turn by the cluster's ranks, so a rank produces every cs-th block and
//    its `empty` barrier of a slot completes one phase per block it produces into that slot: with
//    ns >= cs (cs divides ns) every use of the slot, with ns = 4 < cs = 8 (the ring shrunk so
//    that larger matrices fit shared memory) every other use.
//  * Operand panels (A21, D or W) stream through a ring of shared-memory stages several units
//    ahead: a unit is 64 complex rows x 32 columns of the factor, loaded by a producer warp as
//    four TMA boxes of 32 real rows x 32 columns in the 128-byte/32-byte-atom swizzle, which is
//    the tensor core's MN-major TF32 layout.  The D_(j+1) multiply of the forward sweep is just
//    two more units in the producing CTA's stream.
//  * A unit's product is one real GEMM of M = 128 (rows 2r, 2r + 1 = Re, Im of complex row r),
//    N = 32 (the block's real parts, then its imaginary parts) and K = 32 on tcgen05 kind::tf32
//    with the accumulator in tensor memory.  FP32 accuracy comes from the TF32 hi/lo split of
//    both operands and three products, A_hi [B_hi | B_lo] (N = 64) and A_lo B_hi (N = 32) into
//    the same columns.  The compute warps split each landed unit in place (hi) and into a lo
//    buffer and each arrives on the unit's `split` barrier; an MMA warp issues the products and
//    commits them to the barriers that free the ring stage, the lo buffer and (after a tile's
//    last unit) mark the accumulator full, so splitting, issuing and the tensor core overlap
//    across units.  The epilogue of a tile reads the accumulator once:
//    lane m of TMEM is real row m, and a shuffle between lanes 2r and 2r + 1 forms
//    Re = Ar Yr - Ai Yi and Im = Ar Yi + Ai Yr.
//
// Every barrier wait is bounded.  A wait that runs out marks the job aborted (JobDev::conv =
// kAborted), which also ends the other CTAs' waits; the job's tau00_l step reports it in the
// context's error word, and the refinement re-solves that job in FP64.

#include <cuda_runtime.h>

#include "cluster.cuh"
#include "common.cuh"
#include "cplx.cuh"
#include "umma.cuh"

namespace b200 {
namespace {

using namespace cx;
using namespace cl;

constexpr int kThreads = 256;             // compute threads (8 warps)
constexpr int kBlock = kThreads + 64;     // and the producer and MMA warps
constexpr int kWarps = kThreads / 32;
constexpr int kCols = 16;                  // right-hand-side columns held (b <= 16)
constexpr int kUnit = 32;                  // factor columns per unit: the MMA's K
constexpr int kUnitFloats = 128 * kUnit;   // 128 real rows (the MMA's M) x 32 columns
constexpr unsigned kUnitBytes = kUnitFloats * 4;
constexpr int kBoxFloats = 32 * kUnit;     // one TMA box: 32 real rows x 32 columns
constexpr int kStages = 3;                 // operand ring depth (units)
constexpr int kTileElems = 64 * kCols;     // one 64-row tile of the right-hand side (float2)
constexpr int kPerThread = kTileElems / kThreads;  // a tile's entries per compute thread
static_assert(kTileElems % kThreads == 0, "tile entries spread evenly over the compute threads");
constexpr int kBFloats = 64 * 64;          // B operand of a 64-row block: N = 64 rows x K = 64
constexpr int kAccCols = 64;               // TMEM columns per accumulator (two of them)
constexpr int kMaxSmem = 227 * 1024;
constexpr long kFlowWaitBound = 1L << 22;  // barrier polls before a wait gives up

// A: MN-major, 32-row boxes 4 KB apart (LBO), 4-column groups 512 B apart (SBO).
// B: K-major, 128-byte rows, 8-row groups 1 KB apart.
constexpr uint32_t kIdescHi = um::idesc_tf32(128, 64, true, false);
constexpr uint32_t kIdescLo = um::idesc_tf32(128, 32, true, false);

// Shared-memory layout (byte offsets from a 1024-byte-aligned base) for cluster size cs and `own`
// resident tiles per CTA.  bd (the D_(j+1) multiply's operand) exists in the forward sweep only.
struct FlowLayout {
  int ns, own;
  int ring, lo, bstep, bd, slots, tiles, bars, tmem, total;
};
__host__ __device__ constexpr int kBars(int ns) { return 2 * ns + 2 * kStages + 9; }
__host__ __device__ inline FlowLayout flow_layout(int cs, int own, bool forward, int ns);
// ns = max(cs, 4) block slots, or 4 for cs = 8 when that does not fit shared memory (N = 4320)
__host__ __device__ inline FlowLayout flow_layout(int cs, int own, bool forward) {
  const FlowLayout L = flow_layout(cs, own, forward, cs > 4 ? cs : 4);
  return (L.total > kMaxSmem && cs > 4) ? flow_layout(cs, own, forward, 4) : L;
}
__host__ __device__ inline FlowLayout flow_layout(int cs, int own, bool forward, int ns) {
  FlowLayout L;
  L.ns = ns;
  L.own = own;
  L.ring = 0;
  L.lo = L.ring + kStages * kUnitBytes;
  L.bstep = L.lo + 2 * kUnitBytes;
  L.bd = L.bstep + kBFloats * 4;
  L.slots = L.bd + (forward ? kBFloats * 4 : 0);
  L.tiles = L.slots + L.ns * kTileElems * 8;
  L.bars = L.tiles + own * kTileElems * 8;
  L.tmem = L.bars + kBars(L.ns) * 8;
  L.total = L.tmem + 16 + 1024;  // + the alignment of the dynamic shared-memory base
  return L;
}

// The job's abort word: JobDev::conv (null for an initial solve without refinement state).
__device__ __forceinline__ bool job_aborted(const int *conv) {
  return conv != nullptr && *reinterpret_cast<volatile const int *>(conv) == kAborted;
}
__device__ __forceinline__ void job_abort(int *conv) {
  if (conv != nullptr) atomicExch(conv, kAborted);
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
// when the bound ran out or the job was aborted.  Cluster-scope acquire for the ring slots'
// barriers, which other CTAs arrive on; CTA scope for the rest.
template <bool kCluster>
__device__ __forceinline__ bool wait_phase(unsigned long long *bar, unsigned parity, const int *conv) {
  for (long i = 0; i < kFlowWaitBound; ++i) {
    if (kCluster ? mbar_try_cluster(bar, parity) : mbar_try_cta(bar, parity)) return true;
    if ((i & 1023) == 1023 && job_aborted(conv)) return false;
  }
  return false;
}
__device__ __forceinline__ bool wait_local(unsigned long long *bar, unsigned parity, const int *conv) {
  return wait_phase<false>(bar, parity, conv);
}
// The same for every compute thread, with a uniform outcome.
template <bool kCluster>
__device__ __forceinline__ bool cta_wait(unsigned long long *bar, unsigned parity, const int *conv) {
  return compute_and(wait_phase<kCluster>(bar, parity, conv));
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
  __device__ bool dmul() const { return d; }  // a D unit (its B is the tile, not the slot)
  // Whether the item after this one continues the same tile (call after next()).
  __device__ bool same_tile(int j0, int t0, bool d0) const { return !fin && j == j0 && t == t0 && d == d0 && h != 0; }
  __device__ bool same_tile() const { return same_tile(pj, pt, pd); }
  int pj, pt;
  bool pd;
  __device__ void mark() {
    pj = j;
    pt = t;
    pd = d;
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
  __device__ bool same_tile(int s0, int t0) const { return !fin && s == s0 && t == t0 && h != 0; }
  __device__ bool dmul() const { return false; }
  __device__ bool same_tile() const { return same_tile(ps, pt); }
  int ps, pt;
  __device__ void mark() {
    ps = s;
    pt = t;
  }
};

// Shared-memory views of one CTA.
struct FlowSmem {
  float *ring, *lo, *bstep, *bd;
  float2 *slots, *tiles;
  unsigned long long *full, *empty, *ring_full, *ring_empty, *lo_free, *acc_full, *split, *acc_empty, *drain;
  unsigned *tmem;
  __device__ FlowSmem(unsigned char *sm, const FlowLayout &L)
      : ring(reinterpret_cast<float *>(sm + L.ring)),
        lo(reinterpret_cast<float *>(sm + L.lo)),
        bstep(reinterpret_cast<float *>(sm + L.bstep)),
        bd(reinterpret_cast<float *>(sm + L.bd)),
        slots(reinterpret_cast<float2 *>(sm + L.slots)),
        tiles(reinterpret_cast<float2 *>(sm + L.tiles)),
        full(reinterpret_cast<unsigned long long *>(sm + L.bars)),
        empty(full + L.ns),
        ring_full(full + 2 * L.ns),
        ring_empty(ring_full + kStages),
        lo_free(ring_empty + kStages),
        acc_full(lo_free + 2),
        split(acc_full + 2),
        acc_empty(split + 2),
        drain(acc_empty + 2),
        tmem(reinterpret_cast<unsigned *>(sm + L.tmem)) {}
};

// The dynamic shared memory rounded up to 1024 bytes (the swizzle patterns' period).  Every CTA
// of the kernel gets the same offset, so distributed shared-memory addresses line up.
__device__ __forceinline__ unsigned char *aligned_smem(unsigned char *sm) {
  return sm + ((1024u - (smem_u32(sm) & 1023u)) & 1023u);
}

// Barriers: full[s] completes a phase when the 8 compute warps of the slot's producer have stored
// the block (or, for a slot filled by the CTA itself, when it arrives 8 times); empty[s] when all
// cs CTAs are done with the slot's current use; ring_full[s] when the TMA loads of the unit in ring
// stage s have landed; ring_empty[s] when the MMAs reading it have completed (a tcgen05 commit);
// lo_free[i] the same for lo buffer i; split[i] when the 8 compute warps have split the unit in lo
// buffer i (and built its B); acc_full[i] when the last MMA into accumulator i has completed;
// acc_empty[i] when the 8 compute warps have read accumulator i out; drain at the end, once every
// MMA of the CTA has.
__device__ __forceinline__ void init_barriers(const FlowSmem &S, int ns, int cs) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < ns; ++s) {
      mbar_init(S.full + s, kWarps);
      mbar_init(S.empty + s, cs);
    }
    for (int s = 0; s < kStages; ++s) {
      mbar_init(S.ring_full + s, 1);
      mbar_init(S.ring_empty + s, 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(S.lo_free + i, 1);
      mbar_init(S.acc_full + i, 1);
      mbar_init(S.split + i, kWarps);
      mbar_init(S.acc_empty + i, kWarps);
    }
    mbar_init(S.drain, 1);
    fence_mbar_init();
  }
}

// Start of a kernel: barriers, and warp 0 allocates the two accumulators in tensor memory.  The
// caller's cluster_sync() publishes both.
__device__ __forceinline__ void flow_setup(const FlowSmem &S, int ns, int cs) {
  init_barriers(S, ns, cs);
  if (threadIdx.x < 32) um::alloc(S.tmem, 2 * kAccCols);
  um::fence_before();
}
// End of a kernel: the MMA warp waits until every MMA it issued has completed, then (after the
// cluster barrier: no CTA leaves while another may still store into its shared memory) warp 0
// frees the tensor memory.
__device__ __forceinline__ void flow_teardown(const FlowSmem &S, uint32_t tmem) {
  if (threadIdx.x == kThreads + 32) {
    um::commit(S.drain);
    wait_local(S.drain, 0, nullptr);
  }
  um::fence_before();
  cluster_sync();
  if (threadIdx.x < 32) {
    um::fence_after();
    um::dealloc(tmem, 2 * kAccCols);
  }
}

// The producer warp's lane 0: streams the CTA's units, in consumption order, into ring stage
// v % kStages by four TMA loads each (32 real rows x 32 columns per box), reusing a stage once the
// MMAs of its previous unit have completed; then waits for its last loads, so that none lands
// after the CTA has left.
template <class Items>
__device__ void produce_units(Items pf, const FlowSmem &S, const CUtensorMap *map, int slot, int *conv) {
  int issued = 0;
  bool ok = true;
  for (; !pf.fin; pf.next(), ++issued) {
    const int st = issued % kStages, round = issued / kStages;
    if (round > 0 && !wait_local(S.ring_empty + st, (round - 1) & 1, conv)) {
      ok = false;
      break;
    }
    mbar_expect_tx(S.ring_full + st, kUnitBytes);
    float *dst = S.ring + st * kUnitFloats;
    const int x = 2 * pf.row0(), y = pf.col0();
#pragma unroll
    for (int q = 0; q < 4; ++q) tma_load_3d(dst + q * kBoxFloats, map, x + 32 * q, y, slot, S.ring_full + st);
  }
  if (!ok) job_abort(conv);
  for (int v = max(0, issued - kStages); v < issued; ++v)
    wait_local(S.ring_full + v % kStages, (v / kStages) & 1, nullptr);
}

// B operand of a 64-row block of the right-hand side (column-major src[c * 64 + kk]; rows kk >=
// valid read as zero): K-major with 128-byte swizzle, N rows n = 16 part + c for part 0 / 1 the
// TF32 hi of the real / imaginary parts and part 2 / 3 their lo; K = the block's 64 rows in two
// halves of 32 (8 KB apart), one per unit.  Lane = K row, so every store of a warp hits one
// 128-byte row.
__device__ __forceinline__ void build_b(float *B, const float2 *src, int valid) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int pr = 4 * warp + i, c = pr & 15, h = pr >> 4, kk = 32 * h + lane;
    const float2 y = kk < valid ? src[c * 64 + kk] : make_float2(0.f, 0.f);
    const float hr = um::tf32_round(y.x), hi = um::tf32_round(y.y);
    float *Bh = B + h * 2048 + (lane & 3);
    const int chunk = lane >> 2;
    // row n: (n >> 3) * 256 + (n & 7) * 32 floats, 16-byte chunk (K / 4) ^ (n & 7)
    const auto at = [&](int n) { return (n >> 3) * 256 + (n & 7) * 32 + (((chunk ^ (n & 7)) & 7) << 2); };
    Bh[at(c)] = hr;
    Bh[at(16 + c)] = hi;
    Bh[at(32 + c)] = y.x - hr;
    Bh[at(48 + c)] = y.y - hi;
  }
}

// TF32 hi/lo split of the unit in a ring stage: hi in place, lo into `lo`; factor columns >= ncol
// (past the block, or padding of the slot) become zero.  Thread: K row tid / 8 of each box, one
// 16-byte chunk per box (the swizzle permutes chunks within a row only).
__device__ __forceinline__ void split_unit(float *a, float *lo, int ncol) {
  const int tid = threadIdx.x;
  const bool live = (tid >> 3) < ncol;
  float4 *A4 = reinterpret_cast<float4 *>(a);
  float4 *L4 = reinterpret_cast<float4 *>(lo);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int f = tid + 256 * q;
    float4 h = make_float4(0.f, 0.f, 0.f, 0.f), l = h;
    if (live) {
      const float4 x = A4[f];
      h = make_float4(um::tf32_round_int(x.x), um::tf32_round_int(x.y), um::tf32_round_int(x.z),
                      um::tf32_round_int(x.w));
      l = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
    }
    A4[f] = h;
    L4[f] = l;
  }
}

// One unit on the compute side: wait for its load and for its lo buffer, split it, and arrive
// (per warp) on the unit's split barrier.  A warp in which a wait ran out marks the job aborted
// and skips the rest (all its lanes alike, so the warp-wide sync below is reached by all or none),
// so the accumulator never fills and the tile's vote fails everywhere.
__device__ __forceinline__ void unit_split(const FlowSmem &S, int u, int ncol, int *conv) {
  const int st = u % kStages;
  bool okt = wait_local(S.ring_full + st, (u / kStages) & 1, conv);
  if (okt && u >= 2) okt = wait_local(S.lo_free + (u & 1), ((u >> 1) - 1) & 1, conv);
  okt = __all_sync(0xffffffffu, okt);
  if (!okt) {
    job_abort(conv);
    return;
  }
  split_unit(S.ring + st * kUnitFloats, S.lo + (u & 1) * kUnitFloats, ncol);
  fence_proxy_async();  // the split (and any B build before it) is visible to the tensor core
  __syncwarp();
  if ((threadIdx.x & 31) == 0) mbar_arrive_local(S.split + (u & 1), 1);
}

// The MMA warp's lane 0: for each unit, in the compute warps' order, waits for its split, then
// issues A_hi [B_hi | B_lo] into accumulator columns 0-63 and A_lo B_hi into columns 0-31 per
// 8-column K step, against the 32-row half of the tile's B (the step's block, or for D units the
// tile).  Commits free the ring stage and the lo buffer, and after a tile's last unit mark the
// accumulator full; a tile's first MMA waits until the compute warps have read out the
// accumulator's previous tile.
template <class Items>
__device__ void issue_units(Items it, const FlowSmem &S, uint32_t tmem, int *conv) {
  const uint32_t bstep = smem_u32(S.bstep), bd = smem_u32(S.bd);
  int u = 0, nt = 0;
  bool ok = true;
  while (ok && !it.fin) {
    it.mark();
    const uint32_t b = it.dmul() ? bd : bstep, acc = tmem + (uint32_t)((nt & 1) * kAccCols);
    if (nt >= 2) ok = wait_local(S.acc_empty + (nt & 1), ((nt >> 1) - 1) & 1, conv);
    bool first = true, last = false;
    while (ok && !last) {
      const int h = it.h, st = u % kStages;
      it.next();
      last = !it.same_tile();
      ok = wait_local(S.split + (u & 1), (u >> 1) & 1, conv);
      if (!ok) break;
      um::fence_after();
      const uint32_t sa = smem_u32(S.ring + st * kUnitFloats), sl = smem_u32(S.lo + (u & 1) * kUnitFloats);
      const uint32_t sb = b + (uint32_t)h * 8192u;
#pragma unroll
      for (int ks = 0; ks < kUnit / 8; ++ks) {
        const uint64_t dh = um::sdesc(sa + ks * 1024, 4096, 512, um::kSw128Base32b);
        const uint64_t dl = um::sdesc(sl + ks * 1024, 4096, 512, um::kSw128Base32b);
        const uint64_t db = um::sdesc(sb + ks * 32, 16, 1024, um::kSw128);
        um::mma_tf32(acc, dh, db, kIdescHi, (first && ks == 0) ? 0u : 1u);
        um::mma_tf32(acc, dl, db, kIdescLo, 1u);
      }
      um::commit(S.ring_empty + st);
      um::commit(S.lo_free + (u & 1));
      if (last) um::commit(S.acc_full + (nt & 1));
      first = false;
      ++u;
    }
    ++nt;
  }
  if (!ok) job_abort(conv);
}

// Epilogue read of accumulator `ab`: thread (warp w, lane) holds complex row r = m / 2 of the 64 x 16
// product, m = 32 (w % 4) + lane, part p = m % 2 (0 real, 1 imaginary), columns c0 .. c0 + 7 with
// c0 = 8 (w / 4).  Columns 0-15 of the accumulator hold the products with the block's real parts,
// 16-31 with its imaginary parts, 32-63 the same for the lo halves.  Each warp then arrives on
// the accumulator's `empty` barrier.
__device__ __forceinline__ void acc_read(const FlowSmem &S, uint32_t tmem, int ab, float (&v)[8]) {
  const int w = threadIdx.x >> 5;
  const uint32_t base = tmem + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)(ab * kAccCols + 8 * (w >> 2));
  uint32_t d0[8], d1[8], d2[8], d3[8];
  um::ld_32x32b_x8(base, d0);
  um::ld_32x32b_x8(base + 16, d1);
  um::ld_32x32b_x8(base + 32, d2);
  um::ld_32x32b_x8(base + 48, d3);
  um::wait_ld();
  um::fence_before();
  __syncwarp();
  if ((threadIdx.x & 31) == 0) mbar_arrive_local(S.acc_empty + ab, 1);
  const bool im = threadIdx.x & 1;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float s1 = __uint_as_float(d0[i]) + __uint_as_float(d2[i]);  // A_p Yr
    const float s2 = __uint_as_float(d1[i]) + __uint_as_float(d3[i]);  // A_p Yi
    const float o = __shfl_xor_sync(0xffffffffu, s2, 1);               // A_(1-p) Yi
    v[i] = im ? s1 + o : s1 - o;
  }
}

// R (or Y) tile update from accumulator `nt`: rows row0 + m / 2 in [lo, hi) of the resident
// tile `tile` (FP32, column-major) minus the product.  False, for every compute thread, when the
// wait for the accumulator ran out.
__device__ __forceinline__ bool tile_update(const FlowSmem &S, uint32_t tmem, int nt, float *tile, int row0, int lo,
                                            int hi, const int *conv) {
  if (!cta_wait<false>(S.acc_full + (nt & 1), (nt >> 1) & 1, conv)) return false;
  um::fence_after();
  float v[8];
  acc_read(S, tmem, nt & 1, v);
  const int w = threadIdx.x >> 5, m = 32 * (w & 3) + (threadIdx.x & 31), c0 = 8 * ((w >> 2) & 1);
  const int gr = row0 + (m >> 1);
  if (gr >= lo && gr < hi) {
#pragma unroll
    for (int i = 0; i < 8; ++i) tile[(c0 + i) * 128 + m] -= v[i];
  }
  return true;
}
// A tile update left for later: it runs after the next tile's units are split, so the tile's MMAs
// overlap that split instead of stalling the compute warps.  Tiles on the block chain (the next
// block's tile, the D multiply) are never deferred.
struct Deferred {
  int nt, row0, lo, hi;
  float *tile;
  __device__ bool flush(const FlowSmem &S, uint32_t tmem, const int *conv) {
    if (nt < 0) return true;
    const bool ok = tile_update(S, tmem, nt, tile, row0, lo, hi, conv);
    nt = -1;
    return ok;
  }
};

// Grid (cs, njobs), cluster (cs, 1, 1), 320 threads: 8 compute warps, the producer warp and the
// MMA warp.
// Refinement rounds only (the initial solve has B = 0 above the central block).  own_max:
// resident tiles per CTA (ceil(tiles / cs)).
__global__ void __launch_bounds__(kBlock, 1)
    forward_flow_kernel(const JobDev *__restrict__ jobs, int own_max, const __grid_constant__ CUtensorMap fmap,
                        int col0) {
  const JobDev &J = jobs[blockIdx.y];
  // uniform over the cluster: the flag changes only between launches
  if (converged(J.conv) || J.n == 0 || J.inactive) return;
  const int q = cluster_rank(), cs = cluster_size(), csm = cs - 1, lcs = __ffs(cs) - 1;
  const FlowLayout L = flow_layout(cs, own_max, true);
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  const FlowSmem S(aligned_smem(sm_raw), L);
  // this launch's right-hand-side columns: [col0, col0 + b) of R and Y
  const int n = J.n, N = J.N, ld = J.ld, b = min(kCols, J.b - col0), ns = L.ns, nsm = ns - 1, lns = __ffs(ns) - 1;
  double2 *const Rb = J.R + (size_t)col0 * ld;
  double2 *const Yb = J.Y + (size_t)col0 * ld;
  int *conv = J.conv;
  const int tid = threadIdx.x, warp = tid >> 5, m = 32 * (warp & 3) + (tid & 31), r = m >> 1, p = m & 1;
  const int c0 = 8 * ((warp >> 2) & 1);
  const int nsteps = (n + 63) / 64, T = (N + 63) / 64;

  flow_setup(S, ns, cs);
  // own tiles of R in FP32, zero past row N and column b
  if (tid < kThreads)
    for (int i = 0; q + i * cs < T; ++i) {
      const int t = q + i * cs;
      float2 v[kPerThread];  // a tile's loads in flight together, then its stores
#pragma unroll
      for (int j = 0; j < kPerThread; ++j) {
        const int e = tid + j * kThreads, c = e >> 6, rr = e & 63, gr = 64 * t + rr;
        v[j] = (c < b && gr < N) ? to_v<float2>(__ldcg(Rb + (size_t)gr + (size_t)c * ld)) : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int j = 0; j < kPerThread; ++j) S.tiles[i * kTileElems + tid + j * kThreads] = v[j];
    }
  cluster_sync();  // barriers and tensor memory set up in every CTA before any remote arrival or store
  um::fence_after();
  const uint32_t tmem = *S.tmem;

  FwdItems it{n, N, cs, csm, q, nsteps, T};
  it.begin();
  if (tid >= kThreads) {
    if (tid == kThreads)
      produce_units(it, S, &fmap, J.slot, conv);
    else if (tid == kThreads + 32)
      issue_units(it, S, tmem, conv);
    __syncwarp();
  } else {
    int u = 0, nt = 0;  // units consumed, tiles started
    bool ok = true;
    Deferred dq{-1};
    for (int j = -1; j < nsteps && ok; ++j) {
      if (j >= 0) {
        ok = dq.flush(S, tmem, conv);  // its MMAs read the operand that this step overwrites
        if (!ok) break;
        ok = cta_wait<true>(S.full + (j & nsm), (j >> lns) & 1, conv);  // Y_j is in slot j % ns
        if (!ok) break;
        if (!it.fin && it.j == j) build_b(S.bstep, S.slots + (j & nsm) * kTileElems, min(64, n - 64 * j));
        fence_proxy_async();
        compute_sync();  // every warp is done with slot j % ns
        if (tid == 0) mbar_arrive_cluster(S.empty + (j & nsm), fwd_producer(j + ns, csm));
      }
      while (ok && !it.fin && it.j == j) {
        const int t = it.t;
        const bool dk = it.d;
        float2 *Rt = S.tiles + (t >> lcs) * kTileElems;
        if (dk) {
          compute_sync();  // tile j + 1 is updated (its update is never deferred)
          build_b(S.bd, Rt, min(64, n - 64 * t));
        }
        bool last;
        do {
          const int ncol = it.ncol();
          it.next();
          last = !it.same_tile(j, t, dk);
          unit_split(S, u++, ncol, conv);
        } while (!last);
        const int me = nt++;
        if (!dk) {
          // R[tile t] -= A21_j Y_j for the rows below the block
          const int lo = 64 * j + min(64, n - 64 * j);
          float *Rf = reinterpret_cast<float *>(Rt);
          if (t != j + 1) {
            ok = dq.flush(S, tmem, conv);
            dq = Deferred{me, 64 * t, lo, N, Rf};
          } else {
            ok = tile_update(S, tmem, me, Rf, 64 * t, lo, N, conv);
          }
        } else {
          ok = cta_wait<false>(S.acc_full + (me & 1), (me >> 1) & 1, conv);
          if (!ok) break;
          um::fence_after();
          float v[8];
          acc_read(S, tmem, me & 1, v);
          // Y_(j+1) = D_(j+1) R_(j+1): into J.Y and into slot (j + 1) % ns of every CTA
          const int jd = j + 1, kd = 64 * jd, kbd = min(64, n - kd), slot = jd & nsm;
          // this rank's phases of the slot's empty barrier: one per block it produced into the slot
          if (jd >= ns) ok = cta_wait<true>(S.empty + slot, ((jd - ns) >> max(lns, lcs)) & 1, conv);
          if (!ok) break;
          const float *dst = reinterpret_cast<const float *>(S.slots + slot * kTileElems);
          const bool live = r < kbd;
          double *Yd = reinterpret_cast<double *>(Yb);
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int c = c0 + i;
            if (!live) v[i] = 0.f;
            if (live && c < b) Yd[2 * ((size_t)(kd + r) + (size_t)c * ld) + p] = (double)v[i];
          }
          for (int pc = 0; pc < cs; ++pc) {
            const unsigned rb = remote_u32(dst, pc) + 4u * (unsigned)m;
#pragma unroll
            for (int i = 0; i < 8; ++i) st_remote_f32(rb + 512u * (unsigned)(c0 + i), v[i]);
          }
          __syncwarp();
          if ((tid & 31) == 0)
            for (int pc = 0; pc < cs; ++pc) mbar_arrive_cluster(S.full + slot, pc);
        }
      }
    }
    if (ok) ok = dq.flush(S, tmem, conv);
    if (ok) {
      compute_sync();  // every tile update is done
      // the central rows of R for the Schur solve
      for (int i = 0; q + i * cs < T; ++i) {
        const int t = q + i * cs;
        if (64 * t + 63 < n) continue;
        for (int e = tid; e < kTileElems; e += kThreads) {
          const int c = e >> 6, gr = 64 * t + (e & 63);
          if (c < b && gr >= n && gr < N) Rb[(size_t)gr + (size_t)c * ld] = to_d(S.tiles[i * kTileElems + e]);
        }
      }
    } else if (tid == 0) {
      job_abort(conv);
    }
  }
  flow_teardown(S, tmem);
}

// Grid (cs, njobs), cluster (cs, 1, 1), 320 threads.  mode 0 sets X = Y, mode 1 adds X += Y
// (and skips converged jobs).
__global__ void __launch_bounds__(kBlock, 1)
    backward_flow_kernel(const JobDev *__restrict__ jobs, int own_max, int mode,
                         const __grid_constant__ CUtensorMap fmap, int col0) {
  const JobDev &J = jobs[blockIdx.y];
  if ((mode == 1 && converged(J.conv)) || J.inactive) return;
  const int q = cluster_rank(), cs = cluster_size(), csm = cs - 1, lcs = __ffs(cs) - 1;
  const FlowLayout L = flow_layout(cs, own_max, false);
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  const FlowSmem S(aligned_smem(sm_raw), L);
  // bc: rows of the central block; b: this launch's right-hand-side columns [col0, col0 + b) of Y, X
  const int n = J.n, ld = J.ld, bc = J.b, b = min(kCols, J.b - col0), ns = L.ns, nsm = ns - 1,
            lns = __ffs(ns) - 1;
  const double2 *const Yb = J.Y + (size_t)col0 * ld;
  double2 *const Xb = J.X + (size_t)col0 * ld;
  int *conv = J.conv;
  const int tid = threadIdx.x;
  const int kstart = n > 0 ? ((n - 1) / 64) * 64 : 0;  // last block
  const int nsteps = n > 0 ? kstart / 64 + 2 : 1;       // central block + blocks kstart .. 0
  const int p0 = kstart / 64 + 1;
  const int Tn = (n + 63) / 64;                         // tiles with rows above the central block

  flow_setup(S, ns, cs);
  if (tid < kThreads) {
    // own tiles of Y (rows < n) in FP32
    for (int i = 0; q + i * cs < Tn; ++i) {
      const int t = q + i * cs;
      float2 v[kPerThread];  // a tile's loads in flight together, then its stores
#pragma unroll
      for (int j = 0; j < kPerThread; ++j) {
        const int e = tid + j * kThreads, c = e >> 6, gr = 64 * t + (e & 63);
        v[j] = (c < b && gr < n) ? to_v<float2>(__ldcg(Yb + (size_t)gr + (size_t)c * ld)) : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int j = 0; j < kPerThread; ++j) S.tiles[i * kTileElems + tid + j * kThreads] = v[j];
    }
    // step 0, the central block from the Schur solve: every CTA fills its own slot 0 (column-major)
    for (int e = tid; e < kTileElems; e += kThreads) {
      const int c = e >> 6, row = e & 63;
      S.slots[e] = (row < bc && c < b) ? to_v<float2>(__ldcg(Yb + (size_t)(n + row) + (size_t)c * ld))
                                       : make_float2(0.f, 0.f);
    }
    if (q == 0) {  // X_c (+)= Y_c
      for (int e = tid; e < bc * b; e += kThreads) {
        const size_t idx = (size_t)(n + e % bc) + (size_t)(e / bc) * ld;
        const double2 y = __ldcg(Yb + idx);
        if (mode == 0) {
          Xb[idx] = y;
        } else {
          const double2 x = Xb[idx];
          Xb[idx] = make_double2(x.x + y.x, x.y + y.y);
        }
      }
    }
  }
  cluster_sync();  // barriers and tensor memory set up in every CTA before any remote arrival or store
  um::fence_after();
  const uint32_t tmem = *S.tmem;
  if (tid == 0) mbar_arrive_local(S.full, kWarps);

  BwdItems it{n, bc, cs, csm, q, kstart, nsteps};
  it.begin();
  if (tid >= kThreads) {
    if (tid == kThreads)
      produce_units(it, S, &fmap, J.slot, conv);
    else if (tid == kThreads + 32)
      issue_units(it, S, tmem, conv);
    __syncwarp();
  } else {
    int u = 0, nt = 0;
    bool ok = true;
    Deferred dq{-1};
    for (int s = 0; s < nsteps && ok; ++s) {
      ok = dq.flush(S, tmem, conv);  // its MMAs read the operand that this step overwrites
      if (!ok) break;
      ok = cta_wait<true>(S.full + (s & nsm), (s >> lns) & 1, conv);  // block s is in slot s % ns
      if (!ok) break;
      const int ks = s == 0 ? n : kstart - 64 * (s - 1);
      const int tnext = s + 1 < nsteps ? (kstart - 64 * s) / 64 : -1;  // tile of block s + 1
      if (!it.fin && it.s == s) build_b(S.bstep, S.slots + (s & nsm) * kTileElems, s == 0 ? bc : min(64, n - ks));
      fence_proxy_async();
      compute_sync();  // every warp is done with slot s % ns
      if (tid == 0) mbar_arrive_cluster(S.empty + (s & nsm), bwd_producer(s + ns, p0, csm));
      while (ok && !it.fin && it.s == s) {
        const int t = it.t;
        bool last;
        do {
          const int ncol = it.ncol();
          it.next();
          last = !it.same_tile(s, t);
          unit_split(S, u++, ncol, conv);
        } while (!last);
        const int me = nt++;
        // Y[tile t] -= W[tile t, block s] Y_s for the rows above the block
        float2 *Yt = S.tiles + (t >> lcs) * kTileElems;
        float *Yf = reinterpret_cast<float *>(Yt);
        if (t != tnext) {
          ok = dq.flush(S, tmem, conv);
          dq = Deferred{me, 64 * t, 0, ks, Yf};
        } else {
          ok = tile_update(S, tmem, me, Yf, 64 * t, 0, ks, conv);
          if (!ok) break;
          // the rows of block s + 1 are final: X (+)= Y there, and the block to every CTA
          const int kn = 64 * tnext, kbn = min(64, n - kn), slot = (s + 1) & nsm;
          if (s + 1 >= ns)
            ok = cta_wait<true>(S.empty + slot, (((s + 1) - ns) >> max(lns, lcs)) & 1, conv);
          else
            compute_sync();
          if (!ok) break;
          const float4 *src = reinterpret_cast<const float4 *>(Yt);
          const float4 *dst = reinterpret_cast<const float4 *>(S.slots + slot * kTileElems);
          float4 yv[2];
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            // float4 f: column c = f / 32, complex rows 2 (f % 32) and 2 (f % 32) + 1
            const int f = tid + kThreads * i, r0 = 2 * (f & 31);
            float4 y = src[f];
            if (r0 >= kbn) y.x = y.y = 0.f;
            if (r0 + 1 >= kbn) y.z = y.w = 0.f;
            yv[i] = y;
            for (int pc = 0; pc < cs; ++pc) st_remote(remote_u32(dst + f, pc), y);
          }
          __syncwarp();
          if ((tid & 31) == 0)
            for (int pc = 0; pc < cs; ++pc) mbar_arrive_cluster(S.full + slot, pc);
          // X (+)= Y on the block's rows once the block is out: the read of X (mode 1) then
          // stays off the chain of steps
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int f = tid + kThreads * i, c = f >> 5, r0 = 2 * (f & 31);
            if (c >= b) continue;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              if (r0 + e >= kbn) continue;
              const size_t idx = (size_t)(kn + r0 + e) + (size_t)c * ld;
              const double2 yd = make_double2(e ? yv[i].z : yv[i].x, e ? yv[i].w : yv[i].y);
              if (mode == 0) {
                Xb[idx] = yd;
              } else {
                const double2 x = Xb[idx];
                Xb[idx] = make_double2(x.x + yd.x, x.y + yd.y);
              }
            }
          }
        }
      }
    }
    if (ok) ok = dq.flush(S, tmem, conv);
    if (!ok && tid == 0) job_abort(conv);
  }
  flow_teardown(S, tmem);
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

// Cluster size: the largest of 8, 4, 2, 1 whose layout fits and whose clusters for all active jobs
// (active_hint of them when given, else njobs) are resident at once; else the smallest that fits
// (the jobs then run in waves).  Clusters of converged jobs leave at once, so the grid always
// covers all njobs.  Not launched (*launched false) when no cluster size up to 8 holds the tiles in
// shared memory.
cudaError_t launch_flow_sweep(const JobDev *jobs, int njobs, int b, int max_N, bool forward, int mode,
                              const CUtensorMap *fmap, cudaStream_t s, bool *launched, int active_hint) {
  *launched = false;
  if (njobs <= 0 || b > 2 * kCols || max_N <= 0 || fmap == nullptr) return cudaSuccess;
  const int T = (max_N + 63) / 64;
  const void *kern = forward ? reinterpret_cast<const void *>(forward_flow_kernel)
                             : reinterpret_cast<const void *>(backward_flow_kernel);
  const int want = active_hint > 0 && active_hint < njobs ? active_hint : njobs;
  int cs = 0, fallback = 0;
  for (int c = 8; c >= 1; c >>= 1) {
    const FlowLayout L = flow_layout(c, (T + c - 1) / c, forward);
    if (L.total > kMaxSmem) break;
    fallback = c;
    const cudaError_t e = ensure_smem(kern, L.total);
    if (e != cudaSuccess) return e;
    if (active_clusters(kern, c, L.total) >= want) {
      cs = c;
      break;
    }
  }
  if (cs == 0) cs = fallback;
  if (cs == 0) return cudaSuccess;
  const FlowLayout L = flow_layout(cs, (T + cs - 1) / cs, forward);
  cudaError_t e = ensure_smem(kern, L.total);
  if (e != cudaSuccess) return e;
  // the sweeps are column-separable: more than kCols right-hand-side columns take one launch per
  // kCols of them (the factor units stream once per launch)
  for (int col0 = 0; col0 < b && e == cudaSuccess; col0 += kCols) {
    if (forward)
      e = launch_cluster(forward_flow_kernel, cs, njobs, kBlock, L.total, s, jobs, L.own, *fmap, col0);
    else
      e = launch_cluster(backward_flow_kernel, cs, njobs, kBlock, L.total, s, jobs, L.own, mode, *fmap, col0);
  }
  if (e == cudaSuccess) *launched = true;
  return e;
}

}  // namespace b200
