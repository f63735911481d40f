// C ABI of b200tau (include/b200tau.h): context, uploads and the batched solve driver.
//
// The context replaces the reference's per-thread DeviceStorage (src/Accelerator/
// DeviceStorage.hpp:55-144, DeviceStorage.cu:87-225) and DeviceAtom/DeviceConstants
// (DeviceStorage.cu:341-404): it owns the device tmatStore copy, one device record per atom,
// the angular tables, a stream, and a workspace of `slots` jobs (KKR matrix M in FP64, factor
// storage F in FP64 or FP32, and the N x b solution / residual / correction blocks).  A solve call
// packs the jobs into waves of at most `slots` jobs (largest N first), and per wave runs
//   kkr_build -> block elimination of F -> (refinement against M) -> tau00_l
// on the context stream.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/b200tau.h"
#include "common.cuh"

using namespace b200;

namespace {

struct AtomDev {
  int L = 0;
  int N = 0;       // n_spin_cant * nrmat
  int b = 0;       // kkrsz_ns of the central site
  unsigned char *dev = nullptr;  // one device buffer holding the five arrays below
  int cap_L = 0;                 // sites it has room for (re-registering a LIZ that fits reuses it)
  double *pos = nullptr;   // device, 3 x L
  int *lmax = nullptr;     // device, L
  int *store = nullptr;    // device, L
  int *perm = nullptr;     // device, L
  int *off = nullptr;      // device, L+1
  int store0 = 0;          // host copy of store[0]
  std::vector<int> h_store;
  double2 ubr[4], ubrd[4];
  bool valid = false;
};

// Bytes of an atom's device record for L sites: pos (3 L doubles), then lmax, store, perm (L ints
// each) and off (L + 1 ints).
size_t atom_bytes(int L) { return sizeof(double) * 3 * (size_t)L + sizeof(int) * (4 * (size_t)L + 1); }

// How a precision runs: factor type, refinement steps (0: direct from the Schur block).
struct Plan {
  FactorKind fk;
  int steps;
  bool f_separate;  // F is a second buffer (M kept for residuals)
};

}  // namespace

// One FP64 re-solve graph of a context (capi.cu, fallback_graph).
struct FallbackGraph {
  std::vector<long long> key;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

// One captured wave pipeline (capi.cu, wave_graph): build, elimination, refinement and tau00_l of
// every wave with the same shape and buffers; `launches` kernels per launch.
struct WaveGraph {
  std::vector<long long> key;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long launches = 0;
};

struct b200tau_ctx {
  int device = 0;
  int lmax = 3, ns = 1, npola = 1, kkrsz = 16, b = 16, blk = 1024;
  cudaStream_t stream = nullptr;
  Lookahead la;  // second stream and events of the elimination's look-ahead
  std::string err;
  AngularTables *d_tables = nullptr;
  double2 *d_tmat = nullptr;
  long tmat_ld = 0;
  int nstore = 0;
  int group_size = 0;
  std::vector<AtomDev> atoms;
  // workspace (per slot: M ld*ld double2, F ld*ld of the factor type, vec 3*ld*b double2)
  double2 *d_M = nullptr;
  unsigned char *d_F = nullptr;
  double2 *d_vec = nullptr;
  size_t m_elems = 0, f_bytes = 0, vec_elems = 0;
  int slots = 0;
  JobDev *d_jobs = nullptr;
  int jobs_cap = 0;
  JobDev *d_jobs3 = nullptr;  // the FP64 re-solve records of a mixed wave
  int jobs3_cap = 0;
  int *d_info = nullptr;   // 2 x slots: the wave's jobs, then their FP64 re-solve records
  int *d_conv = nullptr;   // per slot: refinement converged
  int *d_active = nullptr;  // slots + 1: the jobs still refining (residual launches)
  double *d_cnorm = nullptr;  // per slot: relative size of the last refinement correction
  int *d_err = nullptr;    // device error flags
  double2 *d_out = nullptr;
  size_t out_cap = 0;
  double2 *d_t0 = nullptr;  // dense-solve t0
  // adjoint (b200tau_solve_vjp): M^-1 per slot, and the call's cotangents / gradients
  double2 *d_V = nullptr;
  size_t v_elems = 0;
  int v_slots = 0;
  double2 *d_adj = nullptr;
  size_t adj_cap = 0;
  unsigned char *d_tdiag = nullptr;  // per (store, energy, spin) t block: exactly diagonal
  size_t tmat_cap = 0, tdiag_cap = 0;  // elements / flags the two buffers hold
  // per-job singular-pivot status of the last solve call, copied back wave by wave without a wait,
  // and the device error word read back with the outputs
  int *h_info = nullptr;
  int h_info_cap = 0, info_jobs = 0;
  std::vector<int> info_order;  // caller's job index of each entry of h_info
  int *h_err = nullptr;
  long table_polls = kTablePolls;  // first wait of the KKR build's table copy (b200tau_set_build_wait)
  int pivoting = B200TAU_PIVOT_AUTO;  // b200tau_set_pivoting
  int *d_piv = nullptr;               // panel pivoting's per-slot buffers (pivot_ints(ld) each)
  size_t piv_ints = 0;
  int piv_slots = 0;
  long launches = 0;
  bool fallback_on = true;
  double2 *d_ffb = nullptr;  // FP64 factor storage of those re-solves, one per slot
  size_t ffb_elems = 0;
  int *d_fbcount = nullptr;  // their number (device counter of the last solve call)
  int max_slots = 64;
  // refinement rounds, FP64 and MIXED; MIXED stops early per job once the correction estimate
  // is below kRefineTol of tau00 (block_lu.cu, converge_check_kernel)
  int refine_steps[2] = {1, 10};
  // profiling of the trailing-update launches (b200tau_set_profiling)
  bool profiling = false;
  std::vector<cudaEvent_t> events;
  KernelTimer timer;
  double prof_ms = 0.0, prof_flops = 0.0;
  long prof_launches = 0;
  // phase timing (b200tau_profile_phases): event pairs around build, elimination, refinement
  std::vector<cudaEvent_t> pev;
  std::vector<int> pev_phase;
  int pev_used = 0;
  double phase_ms[3] = {0.0, 0.0, 0.0};
  // tensor-core trailing update of the mixed path: operand packs + TMA descriptors
  int mixed_engine = B200TAU_ENGINE_TENSOR;
  int mixed_sweep = B200TAU_SWEEP_FP32;  // arithmetic of the mixed path's correction solve
  TcMaps tc;
  float *d_pack = nullptr;
  int tc_ld = 0, tc_slots = 0;
  // the mixed path's FP64 re-solve as graphs with a conditional body (fallback_graph)
  cudaStream_t cap_stream = nullptr;
  std::vector<FallbackGraph> fb;  // most recently used last
  std::vector<WaveGraph> wg;      // captured wave pipelines, most recently used last
  bool graphs_on = true;          // b200tau_set_graphs
  int pair_min_rest = kPairMinRest;  // b200tau_set_paired_steps
  // (N rounded up to 64, min_rest) from b200tau_autotune_paired_steps: a wave whose largest N
  // falls in a tuned bucket uses that bucket's threshold; the autotuner's trials set pair_trial
  std::vector<std::pair<int, int>> pair_table;
  int pair_trial = -1;
  // b200tau_set_keep_factors: the last FP64 solve's wave (factors F, KKR matrix M, refined X, slots
  // in `kept_order` order), reusable once by b200tau_solve_vjp on the same jobs
  bool keep_factors = false;
  bool kept_valid = false;
  std::vector<b200tau_job> kept_jobs;
  std::vector<int> kept_order;
  int kept_ld = 0;
  // converged flags after the first refinement rounds, copied back without a wait: the next
  // call's estimate of how many jobs the later rounds' sweeps serve
  int *h_hint = nullptr;
  cudaEvent_t hint_ev = nullptr;
  bool hint_pending = false;
  int h_hint_cap = 0, hint_n = 0, active_hint = 0;
};

namespace {

int fail(b200tau_ctx *c, int code, const char *fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return code;
}

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? B200TAU_ERR_OOM : B200TAU_ERR_CUDA, \
                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

void free_atom(AtomDev &a) {
  cudaFree(a.dev);
  a = AtomDev();
}

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// B200TAU_PIVOT_AUTO takes panel pivoting for FP32 factors from this N up: the row selection's
// latency per step is then small beside the trailing update, and the MIXED refinement of these
// (non-collinear, N = 4320) matrices needs it.  FP64 factors keep the pivots inside the diagonal
// blocks: as accurate on these matrices (within the reference's own zgesv / zblock_lu spread) and
// faster.
constexpr int kPanelAutoN = 3000;

bool use_panel(const b200tau_ctx *ctx, int maxN, FactorKind fk) {
  return ctx->pivoting == B200TAU_PIVOT_PANEL ||
         (ctx->pivoting == B200TAU_PIVOT_AUTO && fk == kFactorFP32 && maxN >= kPanelAutoN);
}

int ensure_piv(b200tau_ctx *ctx, int ld, int slots) {
  const size_t per = (size_t)pivot_ints(ld);
  if (ctx->d_piv && per <= ctx->piv_ints && slots <= ctx->piv_slots) return B200TAU_OK;
  CK(cudaStreamSynchronize(ctx->stream));  // (work still queued may use the old buffers)
  cudaFree(ctx->d_piv);
  ctx->d_piv = nullptr;
  ctx->piv_ints = std::max(per, ctx->piv_ints);
  ctx->piv_slots = std::max(slots, ctx->piv_slots);
  CK(cudaMalloc(&ctx->d_piv, sizeof(int) * ctx->piv_ints * ctx->piv_slots));
  return B200TAU_OK;
}

Plan plan_for(const b200tau_ctx *ctx, int prec) {
  Plan p;
  p.steps = ctx->refine_steps[prec == B200TAU_PREC_MIXED ? 1 : 0];
  p.fk = prec == B200TAU_PREC_MIXED ? kFactorFP32 : kFactorFP64;
  p.f_separate = (p.fk == kFactorFP32) || p.steps > 0;
  return p;
}

size_t f_elem_bytes(const Plan &p) { return p.fk == kFactorFP32 ? sizeof(float2) : sizeof(double2); }

int ensure_workspace(b200tau_ctx *ctx, int ld, int slots, const Plan &p) {
  const size_t m_need = (size_t)ld * ld;
  const size_t f_need = p.f_separate ? m_need * f_elem_bytes(p) : 0;
  const size_t v_need = (size_t)3 * ld * kMaxB;
  const bool ok = ctx->d_M && m_need <= ctx->m_elems && f_need <= ctx->f_bytes &&
                  v_need <= ctx->vec_elems && slots <= ctx->slots;
  if (ok) return B200TAU_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  cudaFree(ctx->d_M);
  cudaFree(ctx->d_F);
  cudaFree(ctx->d_vec);
  cudaFree(ctx->d_info);
  cudaFree(ctx->d_conv);
  cudaFree(ctx->d_active);
  cudaFree(ctx->d_cnorm);
  ctx->d_M = nullptr;
  ctx->d_F = nullptr;
  ctx->d_vec = nullptr;
  ctx->d_info = nullptr;
  ctx->d_conv = nullptr;
  ctx->d_active = nullptr;
  ctx->d_cnorm = nullptr;
  const size_t m_el = std::max(m_need, ctx->m_elems);
  const size_t f_b = std::max(f_need, ctx->f_bytes);
  const size_t v_el = std::max(v_need, ctx->vec_elems);
  const int sl = std::max(slots, ctx->slots);
  CK(cudaMalloc(&ctx->d_M, m_el * sl * sizeof(double2)));
  if (f_b) CK(cudaMalloc(&ctx->d_F, f_b * sl));
  CK(cudaMalloc(&ctx->d_vec, v_el * sl * sizeof(double2)));
  CK(cudaMalloc(&ctx->d_info, sizeof(int) * 2 * sl));
  CK(cudaMalloc(&ctx->d_conv, sizeof(int) * sl));
  CK(cudaMalloc(&ctx->d_active, sizeof(int) * (sl + 1)));
  CK(cudaMalloc(&ctx->d_cnorm, sizeof(double) * sl));
  ctx->m_elems = m_el;
  ctx->f_bytes = f_b;
  ctx->vec_elems = v_el;
  ctx->slots = sl;
  return B200TAU_OK;
}

int ensure_jobs(b200tau_ctx *ctx, int n) {
  if (n <= ctx->jobs_cap) return B200TAU_OK;
  cudaFree(ctx->d_jobs);
  ctx->d_jobs = nullptr;
  CK(cudaMalloc(&ctx->d_jobs, sizeof(JobDev) * n));
  ctx->jobs_cap = n;
  return B200TAU_OK;
}

int ensure_out(b200tau_ctx *ctx, size_t n) {
  if (n <= ctx->out_cap) return B200TAU_OK;
  cudaFree(ctx->d_out);
  ctx->d_out = nullptr;
  CK(cudaMalloc(&ctx->d_out, sizeof(double2) * n));
  ctx->out_cap = n;
  return B200TAU_OK;
}

int choose_slots(b200tau_ctx *ctx, int ld, int njobs, const Plan &p, size_t extra_per_slot = 0) {
  size_t freeb = 0, totalb = 0;
  if (cudaMemGetInfo(&freeb, &totalb) != cudaSuccess) freeb = (size_t)8 << 30;
  // memory already held by the context's workspace counts as available to it
  freeb += ctx->m_elems * ctx->slots * sizeof(double2) + ctx->f_bytes * ctx->slots;
  const size_t per = (size_t)ld * ld * (sizeof(double2) + (p.f_separate ? f_elem_bytes(p) : 0)) +
                     (size_t)3 * ld * kMaxB * sizeof(double2) + extra_per_slot;
  const size_t budget = freeb / 2;
  int s = (int)std::max<size_t>(1, budget / std::max<size_t>(per, 1));
  s = std::min(s, ctx->max_slots);
  s = std::min(s, njobs);
  return std::max(s, 1);
}

void fill_slot(b200tau_ctx *ctx, JobDev &J, int slot, int ld, const Plan &p) {
  J.M = ctx->d_M + (size_t)slot * ctx->m_elems;
  J.F = p.f_separate ? static_cast<void *>(ctx->d_F + (size_t)slot * ctx->f_bytes) : static_cast<void *>(J.M);
  double2 *v = ctx->d_vec + (size_t)slot * ctx->vec_elems;
  J.X = v;
  J.R = v + (size_t)ld * kMaxB;
  J.Y = v + (size_t)2 * ld * kMaxB;
  J.ld = ld;
  J.conv = ctx->d_conv + slot;
  J.cnorm = ctx->d_cnorm + slot;
  J.slot = slot;
  J.err = ctx->d_err;
  J.piv = nullptr;
}

// N x N workspace per slot for M^-1 (adjoint, full tau).
int ensure_v(b200tau_ctx *ctx, int ld, int slots) {
  const size_t v_need = (size_t)ld * ld;
  if (ctx->d_V && v_need <= ctx->v_elems && slots <= ctx->v_slots) return B200TAU_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  cudaFree(ctx->d_V);
  ctx->d_V = nullptr;
  ctx->v_elems = std::max(v_need, ctx->v_elems);
  ctx->v_slots = std::max(slots, ctx->v_slots);
  CK(cudaMalloc(&ctx->d_V, sizeof(double2) * ctx->v_elems * ctx->v_slots));
  return B200TAU_OK;
}

TmatView tmat_view(const b200tau_ctx *ctx) {
  TmatView v;
  v.tmat = ctx->d_tmat;
  v.tmat_ld = ctx->tmat_ld;
  v.blk = ctx->blk;
  v.kkrsz = ctx->kkrsz;
  v.ns = ctx->ns;
  v.bstore = ctx->ns * ctx->kkrsz;
  v.colpol = ctx->npola != ctx->ns ? 1 : 0;
  return v;
}

// The slot's panel-pivoting buffer (ensure_piv has sized it for the call).
int *slot_piv(const b200tau_ctx *ctx, int slot) { return ctx->d_piv + (size_t)slot * ctx->piv_ints; }

// Clears the per-slot status of the first nw slots: singular-pivot info, converged flag, last
// correction size.
int reset_slot_status(b200tau_ctx *ctx, int nw) {
  CK(cudaMemsetAsync(ctx->d_info, 0, sizeof(int) * nw, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_info + ctx->slots, 0, sizeof(int) * nw, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_conv, 0, sizeof(int) * nw, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_cnorm, 0, sizeof(double) * nw, ctx->stream));
  return B200TAU_OK;
}

BuildParams build_params(const b200tau_ctx *ctx, const Plan &p) {
  BuildParams bp;
  bp.tables = ctx->d_tables;
  bp.tmat = ctx->d_tmat;
  bp.tmat_ld = ctx->tmat_ld;
  bp.blk = ctx->blk;
  bp.kkrsz = ctx->kkrsz;
  bp.ns = ctx->ns;
  bp.npola = ctx->npola;
  bp.f_kind = !p.f_separate ? 0 : (p.fk == kFactorFP32 ? 2 : 1);
  bp.tdiag = ctx->d_tdiag;
  bp.group = ctx->group_size;
  bp.g_mode = 0;
  bp.table_polls = ctx->table_polls;
  return bp;
}

// Phase timing: an event before and after each phase on the context stream, read back by
// b200tau_profile_phases.  Phases: 0 KKR build, 1 block elimination, 2 refinement and tau00_l.
int drain_phases(b200tau_ctx *ctx);

int phase_begin(b200tau_ctx *ctx) {
  if (!ctx->profiling || ctx->pev.empty()) return B200TAU_OK;
  if (ctx->pev_used + 2 > (int)ctx->pev.size()) {
    int rc = drain_phases(ctx);
    if (rc) return rc;
  }
  CK(cudaEventRecord(ctx->pev[ctx->pev_used], ctx->stream));
  return B200TAU_OK;
}

int phase_end(b200tau_ctx *ctx, int phase) {
  if (!ctx->profiling || ctx->pev.empty()) return B200TAU_OK;
  CK(cudaEventRecord(ctx->pev[ctx->pev_used + 1], ctx->stream));
  ctx->pev_phase[ctx->pev_used / 2] = phase;
  ctx->pev_used += 2;
  return B200TAU_OK;
}

int drain_phases(b200tau_ctx *ctx) {
  if (ctx->pev_used == 0) return B200TAU_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i + 1 < ctx->pev_used; i += 2) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->pev[i], ctx->pev[i + 1]));
    ctx->phase_ms[ctx->pev_phase[i / 2]] += ms;
  }
  ctx->pev_used = 0;
  return B200TAU_OK;
}

// Device pipeline for one wave whose JobDev records are already in ctx->d_jobs.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// 3-D float tensor (kTcKMax floats per row, `rows` rows per slot, `slots` slots) read in
// kTcChunk x box_rows boxes with 128-byte swizzle; out-of-range rows read as zero.
int encode_pack_map(b200tau_ctx *ctx, EncodeTiledFn enc, CUtensorMap *map, float *base, int rows, int slots,
                    int box_rows) {
  const cuuint64_t dims[3] = {(cuuint64_t)kTcKMax, (cuuint64_t)rows, (cuuint64_t)slots};
  const cuuint64_t strides[2] = {kTcKMax * sizeof(float), (cuuint64_t)rows * kTcKMax * sizeof(float)};
  const cuuint32_t box[3] = {(cuuint32_t)kTcChunk, (cuuint32_t)box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(ctx, B200TAU_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return B200TAU_OK;
}

int ensure_tc(b200tau_ctx *ctx, int ld, int slots) {
  if (ctx->d_pack && ld <= ctx->tc_ld && slots <= ctx->tc_slots) return B200TAU_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  cudaFree(ctx->d_pack);
  ctx->d_pack = nullptr;
  ld = std::max(ld, ctx->tc_ld);
  slots = std::max(slots, ctx->tc_slots);
  const size_t a_slot = (size_t)2 * ld * kTcKMax, b_slot = (size_t)ld * kTcKMax;
  const int counter_slots = (ld / kNb + 1) * kTcCountersPerStep;
  const size_t pack_bytes = sizeof(float) * 2 * (a_slot + b_slot) * slots;
  CK(cudaMalloc(&ctx->d_pack, pack_bytes + sizeof(int) * counter_slots));
  // pack rows past a step's trailing block feed only F's padding, but must be finite numbers
  CK(cudaMemset(ctx->d_pack, 0, pack_bytes + sizeof(int) * counter_slots));
  TcMaps &t = ctx->tc;
  t.a_slot = a_slot;
  t.b_slot = b_slot;
  t.a_hi = ctx->d_pack;
  t.a_lo = t.a_hi + a_slot * slots;
  t.b_hi = t.a_lo + a_slot * slots;
  t.b_lo = t.b_hi + b_slot * slots;
  t.counters = reinterpret_cast<int *>(t.b_lo + b_slot * slots);
  t.counter_slots = counter_slots;
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
  if (!fn || q != cudaDriverEntryPointSuccess) return fail(ctx, B200TAU_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  EncodeTiledFn enc = reinterpret_cast<EncodeTiledFn>(fn);
  int rc;
  if ((rc = encode_pack_map(ctx, enc, &t.tA_hi, t.a_hi, 2 * ld, slots, 128))) return rc;
  if ((rc = encode_pack_map(ctx, enc, &t.tA_lo, t.a_lo, 2 * ld, slots, 128))) return rc;
  if ((rc = encode_pack_map(ctx, enc, &t.tB_hi, t.b_hi, ld, slots, 256))) return rc;
  if ((rc = encode_pack_map(ctx, enc, &t.tB_lo, t.b_lo, ld, slots, 256))) return rc;
  if ((rc = encode_pack_map(ctx, enc, &t.tB2_hi, t.b_hi, ld, slots, 128))) return rc;
  if ((rc = encode_pack_map(ctx, enc, &t.tB2_lo, t.b_lo, ld, slots, 128))) return rc;
  ctx->tc_ld = ld;
  ctx->tc_slots = slots;
  return B200TAU_OK;
}

// Tensor map over the FP32 factor slots of the current wave (floats; column c of slot z starts at
// z * f_bytes + c * 2 ld * 4 bytes), the destination of the tensor-core update's TMA reduce-add.
int encode_factor_map(b200tau_ctx *ctx, int ld, int slots) {
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
  if (!fn || q != cudaDriverEntryPointSuccess) return fail(ctx, B200TAU_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  EncodeTiledFn enc = reinterpret_cast<EncodeTiledFn>(fn);
  const cuuint64_t dims[3] = {(cuuint64_t)2 * ld, (cuuint64_t)ld, (cuuint64_t)slots};
  const cuuint64_t strides[2] = {(cuuint64_t)2 * ld * sizeof(float), (cuuint64_t)ctx->f_bytes};
  const cuuint32_t box[3] = {128, (cuuint32_t)kTcPieceCols, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(&ctx->tc.tF, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, ctx->d_F, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(ctx, B200TAU_ERR_CUDA, "cuTensorMapEncodeTiled (F) failed (%d)", (int)r);
  const cuuint32_t wbox[3] = {32, (cuuint32_t)kTcPieceCols, 1};
  r = enc(&ctx->tc.tFw, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, ctx->d_F, dims, strides, wbox, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(ctx, B200TAU_ERR_CUDA, "cuTensorMapEncodeTiled (F, warp box) failed (%d)", (int)r);
  // the sweeps' operand units: 32 real rows x 32 columns per box, in the tensor core's MN-major
  // TF32 layout (128-byte swizzle on 32-byte atoms)
  const cuuint32_t ubox[3] = {32, 32, 1};
  r = enc(&ctx->tc.tFu, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, ctx->d_F, dims, strides, ubox, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(ctx, B200TAU_ERR_CUDA, "cuTensorMapEncodeTiled (F units) failed (%d)", (int)r);
  return B200TAU_OK;
}

// Fold the recorded (start, stop) event pairs into the profile totals.
int drain_timer(b200tau_ctx *ctx) {
  if (!ctx->profiling || ctx->timer.used == 0) return B200TAU_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i + 1 < ctx->timer.used; i += 2) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->timer.ev[i], ctx->timer.ev[i + 1]));
    ctx->prof_ms += ms;
    ctx->prof_launches += 1;
  }
  ctx->timer.used = 0;
  return B200TAU_OK;
}

// Algorithmic FLOPs of the trailing updates of one wave: sum over steps and jobs of
// 8 (N - k - kb)^2 kb (complex multiply-add = 8 real FLOPs).
// Algorithmic complex FLOPs of the tensor-core update launches (the ones the profiler times): per
// single step 8 rest^2 kb; per paired step (the elimination's schedule, block_lu.cu) only the
// combined pass over the trailing block after the second step, 8 rest2^2 (kb + kb2) -- the strips
// of the first step run as SIMT tiles outside the timed launches.
double trailing_flops(const std::vector<JobDev> &h, const Lookahead &la, int max_n, int max_N) {
  double f = 0.0;
  for (const JobDev &J : h)
    for (int k = 0; k < J.n; k += kNb) {
      const int k2 = k + kNb;
      const double kb = std::min(kNb, J.n - k);
      if (la.pair_min_rest > 0 && k2 < la.min_n && k2 + kNb < max_n && max_N - k2 - kNb >= la.pair_min_rest) {
        const double kb2 = std::min(kNb, J.n - k2);
        const double rest2 = J.N - k2 - kb2;
        f += 8.0 * rest2 * rest2 * (kb + kb2);
        k = k2;
        continue;
      }
      const double rest = J.N - k - kb;
      f += 8.0 * rest * rest * kb;
    }
  return f;
}


// Refinement rounds after which the jobs still refining are copied back (without a wait) as the
// next call's estimate of how many the later rounds' sweeps serve.
constexpr int kHintAfterRounds = 2;

// FP64 storage for re-solving any job of a mixed wave (one ld x ld block per slot) and the
// device counter of re-solved jobs.
int ensure_fallback(b200tau_ctx *ctx, int ld) {
  const size_t need = (size_t)ld * ld * ctx->slots;
  if (!ctx->d_fbcount) {
    CK(cudaMalloc(&ctx->d_fbcount, sizeof(int)));
    CK(cudaMemsetAsync(ctx->d_fbcount, 0, sizeof(int), ctx->stream));
  }
  if (ctx->jobs3_cap < ctx->slots) {
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->d_jobs3);
    ctx->d_jobs3 = nullptr;
    CK(cudaMalloc(&ctx->d_jobs3, sizeof(JobDev) * ctx->slots));
    ctx->jobs3_cap = ctx->slots;
  }
  if (ctx->d_ffb && need <= ctx->ffb_elems) return B200TAU_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  cudaFree(ctx->d_ffb);
  ctx->d_ffb = nullptr;
  CK(cudaMalloc(&ctx->d_ffb, sizeof(double2) * need));
  ctx->ffb_elems = need;
  return B200TAU_OK;
}

void destroy_fallback_graph(FallbackGraph &f) {
  if (f.exec) cudaGraphExecDestroy(f.exec);  // (a launch still in flight completes first)
  if (f.graph) cudaGraphDestroy(f.graph);
  f.exec = nullptr;
  f.graph = nullptr;
}

void drop_fallback_graphs(b200tau_ctx *ctx) {
  for (auto &f : ctx->fb) destroy_fallback_graph(f);
  ctx->fb.clear();
}

// Graph shapes kept per context: the waves of a call are full but for the last one.
constexpr size_t kFallbackGraphs = 4;
// Wave pipelines kept per context (the waves of an uneven batch have a few shapes).
constexpr size_t kWaveGraphs = 16;

void destroy_wave_graph(WaveGraph &g) {
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.graph) cudaGraphDestroy(g.graph);
  g.exec = nullptr;
  g.graph = nullptr;
}

void drop_wave_graphs(b200tau_ctx *ctx) {
  for (auto &g : ctx->wg) destroy_wave_graph(g);
  ctx->wg.clear();
}

// The FP64 re-solve of a mixed wave as one graph: a gate kernel, then a conditional node whose
// body - the re-solve records (converged jobs inactive), FP64 block elimination, the FP64
// refinement rounds and tau00 - runs only when some job did not converge.  So the host queues
// the re-solve without waiting for the refinement's outcome, and a wave whose jobs all converged
// pays one small launch for it.  The body is captured for the call's bounds (N <= ld, n <= ld - b;
// its kernels skip the steps and rows beyond each job's own), so every wave of nw jobs shares one
// graph; a graph is built on first use of its (nw, buffers) and kept (the records themselves are
// read from device memory when the graph runs).
int fallback_graph(b200tau_ctx *ctx, int nw, int ld, int b, int ns, int kkrsz, bool panel, cudaGraphExec_t *out) {
  const int steps = std::max(1, ctx->refine_steps[0]);
  const int maxN = ld, maxn = ld - b;
  int *finfo = ctx->d_info + ctx->slots;
  const std::vector<long long> key = {nw, ld, b, ns, kkrsz, steps, ctx->slots, panel ? 1 : 0,
                                      (long long)(uintptr_t)ctx->d_jobs, (long long)(uintptr_t)ctx->d_jobs3,
                                      (long long)(uintptr_t)ctx->d_ffb, (long long)(uintptr_t)ctx->d_info,
                                      (long long)(uintptr_t)ctx->d_fbcount, (long long)(uintptr_t)ctx->d_err};
  for (size_t i = 0; i < ctx->fb.size(); ++i)
    if (ctx->fb[i].key == key) {
      const FallbackGraph f = ctx->fb[i];  // most recently used last
      ctx->fb.erase(ctx->fb.begin() + (long)i);
      ctx->fb.push_back(f);
      *out = f.exec;
      return B200TAU_OK;
    }
  if (!ctx->cap_stream) CK(cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
  FallbackGraph f;
  f.key = key;
  cudaError_t e = cudaGraphCreate(&f.graph, 0);
  cudaGraphConditionalHandle h;
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, f.graph, 0, cudaGraphCondAssignDefault);
  cudaGraphNode_t gate = nullptr, cond = nullptr;
  if (e == cudaSuccess) e = add_fallback_gate_node(f.graph, &gate, ctx->d_jobs, nw, h);
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  if (e == cudaSuccess) e = cudaGraphAddNode(&cond, f.graph, &gate, 1, &cp);
  if (e == cudaSuccess) {
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(ctx->cap_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      e = launch_fallback_prepare(ctx->d_jobs, ctx->d_jobs3, nw, ctx->d_ffb, (size_t)ld * ld, maxN, ctx->d_fbcount,
                                  panel, ctx->cap_stream, nullptr);
      if (e == cudaSuccess)
        e = launch_eliminate(kFactorFP64, ctx->d_jobs3, nw, maxn, maxN, finfo, ctx->cap_stream, nullptr, nullptr,
                             nullptr, ctx->d_err, true, nullptr, panel);
      if (e == cudaSuccess)
        e = launch_solve_refine(kFactorFP64, ctx->d_jobs3, nw, maxn, maxN, b, steps, ns, kkrsz, finfo,
                                ctx->cap_stream, nullptr);
      cudaGraph_t captured = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(ctx->cap_stream, &captured);
      if (e == cudaSuccess) e = ec;
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&f.exec, f.graph, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    destroy_fallback_graph(f);
    return fail(ctx, B200TAU_ERR_CUDA, "building the FP64 re-solve graph: %s", cudaGetErrorString(e));
  }
  if (ctx->fb.size() >= kFallbackGraphs) {
    destroy_fallback_graph(ctx->fb.front());
    ctx->fb.erase(ctx->fb.begin());
  }
  ctx->fb.push_back(f);
  *out = f.exec;
  return B200TAU_OK;
}

// The previous call's count of jobs still refining after kHintAfterRounds rounds, once its copy
// has landed (never waits for it).
void refresh_active_hint(b200tau_ctx *ctx) {
  if (!ctx->hint_pending) return;
  const cudaError_t q = cudaEventQuery(ctx->hint_ev);
  if (q == cudaErrorNotReady) {
    if (cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();
    return;
  }
  ctx->hint_pending = false;
  if (q != cudaSuccess) return;
  int active = 0;
  for (int w = 0; w < ctx->hint_n; ++w) active += ctx->h_hint[w] == 0;
  ctx->active_hint = active;
}

// Initial solve, `p.steps` refinement rounds (converged jobs skip the later ones: every launch
// covers the wave and the kernels leave converged jobs at once), tau00_l, and the FP64 re-solve of
// jobs that did not converge.  The host never waits inside the wave.  `h` are the wave's records
// as uploaded to ctx->d_jobs.
int run_refinement(b200tau_ctx *ctx, const std::vector<JobDev> &h, int nw, int maxn, int maxN, int b, int ns,
                   int kkrsz, const Plan &p, const CUtensorMap *fmap, bool panel) {
  const bool fp32_sweep = p.fk == kFactorFP32 && ctx->mixed_sweep == B200TAU_SWEEP_FP32;
  refresh_active_hint(ctx);
  CK(launch_refine_begin(p.fk, ctx->d_jobs, nw, maxn, maxN, b, ctx->d_info, ctx->stream, &ctx->launches,
                         fp32_sweep, fmap));
  for (int it = 0; it < p.steps; ++it) {
    const int hint = it >= kHintAfterRounds ? ctx->active_hint : 0;
    CK(launch_refine_round(p.fk, ctx->d_jobs, nw, maxn, maxN, b, true, ctx->d_info, ctx->stream, &ctx->launches,
                           fp32_sweep, fmap, hint, ctx->d_active));
    if (it + 1 == kHintAfterRounds && p.steps > kHintAfterRounds && !ctx->hint_pending) {
      if (ctx->h_hint_cap < nw) {  // (no copy into the old buffer is pending)
        if (ctx->h_hint) cudaFreeHost(ctx->h_hint);
        ctx->h_hint = nullptr;
        ctx->h_hint_cap = 0;
        CK(cudaMallocHost(&ctx->h_hint, sizeof(int) * nw));
        ctx->h_hint_cap = nw;
      }
      if (!ctx->hint_ev) CK(cudaEventCreateWithFlags(&ctx->hint_ev, cudaEventDisableTiming));
      ctx->hint_n = nw;
      CK(cudaMemcpyAsync(ctx->h_hint, ctx->d_conv, sizeof(int) * ctx->hint_n, cudaMemcpyDeviceToHost,
                         ctx->stream));
      CK(cudaEventRecord(ctx->hint_ev, ctx->stream));
      ctx->hint_pending = true;
    }
  }
  CK(launch_refine_end(ctx->d_jobs, nw, ns, kkrsz, ctx->stream, &ctx->launches));
  if (p.fk != kFactorFP32 || !ctx->fallback_on) return B200TAU_OK;
  // Jobs whose FP32-factor refinement did not converge (condition numbers beyond what FP32 block
  // factors can refine, e.g. energies next to the real axis) take the FP64 path instead: an FP64
  // copy of the unmodified M, FP64 block elimination, the FP64 refinement rounds, tau00 from X -
  // the same kernels and arithmetic as a PREC_FP64 solve of the job.
  cudaGraphExec_t fb = nullptr;
  int rc = ensure_fallback(ctx, h[0].ld);
  if (rc || (rc = fallback_graph(ctx, nw, h[0].ld, b, ns, kkrsz, use_panel(ctx, maxN, kFactorFP64), &fb))) return rc;
  CK(cudaGraphLaunch(fb, ctx->stream));
  ctx->launches += 1;
  return B200TAU_OK;
}

int run_pipeline(b200tau_ctx *ctx, const std::vector<JobDev> &h, int nw, int maxn, int maxN, int ld, int ns,
                 int kkrsz, int b, const Plan &p, bool panel) {
  if (ctx->profiling && ctx->timer.used + 4 * (maxn / kNb + 2) > ctx->timer.cap) {
    int rc = drain_timer(ctx);
    if (rc) return rc;
  }
  const TcMaps *tc = nullptr;
  if (p.fk == kFactorFP32 && ctx->mixed_engine == B200TAU_ENGINE_TENSOR) {
    // the jobs' leading dimension `ld` (fill_slot) fixes the column stride of the factor map
    int rc = ensure_tc(ctx, ld, std::max(nw, ctx->slots));
    if (rc) return rc;
    if ((rc = encode_factor_map(ctx, ld, ctx->slots))) return rc;
    tc = &ctx->tc;
  }
  int rc = phase_begin(ctx);
  if (rc) return rc;
  CK(launch_eliminate(p.fk, ctx->d_jobs, nw, maxn, maxN, ctx->d_info, ctx->stream, &ctx->launches,
                      ctx->profiling ? &ctx->timer : nullptr, tc, ctx->d_err, false, &ctx->la, panel));
  if ((rc = phase_end(ctx, 1)) || (rc = phase_begin(ctx))) return rc;
  if (p.steps > 0) {
    if ((rc = run_refinement(ctx, h, nw, maxn, maxN, b, ns, kkrsz, p, tc ? &tc->tFu : nullptr, panel))) return rc;
  } else {
    CK(launch_finalize_direct(p.fk, ctx->d_jobs, nw, ns, kkrsz, ctx->d_info, ctx->stream, &ctx->launches));
  }
  return phase_end(ctx, 2);
}

// The device pipeline of a wave whose records are in ctx->d_jobs, as one CUDA graph: KKR build,
// block elimination (with its look-ahead stream), the initial solve and the refinement rounds (or
// tau00 from the Schur block), tau00_l.  Every kernel reads its job's sizes and pointers from the
// records in device memory, so one graph serves every wave of the same shape and buffers: a solve
// call then costs the host a record copy and a graph launch, and a host that stalls between the
// launches of a wave can no longer leave the GPU idle.  Captured on first use of its key; the
// refinement's later rounds size their sweep clusters for a quarter of the wave's jobs.  The FP64
// re-solve of unconverged mixed jobs stays a separate graph (fallback_graph).
int wave_graph(b200tau_ctx *ctx, int nw, int maxL, int maxn, int maxN, int ld, const Plan &p, bool panel,
               const TcMaps *tc, WaveGraph **out) {
  const bool fp32_sweep = p.fk == kFactorFP32 && ctx->mixed_sweep == B200TAU_SWEEP_FP32;
  const std::vector<long long> key = {
      nw, maxL, maxn, maxN, ld, ctx->b, ctx->ns, ctx->kkrsz, (long long)p.fk, p.steps, p.f_separate ? 1 : 0,
      fp32_sweep ? 1 : 0, panel ? 1 : 0, tc != nullptr ? 1 : 0, ctx->slots, (long long)ctx->f_bytes,
      ctx->tmat_ld, ctx->group_size, ctx->table_polls, (long long)(uintptr_t)ctx->d_jobs,
      (long long)(uintptr_t)ctx->d_info, (long long)(uintptr_t)ctx->d_active, (long long)(uintptr_t)ctx->d_err,
      (long long)(uintptr_t)ctx->d_tmat, (long long)(uintptr_t)ctx->d_tdiag, (long long)(uintptr_t)ctx->d_F,
      (long long)(uintptr_t)ctx->d_pack, ctx->tc_ld, ctx->tc_slots, ctx->la.min_n, ctx->la.pair_min_rest};
  for (size_t i = 0; i < ctx->wg.size(); ++i)
    if (ctx->wg[i].key == key) {
      const WaveGraph g = ctx->wg[i];  // most recently used last
      ctx->wg.erase(ctx->wg.begin() + (long)i);
      ctx->wg.push_back(g);
      *out = &ctx->wg.back();
      return B200TAU_OK;
    }
  if (!ctx->cap_stream) CK(cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
  WaveGraph g;
  g.key = key;
  cudaStream_t cs = ctx->cap_stream;
  long n = 0;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    e = launch_kkr_build(ctx->d_jobs, nw, maxL, build_params(ctx, p), ctx->d_err, cs, &n);
    if (e == cudaSuccess)
      e = launch_eliminate(p.fk, ctx->d_jobs, nw, maxn, maxN, ctx->d_info, cs, &n, nullptr, tc, ctx->d_err, false,
                           &ctx->la, panel);
    if (p.steps > 0) {
      const CUtensorMap *fmap = tc ? &tc->tFu : nullptr;
      if (e == cudaSuccess)
        e = launch_refine_begin(p.fk, ctx->d_jobs, nw, maxn, maxN, ctx->b, ctx->d_info, cs, &n, fp32_sweep, fmap);
      // rounds after kHintAfterRounds size their sweep clusters for a quarter of the wave (most jobs
      // have converged by then; if more are left their clusters run in two waves, which costs about
      // what the smaller clusters would)
      for (int it = 0; it < p.steps && e == cudaSuccess; ++it)
        e = launch_refine_round(p.fk, ctx->d_jobs, nw, maxn, maxN, ctx->b, true, ctx->d_info, cs, &n, fp32_sweep,
                                fmap, it >= kHintAfterRounds ? std::max(1, (nw + 3) / 4) : 0, ctx->d_active);
      if (e == cudaSuccess) e = launch_refine_end(ctx->d_jobs, nw, ctx->ns, ctx->kkrsz, cs, &n);
    } else if (e == cudaSuccess) {
      e = launch_finalize_direct(p.fk, ctx->d_jobs, nw, ctx->ns, ctx->kkrsz, ctx->d_info, cs, &n);
    }
    const cudaError_t ec = cudaStreamEndCapture(cs, &g.graph);
    if (e == cudaSuccess) e = ec;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g.exec, g.graph, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    destroy_wave_graph(g);
    return fail(ctx, B200TAU_ERR_CUDA, "capturing the wave pipeline: %s", cudaGetErrorString(e));
  }
  g.launches = n;
  if (ctx->wg.size() >= kWaveGraphs) {
    destroy_wave_graph(ctx->wg.front());
    ctx->wg.erase(ctx->wg.begin());
  }
  ctx->wg.push_back(g);
  *out = &ctx->wg.back();
  return B200TAU_OK;
}

// Device buffers of one b200tau_solve_vjp call (job-indexed in the caller's order).
struct AdjointBufs {
  const double2 *taubar;   // njobs x b x b
  double2 *tbar;           // sum of L over jobs, x b x b
  double2 *dlogdet;        // same, or null
  const long *site_off;    // host: first output block of each job
};

// The paired-steps threshold of a wave whose largest N is max_N: the autotuner's trial value while
// it runs, else the tuned value of max_N's 64-bucket, else the context's setting.
int pair_min_rest_for(const b200tau_ctx *ctx, int max_N) {
  if (ctx->pair_trial >= 0) return ctx->pair_trial;
  const int bucket = round_up(max_N, 64);
  for (const auto &e : ctx->pair_table)
    if (e.first == bucket) return e.second;
  return ctx->pair_min_rest;
}

int run_wave(b200tau_ctx *ctx, const b200tau_job *jobs, const int *idx, int nw, int ld, const Plan &p,
             double2 *out_base, const AdjointBufs *adj = nullptr, bool reuse_factors = false) {
  std::vector<JobDev> h(nw);
  int maxL = 0, maxN = 0, maxn = 0;
  for (int w = 0; w < nw; ++w) maxN = std::max(maxN, ctx->atoms[jobs[idx[w]].atom].N);
  // the adjoint forms M^-1 from block factors without row moves
  const bool panel = adj == nullptr && use_panel(ctx, maxN, p.fk);
  for (int w = 0; w < nw; ++w) {
    const b200tau_job &jb = jobs[idx[w]];
    const AtomDev &a = ctx->atoms[jb.atom];
    JobDev &J = h[w];
    std::memset(&J, 0, sizeof(J));
    J.energy = make_double2(jb.energy[0], jb.energy[1]);
    J.prel = make_double2(jb.prel[0], jb.prel[1]);
    J.pos = a.pos;
    J.lmax = a.lmax;
    J.store = a.store;
    J.perm = a.perm;
    J.off = a.off;
    fill_slot(ctx, J, w, ld, p);
    if (panel) J.piv = slot_piv(ctx, w);
    J.L = a.L;
    J.N = a.N;
    J.b = a.b;
    J.n = a.N - a.b;
    J.iie = jb.iie;
    J.ispin = jb.ispin;
    const long jsm = (ctx->npola != ctx->ns) ? (long)ctx->kkrsz * ctx->kkrsz * jb.ispin : 0;
    J.t0 = ctx->d_tmat + (long)a.store0 * ctx->tmat_ld + (long)jb.iie * ctx->blk + jsm;
    J.t0_ld = ctx->b;
    J.out = out_base + (size_t)idx[w] * ctx->b * ctx->b;
    J.out_mode = 0;
    if (adj) {  // raw tau00 out; M^-1 workspace; this job's cotangent and gradient blocks
      const size_t bb = (size_t)ctx->b * ctx->b;
      J.out_mode = 1;
      J.V = ctx->d_V + (size_t)w * ctx->v_elems;
      J.taubar = adj->taubar + (size_t)idx[w] * bb;
      J.tbar = adj->tbar + (size_t)adj->site_off[idx[w]] * bb;
      J.dlogdet = adj->dlogdet ? adj->dlogdet + (size_t)adj->site_off[idx[w]] * bb : nullptr;
    }
    for (int k = 0; k < 4; ++k) {
      J.ubr[k] = a.ubr[k];
      J.ubrd[k] = a.ubrd[k];
    }
    maxL = std::max(maxL, a.L);
    maxN = std::max(maxN, a.N);
    maxn = std::max(maxn, a.N - a.b);
  }
  ctx->la.min_n = maxn;
  for (int w = 0; w < nw; ++w) ctx->la.min_n = std::min(ctx->la.min_n, h[w].n);
  ctx->la.pair_min_rest = pair_min_rest_for(ctx, maxN);
  CK(cudaMemcpyAsync(ctx->d_jobs, h.data(), sizeof(JobDev) * nw, cudaMemcpyHostToDevice, ctx->stream));
  if (reuse_factors) {
    // the forward solve of these jobs left M, its FP64 block factors and the refined X in these
    // slots: raw tau00 from X, then the adjoint's own launches, no second factorisation
    CK(launch_refine_end(ctx->d_jobs, nw, ctx->ns, ctx->kkrsz, ctx->stream, &ctx->launches));
    BuildParams gp = build_params(ctx, p);
    gp.f_kind = 0;
    gp.g_mode = 1;
    CK(launch_kkr_build(ctx->d_jobs, nw, maxL, gp, ctx->d_err, ctx->stream, &ctx->launches));
    CK(launch_inverse(ctx->d_jobs, nw, maxn, maxN, ctx->stream, &ctx->launches));
    CK(launch_vjp_assemble(ctx->d_jobs, nw, maxL, ctx->kkrsz, ctx->ns, ctx->stream, &ctx->launches));
    return B200TAU_OK;
  }
  int rc = reset_slot_status(ctx, nw);
  if (rc) return rc;
  if (ctx->graphs_on && !ctx->profiling && adj == nullptr) {
    const TcMaps *tc = nullptr;
    if (p.fk == kFactorFP32 && ctx->mixed_engine == B200TAU_ENGINE_TENSOR) {
      if ((rc = ensure_tc(ctx, ld, std::max(nw, ctx->slots)))) return rc;
      if ((rc = encode_factor_map(ctx, ld, ctx->slots))) return rc;
      tc = &ctx->tc;
    }
    WaveGraph *g = nullptr;
    if ((rc = wave_graph(ctx, nw, maxL, maxn, maxN, ld, p, panel, tc, &g))) return rc;
    CK(cudaGraphLaunch(g->exec, ctx->stream));
    ctx->launches += g->launches;
    if (p.fk != kFactorFP32 || !ctx->fallback_on || p.steps == 0) return B200TAU_OK;
    cudaGraphExec_t fb = nullptr;
    if ((rc = ensure_fallback(ctx, ld)) ||
        (rc = fallback_graph(ctx, nw, ld, ctx->b, ctx->ns, ctx->kkrsz, use_panel(ctx, maxN, kFactorFP64), &fb)))
      return rc;
    CK(cudaGraphLaunch(fb, ctx->stream));
    ctx->launches += 1;
    return B200TAU_OK;
  }
  if (rc || (rc = phase_begin(ctx))) return rc;
  CK(launch_kkr_build(ctx->d_jobs, nw, maxL, build_params(ctx, p), ctx->d_err, ctx->stream, &ctx->launches));
  if ((rc = phase_end(ctx, 0))) return rc;
  if (ctx->profiling) ctx->prof_flops += trailing_flops(h, ctx->la, maxn, maxN);
  if ((rc = run_pipeline(ctx, h, nw, maxn, maxN, ld, ctx->ns, ctx->kkrsz, ctx->b, p, panel))) return rc;
  if (!adj) return B200TAU_OK;
  // adjoint: G into M's storage (M is no longer needed once X is refined), M^-1 from the factors,
  // then the per-site contractions
  BuildParams gp = build_params(ctx, p);
  gp.f_kind = 0;
  gp.g_mode = 1;
  CK(launch_kkr_build(ctx->d_jobs, nw, maxL, gp, ctx->d_err, ctx->stream, &ctx->launches));
  CK(launch_inverse(ctx->d_jobs, nw, maxn, maxN, ctx->stream, &ctx->launches));
  CK(launch_vjp_assemble(ctx->d_jobs, nw, maxL, ctx->kkrsz, ctx->ns, ctx->stream, &ctx->launches));
  return B200TAU_OK;
}

int check_info(b200tau_ctx *ctx, const int *info, const int *idx, int nw) {
  for (int w = 0; w < nw; ++w)
    if (info[w] != 0)
      return fail(ctx, B200TAU_ERR_SINGULAR,
                  info[w] > 0 ? "job %d: singular diagonal block at column %d"
                              : "job %d: 1 - Delta is singular",
                  idx[w], info[w] > 0 ? info[w] - 1 : 0);
  return B200TAU_OK;
}

// Page-locked host room for the per-job status of a call of n jobs.
int ensure_host_info(b200tau_ctx *ctx, int n) {
  if (n <= ctx->h_info_cap) return B200TAU_OK;
  CK(cudaStreamSynchronize(ctx->stream));  // no copy into the old buffer is pending
  if (ctx->h_info) cudaFreeHost(ctx->h_info);
  ctx->h_info = nullptr;
  ctx->h_info_cap = 0;
  CK(cudaMallocHost(&ctx->h_info, sizeof(int) * (size_t)n));
  ctx->h_info_cap = n;
  return B200TAU_OK;
}

// The status of the last solve call's jobs, once the stream has been synchronised.
int check_host_info(b200tau_ctx *ctx) {
  const int n = ctx->info_jobs;
  ctx->info_jobs = 0;
  return n > 0 ? check_info(ctx, ctx->h_info, ctx->info_order.data(), n) : B200TAU_OK;
}

int validate_jobs(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs) {
  if (!ctx->d_tmat) return fail(ctx, B200TAU_ERR_STATE, "solve before b200tau_upload_tmat");
  for (int j = 0; j < njobs; ++j) {
    const b200tau_job &jb = jobs[j];
    if (jb.atom < 0 || jb.atom >= (int)ctx->atoms.size() || !ctx->atoms[jb.atom].valid)
      return fail(ctx, B200TAU_ERR_ARG, "job %d: atom %d not registered", j, jb.atom);
    if (jb.iie < 0 || jb.iie >= ctx->group_size)
      return fail(ctx, B200TAU_ERR_ARG, "job %d: iie %d outside the uploaded group (%d)", j, jb.iie,
                  ctx->group_size);
    const int nspin = (ctx->npola != ctx->ns) ? 2 : 1;
    if (jb.ispin < 0 || jb.ispin >= nspin)
      return fail(ctx, B200TAU_ERR_ARG, "job %d: ispin %d invalid", j, jb.ispin);
    if (jb.reserved != 0) return fail(ctx, B200TAU_ERR_ARG, "job %d: reserved field must be 0", j);
    const AtomDev &a = ctx->atoms[jb.atom];
    for (int s : a.h_store)
      if (s < 0 || s >= ctx->nstore)
        return fail(ctx, B200TAU_ERR_ARG, "atom %d: store index %d outside tmatStore (%d)", jb.atom,
                    s, ctx->nstore);
  }
  return B200TAU_OK;
}

// Enqueues every wave of the call; the host does not wait.  Each wave's singular-pivot status is
// copied into ctx->h_info (caller order in ctx->info_order) behind the wave, for check_host_info
// after the caller's synchronisation.
int solve_impl(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs, int prec, double2 *dev_out) {
  ctx->info_jobs = 0;
  if (njobs == 0) return B200TAU_OK;
  int rc = validate_jobs(ctx, jobs, njobs);
  if (rc) return rc;
  const Plan p = plan_for(ctx, prec);
  std::vector<int> order(njobs);
  for (int j = 0; j < njobs; ++j) order[j] = j;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return ctx->atoms[jobs[a].atom].N > ctx->atoms[jobs[b].atom].N;
  });
  const int maxN = ctx->atoms[jobs[order[0]].atom].N;
  const int ld = round_up(maxN, 64);
  // mixed with the FP64 re-solve enabled also holds an FP64 copy of M per slot
  const size_t extra = (p.fk == kFactorFP32 && ctx->fallback_on) ? (size_t)ld * ld * sizeof(double2) : 0;
  const int slots = choose_slots(ctx, ld, njobs, p, extra);
  if ((rc = ensure_workspace(ctx, ld, slots, p))) return rc;
  if ((rc = ensure_jobs(ctx, slots))) return rc;
  if ((rc = ensure_host_info(ctx, njobs))) return rc;
  // (the FP64 re-solve of unconverged MIXED jobs may pivot differently from the wave)
  if ((use_panel(ctx, maxN, p.fk) || use_panel(ctx, maxN, kFactorFP64)) && (rc = ensure_piv(ctx, ld, slots)))
    return rc;
  ctx->launches = 0;
  if (ctx->d_fbcount) CK(cudaMemsetAsync(ctx->d_fbcount, 0, sizeof(int), ctx->stream));
  ctx->kept_valid = false;
  for (int w0 = 0; w0 < njobs; w0 += slots) {
    const int nw = std::min(slots, njobs - w0);
    if ((rc = run_wave(ctx, jobs, &order[w0], nw, ld, p, dev_out))) return rc;
    CK(cudaMemcpyAsync(ctx->h_info + w0, ctx->d_info, sizeof(int) * nw, cudaMemcpyDeviceToHost, ctx->stream));
  }
  ctx->info_order = order;
  ctx->info_jobs = njobs;
  // one FP64 wave with M kept beside its block factors, X refined, pivots inside the diagonal blocks:
  // what b200tau_solve_vjp needs from a forward solve
  if (ctx->keep_factors && njobs <= slots && p.fk == kFactorFP64 && p.f_separate && p.steps > 0 &&
      !use_panel(ctx, maxN, p.fk)) {
    ctx->kept_jobs.assign(jobs, jobs + njobs);
    ctx->kept_order = order;
    ctx->kept_ld = ld;
    ctx->kept_valid = true;
  }
  return B200TAU_OK;
}

bool same_jobs(const b200tau_job &a, const b200tau_job &b) {
  return a.atom == b.atom && a.iie == b.iie && a.ispin == b.ispin && a.energy[0] == b.energy[0] &&
         a.energy[1] == b.energy[1] && a.prel[0] == b.prel[0] && a.prel[1] == b.prel[1];
}

// Does the kept forward wave hold exactly these jobs (same order)?
bool kept_matches(const b200tau_ctx *ctx, const b200tau_job *jobs, int njobs) {
  if (!ctx->kept_valid || (int)ctx->kept_jobs.size() != njobs) return false;
  for (int j = 0; j < njobs; ++j)
    if (!same_jobs(ctx->kept_jobs[j], jobs[j])) return false;
  return true;
}

// The device error word as copied to ctx->h_err by the caller's last enqueued read (the stream
// has been synchronised since); a set word is cleared on the device and reported.
int check_host_err(b200tau_ctx *ctx) {
  const int flags = *ctx->h_err;
  if (flags) {
    *ctx->h_err = 0;
    CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return fail(ctx, B200TAU_ERR_TIMEOUT, "a device-side wait exceeded its bound (flags %d)", flags);
  }
  return B200TAU_OK;
}

int check_err_flags(b200tau_ctx *ctx) {
  CK(cudaMemcpyAsync(ctx->h_err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return check_host_err(ctx);
}

int check_prec(b200tau_ctx *ctx, int prec) {
  if (prec != B200TAU_PREC_FP64 && prec != B200TAU_PREC_MIXED)
    return fail(ctx, B200TAU_ERR_ARG, "unknown precision %d", prec);
  return B200TAU_OK;
}

}  // namespace

extern "C" {

int b200tau_create(b200tau_ctx **out, int device, int lmax, int n_spin_cant, int n_spin_pola) {
  if (!out) return B200TAU_ERR_ARG;
  *out = nullptr;
  if (lmax < 0 || lmax > kMaxLmax || (n_spin_cant != 1 && n_spin_cant != 2) ||
      (n_spin_pola != 1 && n_spin_pola != 2) || (n_spin_cant == 2 && n_spin_pola != 2))
    return B200TAU_ERR_ARG;
  b200tau_ctx *ctx = new b200tau_ctx();
  ctx->device = device;
  ctx->lmax = lmax;
  ctx->ns = n_spin_cant;
  ctx->npola = n_spin_pola;
  ctx->kkrsz = (lmax + 1) * (lmax + 1);
  ctx->b = n_spin_cant * ctx->kkrsz;
  ctx->blk = (2 * ctx->kkrsz) * (2 * ctx->kkrsz);
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->la.s2, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->la.panel, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->la.diag, cudaEventDisableTiming);
  AngularTables tab;
  if (build_angular_tables(lmax, &tab)) e = cudaErrorInvalidValue;
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_tables, sizeof(AngularTables));
  if (e == cudaSuccess) e = cudaMemcpy(ctx->d_tables, &tab, sizeof(tab), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_err, sizeof(int));
  if (e == cudaSuccess) *ctx->h_err = 0;
  if (e != cudaSuccess) {
    int code = e == cudaErrorMemoryAllocation ? B200TAU_ERR_OOM : B200TAU_ERR_CUDA;
    b200tau_destroy(ctx);
    return code;
  }
  *out = ctx;
  return B200TAU_OK;
}

void b200tau_destroy(b200tau_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->la.s2) cudaStreamSynchronize(ctx->la.s2);
  for (auto &a : ctx->atoms) free_atom(a);
  cudaFree(ctx->d_tables);
  cudaFree(ctx->d_tmat);
  cudaFree(ctx->d_M);
  cudaFree(ctx->d_F);
  cudaFree(ctx->d_vec);
  cudaFree(ctx->d_jobs);
  cudaFree(ctx->d_jobs3);
  cudaFree(ctx->d_info);
  cudaFree(ctx->d_conv);
  cudaFree(ctx->d_active);
  cudaFree(ctx->d_cnorm);
  cudaFree(ctx->d_err);
  cudaFree(ctx->d_out);
  cudaFree(ctx->d_t0);
  cudaFree(ctx->d_tdiag);
  cudaFree(ctx->d_pack);
  cudaFree(ctx->d_V);
  cudaFree(ctx->d_adj);
  cudaFree(ctx->d_ffb);
  cudaFree(ctx->d_fbcount);
  cudaFree(ctx->d_piv);
  for (auto &e : ctx->events) cudaEventDestroy(e);
  for (auto &e : ctx->pev) cudaEventDestroy(e);
  if (ctx->la.panel) cudaEventDestroy(ctx->la.panel);
  if (ctx->la.diag) cudaEventDestroy(ctx->la.diag);
  if (ctx->la.s2) cudaStreamDestroy(ctx->la.s2);
  drop_fallback_graphs(ctx);
  drop_wave_graphs(ctx);
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  if (ctx->hint_ev) cudaEventDestroy(ctx->hint_ev);
  if (ctx->h_hint) cudaFreeHost(ctx->h_hint);
  if (ctx->h_info) cudaFreeHost(ctx->h_info);
  if (ctx->h_err) cudaFreeHost(ctx->h_err);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char *b200tau_last_error(const b200tau_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void *b200tau_stream(b200tau_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

long b200tau_last_launch_count(const b200tau_ctx *ctx) { return ctx ? ctx->launches : 0; }

long b200tau_last_fallback_count(const b200tau_ctx *ctx) {
  if (!ctx || !ctx->d_fbcount) return 0;
  int n = 0;
  if (cudaSetDevice(ctx->device) != cudaSuccess ||
      cudaMemcpy(&n, ctx->d_fbcount, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  return n;
}

int b200tau_gaunt_numbers(int lmax, double *cgnt) {
  if (lmax < 0 || lmax > kMaxLmax || !cgnt) return B200TAU_ERR_ARG;
  gaunt_numbers(lmax, cgnt);
  return B200TAU_OK;
}

int b200tau_set_profiling(b200tau_ctx *ctx, int enable) {
  if (!ctx) return B200TAU_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  if (enable && ctx->events.empty()) {
    ctx->events.resize(4096);
    for (auto &e : ctx->events) CK(cudaEventCreate(&e));
    ctx->timer.ev = ctx->events.data();
    ctx->timer.cap = (int)ctx->events.size();
  }
  if (enable && ctx->pev.empty()) {
    ctx->pev.resize(512);
    for (auto &e : ctx->pev) CK(cudaEventCreate(&e));
    ctx->pev_phase.assign(ctx->pev.size() / 2, 0);
  }
  ctx->timer.used = 0;
  ctx->pev_used = 0;
  ctx->profiling = enable != 0;
  ctx->prof_ms = ctx->prof_flops = 0.0;
  ctx->prof_launches = 0;
  for (double &m : ctx->phase_ms) m = 0.0;
  return B200TAU_OK;
}

int b200tau_profile_phases(b200tau_ctx *ctx, double *ms3) {
  if (!ctx || !ms3) return B200TAU_ERR_ARG;
  int rc = drain_phases(ctx);
  if (rc) return rc;
  for (int i = 0; i < 3; ++i) ms3[i] = ctx->phase_ms[i];
  return B200TAU_OK;
}

int b200tau_profile_read(b200tau_ctx *ctx, double *ms, long *launches, double *flops) {
  if (!ctx) return B200TAU_ERR_ARG;
  int rc = drain_timer(ctx);
  if (rc) return rc;
  if (ms) *ms = ctx->prof_ms;
  if (launches) *launches = ctx->prof_launches;
  if (flops) *flops = ctx->prof_flops;
  return B200TAU_OK;
}

int b200tau_set_mixed_engine(b200tau_ctx *ctx, int engine) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (engine != B200TAU_ENGINE_TENSOR && engine != B200TAU_ENGINE_SIMT)
    return fail(ctx, B200TAU_ERR_ARG, "unknown engine %d", engine);
  ctx->mixed_engine = engine;
  return B200TAU_OK;
}

int b200tau_set_keep_factors(b200tau_ctx *ctx, int enable) {
  if (!ctx) return B200TAU_ERR_ARG;
  ctx->keep_factors = enable != 0;
  if (!enable) ctx->kept_valid = false;
  return B200TAU_OK;
}

int b200tau_set_paired_steps(b200tau_ctx *ctx, int min_rest) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (min_rest < 0) return fail(ctx, B200TAU_ERR_ARG, "paired steps: min_rest must be >= 0");
  ctx->pair_min_rest = min_rest;
  ctx->pair_table.clear();
  return B200TAU_OK;
}

int b200tau_set_graphs(b200tau_ctx *ctx, int enable) {
  if (!ctx) return B200TAU_ERR_ARG;
  ctx->graphs_on = enable != 0;
  return B200TAU_OK;
}

int b200tau_set_pivoting(b200tau_ctx *ctx, int mode) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (mode != B200TAU_PIVOT_AUTO && mode != B200TAU_PIVOT_BLOCK && mode != B200TAU_PIVOT_PANEL)
    return fail(ctx, B200TAU_ERR_ARG, "unknown pivoting mode %d", mode);
  ctx->pivoting = mode;
  return B200TAU_OK;
}

int b200tau_set_build_wait(b200tau_ctx *ctx, long polls) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (polls < 0) return fail(ctx, B200TAU_ERR_ARG, "build wait polls %ld < 0", polls);
  ctx->table_polls = polls;
  return B200TAU_OK;
}

int b200tau_set_mixed_fallback(b200tau_ctx *ctx, int enable) {
  if (!ctx) return B200TAU_ERR_ARG;
  ctx->fallback_on = enable != 0;
  return B200TAU_OK;
}

int b200tau_set_mixed_sweep(b200tau_ctx *ctx, int sweep) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (sweep != B200TAU_SWEEP_FP64 && sweep != B200TAU_SWEEP_FP32)
    return fail(ctx, B200TAU_ERR_ARG, "unknown sweep arithmetic %d", sweep);
  ctx->mixed_sweep = sweep;
  return B200TAU_OK;
}

int b200tau_set_refinement(b200tau_ctx *ctx, int prec, int steps) {
  if (!ctx) return B200TAU_ERR_ARG;
  int rc = check_prec(ctx, prec);
  if (rc) return rc;
  if (steps < 0 || steps > 16) return fail(ctx, B200TAU_ERR_ARG, "refinement steps %d outside 0..16", steps);
  ctx->refine_steps[prec == B200TAU_PREC_MIXED ? 1 : 0] = steps;
  return B200TAU_OK;
}

int b200tau_upload_tmat(b200tau_ctx *ctx, const double *tmat_store, long ld, int nstore, int blk_size) {
  if (!ctx) return B200TAU_ERR_ARG;
  ctx->kept_valid = false;
  if (!tmat_store || nstore <= 0 || blk_size != ctx->blk || ld < blk_size || ld % blk_size)
    return fail(ctx, B200TAU_ERR_ARG, "upload_tmat: bad arguments (ld %ld, nstore %d, blk %d, expected blk %d)",
                ld, nstore, blk_size, ctx->blk);
  CK(cudaSetDevice(ctx->device));
  const size_t elems = (size_t)ld * nstore;
  const int group = (int)(ld / blk_size);
  const size_t nflags = (size_t)nstore * group * 2;
  if (elems > ctx->tmat_cap || nflags > ctx->tdiag_cap) {
    CK(cudaStreamSynchronize(ctx->stream));  // solves still queued read the old buffers
    if (elems > ctx->tmat_cap) {
      cudaFree(ctx->d_tmat);
      ctx->d_tmat = nullptr;
      ctx->tmat_cap = 0;
      CK(cudaMalloc(&ctx->d_tmat, sizeof(double2) * elems));
      ctx->tmat_cap = elems;
    }
    if (nflags > ctx->tdiag_cap) {
      cudaFree(ctx->d_tdiag);
      ctx->d_tdiag = nullptr;
      ctx->tdiag_cap = 0;
      CK(cudaMalloc(&ctx->d_tdiag, nflags));
      ctx->tdiag_cap = nflags;
    }
  }
  // stream-ordered behind any solve still queued on the context
  CK(cudaMemcpyAsync(ctx->d_tmat, tmat_store, sizeof(double2) * elems, cudaMemcpyHostToDevice, ctx->stream));
  // Which t blocks are exactly diagonal (no spin-orbit or non-spherical coupling): the KKR build
  // then forms the block row t_i G_ij from the diagonal alone.  One flag per (store, energy, spin),
  // found on the device.
  CK(launch_tdiag_flags(ctx->d_tmat, ld, nstore, group, ctx->b, ctx->kkrsz, ctx->npola != ctx->ns,
                        ctx->d_tdiag, ctx->stream));
  // A copy from page-locked memory reads the caller's buffer after cudaMemcpyAsync returns (one
  // from pageable memory is staged before it returns): wait for it, so that the buffer is free
  // when this call returns.
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, tmat_store) == cudaSuccess) {
    if (pa.type == cudaMemoryTypeHost) CK(cudaStreamSynchronize(ctx->stream));
  } else {
    cudaGetLastError();
    CK(cudaStreamSynchronize(ctx->stream));
  }
  ctx->tmat_ld = ld;
  ctx->nstore = nstore;
  ctx->group_size = group;
  return B200TAU_OK;
}

int b200tau_set_atom(b200tau_ctx *ctx, int atom, int num_liz, const double *liz_pos,
                     const int *liz_lmax, const int *liz_store_idx, const double *ubr,
                     const double *ubrd) {
  if (!ctx) return B200TAU_ERR_ARG;
  ctx->kept_valid = false;
  if (atom < 0 || num_liz < 1 || !liz_pos || !liz_lmax || !liz_store_idx)
    return fail(ctx, B200TAU_ERR_ARG, "set_atom: bad arguments");
  if (ctx->ns == 2 && (!ubr || !ubrd))
    return fail(ctx, B200TAU_ERR_ARG, "set_atom: ubr/ubrd required for n_spin_cant = 2");
  for (int i = 0; i < num_liz; ++i)
    if (liz_lmax[i] < 0 || liz_lmax[i] > ctx->lmax || liz_store_idx[i] < 0)
      return fail(ctx, B200TAU_ERR_ARG, "set_atom: site %d has lmax %d / store %d", i, liz_lmax[i],
                  liz_store_idx[i]);
  if (liz_lmax[0] != ctx->lmax)
    return fail(ctx, B200TAU_ERR_ARG, "set_atom: central site lmax %d != maxlmax %d", liz_lmax[0], ctx->lmax);
  CK(cudaSetDevice(ctx->device));
  if ((int)ctx->atoms.size() <= atom) ctx->atoms.resize(atom + 1);
  AtomDev &a = ctx->atoms[atom];
  const int L = num_liz;
  if (L > a.cap_L) {  // a larger LIZ than this record holds: a new device buffer
    CK(cudaStreamSynchronize(ctx->stream));  // solves still queued read the old one
    cudaFree(a.dev);
    a.dev = nullptr;
    a.cap_L = 0;
    CK(cudaMalloc(&a.dev, atom_bytes(L)));
    a.cap_L = L;
  }
  a.valid = false;
  // central site last (see JobDev)
  std::vector<int> perm(L), off(L + 1);
  for (int p = 0; p < L - 1; ++p) perm[p] = p + 1;
  perm[L - 1] = 0;
  off[0] = 0;
  for (int p = 0; p < L; ++p) {
    const int l = liz_lmax[perm[p]];
    off[p + 1] = off[p] + ctx->ns * (l + 1) * (l + 1);
  }
  a.L = L;
  a.N = off[L];
  a.b = ctx->b;
  a.store0 = liz_store_idx[0];
  a.h_store.assign(liz_store_idx, liz_store_idx + L);
  for (int k = 0; k < 4; ++k) {
    a.ubr[k] = ubr ? make_double2(ubr[2 * k], ubr[2 * k + 1]) : make_double2(0, 0);
    a.ubrd[k] = ubrd ? make_double2(ubrd[2 * k], ubrd[2 * k + 1]) : make_double2(0, 0);
  }
  // one host image of the record, one stream-ordered copy (from pageable memory the copy is
  // staged before cudaMemcpyAsync returns, so the image may go out of scope)
  std::vector<unsigned char> img(atom_bytes(L));
  unsigned char *q = img.data();
  std::memcpy(q, liz_pos, sizeof(double) * 3 * L);
  q += sizeof(double) * 3 * L;
  std::memcpy(q, liz_lmax, sizeof(int) * L);
  q += sizeof(int) * L;
  std::memcpy(q, liz_store_idx, sizeof(int) * L);
  q += sizeof(int) * L;
  std::memcpy(q, perm.data(), sizeof(int) * L);
  q += sizeof(int) * L;
  std::memcpy(q, off.data(), sizeof(int) * (L + 1));
  a.pos = reinterpret_cast<double *>(a.dev);
  a.lmax = reinterpret_cast<int *>(a.dev + sizeof(double) * 3 * L);
  a.store = a.lmax + L;
  a.perm = a.store + L;
  a.off = a.perm + L;
  CK(cudaMemcpyAsync(a.dev, img.data(), img.size(), cudaMemcpyHostToDevice, ctx->stream));
  a.valid = true;
  return B200TAU_OK;
}

int b200tau_solve(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs, int prec, double *tau00_l) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (njobs < 0 || (njobs > 0 && (!jobs || !tau00_l)))
    return fail(ctx, B200TAU_ERR_ARG, "solve: bad arguments");
  int rc = check_prec(ctx, prec);
  if (rc) return rc;
  if (njobs == 0) return B200TAU_OK;
  CK(cudaSetDevice(ctx->device));
  const size_t outn = (size_t)njobs * ctx->b * ctx->b;
  if ((rc = ensure_out(ctx, outn))) return rc;
  if ((rc = solve_impl(ctx, jobs, njobs, prec, ctx->d_out))) return rc;
  // outputs, status words and error word behind the waves; one wait
  CK(cudaMemcpyAsync(ctx->h_err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(tau00_l, ctx->d_out, sizeof(double2) * outn, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if ((rc = check_host_err(ctx))) {  // the wait that ran out, not what followed from it
    ctx->info_jobs = 0;
    return rc;
  }
  return check_host_info(ctx);
}

int b200tau_solve_device(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs, int prec,
                         double *tau00_l_dev) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (njobs < 0 || (njobs > 0 && (!jobs || !tau00_l_dev)))
    return fail(ctx, B200TAU_ERR_ARG, "solve_device: bad arguments");
  int rc = check_prec(ctx, prec);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  return solve_impl(ctx, jobs, njobs, prec, reinterpret_cast<double2 *>(tau00_l_dev));
}

int b200tau_sync(b200tau_ctx *ctx) {
  if (!ctx) return B200TAU_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(ctx->h_err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  int rc = check_host_err(ctx);
  if (rc) {
    ctx->info_jobs = 0;
    return rc;
  }
  return check_host_info(ctx);
}

namespace {
struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};
}  // namespace

int b200tau_autotune_paired_steps(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs,
                                  const int *candidates, int ncand, int reps, int *chosen,
                                  float *ms_out) {
  if (!ctx) return B200TAU_ERR_ARG;
  static const int kDefault[] = {0, 512, 768, 1024, 1280, 1536};
  if (!candidates) {
    candidates = kDefault;
    ncand = (int)(sizeof(kDefault) / sizeof(kDefault[0]));
  }
  if (njobs <= 0 || !jobs || ncand < 1 || ncand > 16 || reps < 1 || reps > 16)
    return fail(ctx, B200TAU_ERR_ARG, "autotune: bad arguments");
  for (int c = 0; c < ncand; ++c)
    if (candidates[c] < 0) return fail(ctx, B200TAU_ERR_ARG, "autotune: candidate %d is negative", c);
  int rc = check_prec(ctx, B200TAU_PREC_MIXED);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  const size_t outn = (size_t)njobs * ctx->b * ctx->b;
  if ((rc = ensure_out(ctx, outn))) return rc;
  EventPair ev;
  CK(cudaEventCreate(&ev.a));
  CK(cudaEventCreate(&ev.b));
  int maxN = 0;
  for (int j = 0; j < njobs; ++j)
    if (jobs[j].atom >= 0 && jobs[j].atom < (int)ctx->atoms.size()) maxN = std::max(maxN, ctx->atoms[jobs[j].atom].N);
  const int incumbent = pair_min_rest_for(ctx, maxN);
  float incumbent_ms = -1.0f;
  struct TrialReset {
    b200tau_ctx *c;
    ~TrialReset() { c->pair_trial = -1; }
  } trial_reset{ctx};
  int best = -1;
  float best_ms = 0.0f;
  for (int c = 0; c < ncand; ++c) {
    ctx->pair_trial = candidates[c];
    float cand_ms = 0.0f;
    // one untimed solve (a new threshold is a new wave graph: its capture is not timed), then the
    // fastest of `reps` timed ones
    for (int r = 0; r <= reps; ++r) {
      CK(cudaEventRecord(ev.a, ctx->stream));
      rc = solve_impl(ctx, jobs, njobs, B200TAU_PREC_MIXED, ctx->d_out);
      if (!rc) {
        const cudaError_t e = cudaEventRecord(ev.b, ctx->stream);
        if (e != cudaSuccess) rc = fail(ctx, B200TAU_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
      }
      if (!rc) rc = b200tau_sync(ctx);
      if (rc) return rc;
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, ev.a, ev.b));
      if (r > 0 && (r == 1 || ms < cand_ms)) cand_ms = ms;
    }
    if (ms_out) ms_out[c] = cand_ms;
    if (candidates[c] == incumbent) incumbent_ms = cand_ms;
    if (c == 0 || cand_ms < best_ms) {
      best_ms = cand_ms;
      best = candidates[c];
    }
  }
  ctx->pair_trial = -1;
  // run-to-run noise of a solve is a few per cent: the setting in force stays unless beaten by 2%
  if (incumbent_ms >= 0.0f && best_ms > 0.98f * incumbent_ms) best = incumbent;
  const int bucket = round_up(maxN, 64);
  bool found = false;
  for (auto &e : ctx->pair_table)
    if (e.first == bucket) {
      e.second = best;
      found = true;
    }
  if (!found) ctx->pair_table.emplace_back(bucket, best);
  if (chosen) *chosen = best;
  return B200TAU_OK;
}

int b200tau_solve_dense(b200tau_ctx *ctx, const double *m, int n, int ldm, const double *t0, int b,
                        int prec, double *tau00) {
  if (!ctx) return B200TAU_ERR_ARG;
  ctx->kept_valid = false;
  if (!m || !t0 || !tau00 || n < 1 || b < 1 || b > n || b > kMaxB || ldm < n)
    return fail(ctx, B200TAU_ERR_ARG, "solve_dense: bad arguments (n %d, b %d, ldm %d)", n, b, ldm);
  int rc = check_prec(ctx, prec);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  const Plan p = plan_for(ctx, prec);
  const int ld = round_up(n, 64);
  if ((rc = ensure_workspace(ctx, ld, std::max(1, ctx->slots), p))) return rc;
  if ((rc = ensure_jobs(ctx, 1))) return rc;
  if ((rc = ensure_out(ctx, (size_t)b * b))) return rc;
  if (!ctx->d_t0) CK(cudaMalloc(&ctx->d_t0, sizeof(double2) * kMaxB * kMaxB));
  JobDev J;
  std::memset(&J, 0, sizeof(J));
  fill_slot(ctx, J, 0, ld, p);
  const int r = n - b;  // reorder: central block (first b) goes last
  double2 *W = J.M;
  const size_t es = sizeof(double2);
  const double2 *hm = reinterpret_cast<const double2 *>(m);
  // [Mrr Mr0; M0r M00] <- [M00 M0r; Mr0 Mrr]
  if (r > 0) {
    CK(cudaMemcpy2DAsync(W, ld * es, hm + b + (size_t)b * ldm, ldm * es, r * es, r, cudaMemcpyHostToDevice,
                         ctx->stream));
    CK(cudaMemcpy2DAsync(W + (size_t)r * ld, ld * es, hm + b, ldm * es, r * es, b, cudaMemcpyHostToDevice,
                         ctx->stream));
    CK(cudaMemcpy2DAsync(W + r, ld * es, hm + (size_t)b * ldm, ldm * es, b * es, r, cudaMemcpyHostToDevice,
                         ctx->stream));
  }
  CK(cudaMemcpy2DAsync(W + r + (size_t)r * ld, ld * es, hm, ldm * es, b * es, b, cudaMemcpyHostToDevice,
                       ctx->stream));
  if (p.f_separate) CK(launch_copy_to_factor(p.fk, W, J.F, n, ld, ctx->stream));
  CK(cudaMemcpyAsync(ctx->d_t0, t0, es * b * b, cudaMemcpyHostToDevice, ctx->stream));
  J.N = n;
  J.n = r;
  J.b = b;
  J.t0 = ctx->d_t0;
  J.t0_ld = b;
  J.out = ctx->d_out;
  J.out_mode = 1;
  const bool panel = use_panel(ctx, n, p.fk);
  if (panel) {
    if ((rc = ensure_piv(ctx, ld, 1))) return rc;
    J.piv = slot_piv(ctx, 0);
  }
  CK(cudaMemcpyAsync(ctx->d_jobs, &J, sizeof(J), cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = reset_slot_status(ctx, 1))) return rc;
  ctx->launches = 0;
  if ((rc = run_pipeline(ctx, std::vector<JobDev>{J}, 1, r, n, ld, 1, b, b, p, panel))) return rc;
  int info = 0;
  CK(cudaMemcpyAsync(&info, ctx->d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(tau00, ctx->d_out, es * b * b, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (info) return fail(ctx, B200TAU_ERR_SINGULAR, "solve_dense: singular pivot (info %d)", info);
  return B200TAU_OK;
}

int b200tau_solve_vjp(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs, const double *taubar,
                      double *tau00, double *tbar, double *dlogdet) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (njobs < 0 || (njobs > 0 && (!jobs || !taubar || !tbar)))
    return fail(ctx, B200TAU_ERR_ARG, "solve_vjp: bad arguments");
  if (njobs == 0) return B200TAU_OK;
  CK(cudaSetDevice(ctx->device));
  int rc = validate_jobs(ctx, jobs, njobs);
  if (rc) return rc;
  Plan p = plan_for(ctx, B200TAU_PREC_FP64);
  p.steps = std::max(p.steps, 1);  // X refined against M before the adjoint uses it
  p.f_separate = true;
  std::vector<int> order(njobs);
  for (int j = 0; j < njobs; ++j) order[j] = j;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return ctx->atoms[jobs[a].atom].N > ctx->atoms[jobs[b].atom].N;
  });
  const int maxN = ctx->atoms[jobs[order[0]].atom].N;
  const int ld = round_up(maxN, 64);
  const size_t v_need = (size_t)ld * ld;
  // the factors kept by a forward FP64 solve of these jobs (b200tau_set_keep_factors), used once
  const bool reuse = kept_matches(ctx, jobs, njobs) && ctx->kept_ld == ld && ctx->kept_order == order;
  ctx->kept_valid = false;
  const int slots = reuse ? njobs : choose_slots(ctx, ld, njobs, p, v_need * sizeof(double2));
  if ((rc = ensure_workspace(ctx, ld, slots, p))) return rc;
  if ((rc = ensure_jobs(ctx, slots))) return rc;
  if ((rc = ensure_v(ctx, ld, slots))) return rc;
  // output blocks: job j's sites start at block site_off[j] (caller's job order)
  std::vector<long> site_off(njobs + 1, 0);
  for (int j = 0; j < njobs; ++j) site_off[j + 1] = site_off[j] + ctx->atoms[jobs[j].atom].L;
  const size_t bb = (size_t)ctx->b * ctx->b;
  const size_t nblk = (size_t)site_off[njobs];
  const size_t need = bb * (njobs + nblk * (dlogdet ? 2 : 1));
  if (need > ctx->adj_cap) {
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->d_adj);
    ctx->d_adj = nullptr;
    CK(cudaMalloc(&ctx->d_adj, sizeof(double2) * need));
    ctx->adj_cap = need;
  }
  AdjointBufs adj;
  adj.taubar = ctx->d_adj;
  adj.tbar = ctx->d_adj + bb * njobs;
  adj.dlogdet = dlogdet ? adj.tbar + bb * nblk : nullptr;
  adj.site_off = site_off.data();
  if ((rc = ensure_out(ctx, bb * njobs))) return rc;
  CK(cudaMemcpyAsync(ctx->d_adj, taubar, sizeof(double2) * bb * njobs, cudaMemcpyHostToDevice, ctx->stream));
  ctx->launches = 0;
  std::vector<int> info(slots);
  for (int w0 = 0; w0 < njobs; w0 += slots) {
    const int nw = std::min(slots, njobs - w0);
    if ((rc = run_wave(ctx, jobs, &order[w0], nw, ld, p, ctx->d_out, &adj, reuse))) return rc;
    CK(cudaMemcpyAsync(info.data(), ctx->d_info, sizeof(int) * nw, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if ((rc = check_info(ctx, info.data(), &order[w0], nw))) return rc;
  }
  if (tau00)
    CK(cudaMemcpyAsync(tau00, ctx->d_out, sizeof(double2) * bb * njobs, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(tbar, adj.tbar, sizeof(double2) * bb * nblk, cudaMemcpyDeviceToHost, ctx->stream));
  if (dlogdet)
    CK(cudaMemcpyAsync(dlogdet, adj.dlogdet, sizeof(double2) * bb * nblk, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return check_err_flags(ctx);
}

int b200tau_solve_tau_full(b200tau_ctx *ctx, const b200tau_job *job, double *tau_full, int n) {
  if (!ctx) return B200TAU_ERR_ARG;
  ctx->kept_valid = false;
  if (!job || !tau_full) return fail(ctx, B200TAU_ERR_ARG, "solve_tau_full: bad arguments");
  int rc = validate_jobs(ctx, job, 1);
  if (rc) return rc;
  const AtomDev &a = ctx->atoms[job->atom];
  if (n != a.N) return fail(ctx, B200TAU_ERR_ARG, "solve_tau_full: n %d != N %d", n, a.N);
  CK(cudaSetDevice(ctx->device));
  const int ld = round_up(a.N, 64);
  Plan p;  // FP64 factors in M's own storage; M^-1 from them (no right-hand side to refine)
  p.fk = kFactorFP64;
  p.steps = 0;
  p.f_separate = false;
  if ((rc = ensure_workspace(ctx, ld, std::max(1, ctx->slots), p))) return rc;
  if ((rc = ensure_jobs(ctx, 1))) return rc;
  if ((rc = ensure_v(ctx, ld, 1))) return rc;
  const bool panel = use_panel(ctx, a.N, kFactorFP64);
  if (panel && (rc = ensure_piv(ctx, ld, 1))) return rc;
  JobDev J;
  std::memset(&J, 0, sizeof(J));
  J.energy = make_double2(job->energy[0], job->energy[1]);
  J.prel = make_double2(job->prel[0], job->prel[1]);
  J.pos = a.pos;
  J.lmax = a.lmax;
  J.store = a.store;
  J.perm = a.perm;
  J.off = a.off;
  fill_slot(ctx, J, 0, ld, p);
  J.conv = nullptr;
  J.cnorm = nullptr;
  J.V = ctx->d_V;
  if (panel) J.piv = slot_piv(ctx, 0);
  J.L = a.L;
  J.N = a.N;
  J.b = a.b;
  J.n = a.N - a.b;
  J.iie = job->iie;
  J.ispin = job->ispin;
  CK(cudaMemcpyAsync(ctx->d_jobs, &J, sizeof(J), cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = reset_slot_status(ctx, 1))) return rc;
  ctx->launches = 0;
  CK(launch_kkr_build(ctx->d_jobs, 1, a.L, build_params(ctx, p), ctx->d_err, ctx->stream, &ctx->launches));
  CK(launch_eliminate(kFactorFP64, ctx->d_jobs, 1, J.n, J.N, ctx->d_info, ctx->stream, &ctx->launches, nullptr,
                      nullptr, ctx->d_err, false, nullptr, panel));
  CK(launch_inverse(ctx->d_jobs, 1, J.n, J.N, ctx->stream, &ctx->launches));
  CK(launch_tau_full(ctx->d_jobs, 1, a.L, a.N, tmat_view(ctx), ctx->stream, &ctx->launches));
  // reference site order (central site first): rows/cols [0, r) <-> [b, N), [r, N) <-> [0, b)
  const int r = a.N - a.b, b = a.b;
  const size_t es = sizeof(double2);
  double2 *hm = reinterpret_cast<double2 *>(tau_full);
  const double2 *W = J.M;
  if (r > 0) {
    CK(cudaMemcpy2DAsync(hm + b + (size_t)b * n, n * es, W, ld * es, r * es, r, cudaMemcpyDeviceToHost,
                         ctx->stream));
    CK(cudaMemcpy2DAsync(hm + b, n * es, W + (size_t)r * ld, ld * es, r * es, b, cudaMemcpyDeviceToHost,
                         ctx->stream));
    CK(cudaMemcpy2DAsync(hm + (size_t)b * n, n * es, W + r, ld * es, b * es, r, cudaMemcpyDeviceToHost,
                         ctx->stream));
  }
  CK(cudaMemcpy2DAsync(hm, n * es, W + r + (size_t)r * ld, ld * es, b * es, b, cudaMemcpyDeviceToHost,
                       ctx->stream));
  int info = 0;
  CK(cudaMemcpyAsync(&info, ctx->d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(ctx->h_err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if ((rc = check_host_err(ctx))) return rc;
  if (info) return fail(ctx, B200TAU_ERR_SINGULAR, "solve_tau_full: singular pivot (info %d)", info);
  return B200TAU_OK;
}

int b200tau_build_kkr(b200tau_ctx *ctx, const b200tau_job *job, double *m_out, int n) {
  if (!ctx) return B200TAU_ERR_ARG;
  ctx->kept_valid = false;
  if (!job || !m_out) return fail(ctx, B200TAU_ERR_ARG, "build_kkr: bad arguments");
  int rc = validate_jobs(ctx, job, 1);
  if (rc) return rc;
  const AtomDev &a = ctx->atoms[job->atom];
  if (n != a.N) return fail(ctx, B200TAU_ERR_ARG, "build_kkr: n %d != N %d", n, a.N);
  CK(cudaSetDevice(ctx->device));
  const int ld = round_up(a.N, 64);
  Plan p;
  p.fk = kFactorFP64;
  p.steps = 0;
  p.f_separate = false;
  if ((rc = ensure_workspace(ctx, ld, std::max(1, ctx->slots), p))) return rc;
  if ((rc = ensure_jobs(ctx, 1))) return rc;
  JobDev J;
  std::memset(&J, 0, sizeof(J));
  J.energy = make_double2(job->energy[0], job->energy[1]);
  J.prel = make_double2(job->prel[0], job->prel[1]);
  J.pos = a.pos;
  J.lmax = a.lmax;
  J.store = a.store;
  J.perm = a.perm;
  J.off = a.off;
  fill_slot(ctx, J, 0, ld, p);
  J.L = a.L;
  J.N = a.N;
  J.b = a.b;
  J.n = a.N - a.b;
  J.iie = job->iie;
  J.ispin = job->ispin;
  CK(cudaMemcpyAsync(ctx->d_jobs, &J, sizeof(J), cudaMemcpyHostToDevice, ctx->stream));
  ctx->launches = 0;
  CK(launch_kkr_build(ctx->d_jobs, 1, a.L, build_params(ctx, p), ctx->d_err, ctx->stream, &ctx->launches));
  // undo the central-site-last order: rows/cols [0, r) <-> [b, N), [r, N) <-> [0, b)
  const int r = a.N - a.b, b = a.b;
  const size_t es = sizeof(double2);
  double2 *hm = reinterpret_cast<double2 *>(m_out);
  const double2 *W = J.M;
  if (r > 0) {
    CK(cudaMemcpy2DAsync(hm + b + (size_t)b * n, n * es, W, ld * es, r * es, r, cudaMemcpyDeviceToHost,
                         ctx->stream));
    CK(cudaMemcpy2DAsync(hm + b, n * es, W + (size_t)r * ld, ld * es, r * es, b, cudaMemcpyDeviceToHost,
                         ctx->stream));
    CK(cudaMemcpy2DAsync(hm + (size_t)b * n, n * es, W + r, ld * es, b * es, r, cudaMemcpyDeviceToHost,
                         ctx->stream));
  }
  CK(cudaMemcpy2DAsync(hm, n * es, W + r + (size_t)r * ld, ld * es, b * es, b, cudaMemcpyDeviceToHost,
                       ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return check_err_flags(ctx);
}

}  // extern "C"
