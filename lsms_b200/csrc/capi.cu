// C ABI of b200tau (include/b200tau.h): context, uploads and the batched solve driver.
//
// The context replaces the reference's per-thread DeviceStorage (src/Accelerator/
// DeviceStorage.hpp:55-144, DeviceStorage.cu:87-225) and DeviceAtom/DeviceConstants
// (DeviceStorage.cu:341-404): it owns the device tmatStore copy, one device record per atom,
// the angular tables, a stream, and a workspace of `slots` KKR matrices.  A solve call packs
// the jobs into waves of at most `slots` jobs (largest N first), and per wave runs
//   kkr_build -> FP64 block elimination (or the mixed-precision path) -> finalize
// on the context stream, then copies the tau00_l blocks out.

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

}  // namespace

struct b200tau_ctx {
  int device = 0;
  int lmax = 3, ns = 1, npola = 1, kkrsz = 16, b = 16, blk = 1024;
  cudaStream_t stream = nullptr;
  std::string err;
  AngularTables *d_tables = nullptr;
  double2 *d_tmat = nullptr;
  long tmat_ld = 0;
  int nstore = 0;
  int group_size = 0;
  std::vector<AtomDev> atoms;
  // workspace
  double2 *d_work = nullptr;
  size_t work_elems = 0;   // per slot
  int slots = 0;
  JobDev *d_jobs = nullptr;
  int jobs_cap = 0;
  int *d_info = nullptr;   // per slot
  int *d_err = nullptr;    // device error flags
  double2 *d_out = nullptr;
  size_t out_cap = 0;
  double2 *d_t0 = nullptr;  // dense-solve t0
  long launches = 0;
  int max_slots = 64;
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
  cudaFree(a.pos);
  cudaFree(a.lmax);
  cudaFree(a.store);
  cudaFree(a.perm);
  cudaFree(a.off);
  a = AtomDev();
}

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// Workspace: `slots` matrices of ld x ld complex, ld a multiple of 64.
int ensure_workspace(b200tau_ctx *ctx, int ld, int slots) {
  const size_t need = (size_t)ld * ld;
  if (ctx->d_work && need <= ctx->work_elems && slots <= ctx->slots) return B200TAU_OK;
  cudaFree(ctx->d_work);
  ctx->d_work = nullptr;
  cudaFree(ctx->d_info);
  ctx->d_info = nullptr;
  CK(cudaMalloc(&ctx->d_work, need * slots * sizeof(double2)));
  CK(cudaMalloc(&ctx->d_info, sizeof(int) * slots));
  ctx->work_elems = need;
  ctx->slots = slots;
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

int choose_slots(b200tau_ctx *ctx, int ld, int njobs) {
  size_t freeb = 0, totalb = 0;
  if (cudaMemGetInfo(&freeb, &totalb) != cudaSuccess) freeb = (size_t)8 << 30;
  const size_t per = (size_t)ld * ld * sizeof(double2);
  size_t budget = freeb / 2;
  int s = (int)std::max<size_t>(1, budget / std::max<size_t>(per, 1));
  s = std::min(s, ctx->max_slots);
  s = std::min(s, njobs);
  return std::max(s, 1);
}

// Validate jobs, build the JobDev records for one wave and run the device pipeline.
int run_wave(b200tau_ctx *ctx, const b200tau_job *jobs, const int *idx, int nw, int ld,
             int prec, double2 *out_base) {
  std::vector<JobDev> h(nw);
  int maxL = 0, maxN = 0, maxn = 0;
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
    J.M = ctx->d_work + (size_t)w * ctx->work_elems;
    J.L = a.L;
    J.N = a.N;
    J.b = a.b;
    J.n = a.N - a.b;
    J.ld = ld;
    J.iie = jb.iie;
    J.ispin = jb.ispin;
    const long jsm = (ctx->npola != ctx->ns) ? (long)ctx->kkrsz * ctx->kkrsz * jb.ispin : 0;
    J.t0 = ctx->d_tmat + (long)a.store0 * ctx->tmat_ld + (long)jb.iie * ctx->blk + jsm;
    J.t0_ld = ctx->b;
    J.out = out_base + (size_t)idx[w] * ctx->b * ctx->b;
    J.out_mode = 0;
    for (int k = 0; k < 4; ++k) {
      J.ubr[k] = a.ubr[k];
      J.ubrd[k] = a.ubrd[k];
    }
    maxL = std::max(maxL, a.L);
    maxN = std::max(maxN, a.N);
    maxn = std::max(maxn, a.N - a.b);
  }
  CK(cudaMemcpyAsync(ctx->d_jobs, h.data(), sizeof(JobDev) * nw, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_info, 0, sizeof(int) * nw, ctx->stream));
  BuildParams bp;
  bp.tables = ctx->d_tables;
  bp.tmat = ctx->d_tmat;
  bp.tmat_ld = ctx->tmat_ld;
  bp.blk = ctx->blk;
  bp.kkrsz = ctx->kkrsz;
  bp.ns = ctx->ns;
  bp.npola = ctx->npola;
  CK(launch_kkr_build(ctx->d_jobs, nw, maxL, bp, ctx->d_err, ctx->stream));
  ctx->launches += 1;
  (void)prec;
  CK(launch_lu_fp64(ctx->d_jobs, nw, maxn, maxN, 64, ctx->d_info, ctx->stream, &ctx->launches));
  CK(launch_finalize(ctx->d_jobs, nw, ctx->ns, ctx->kkrsz, ctx->d_info, ctx->stream));
  ctx->launches += 1;
  return B200TAU_OK;
}

int check_info(b200tau_ctx *ctx, const std::vector<int> &info, const int *idx, int nw) {
  for (int w = 0; w < nw; ++w)
    if (info[w] != 0)
      return fail(ctx, B200TAU_ERR_SINGULAR,
                  info[w] > 0 ? "job %d: singular diagonal block at column %d"
                              : "job %d: 1 - Delta is singular",
                  idx[w], info[w] > 0 ? info[w] - 1 : 0);
  return B200TAU_OK;
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
    const AtomDev &a = ctx->atoms[jb.atom];
    for (int s : a.h_store)
      if (s < 0 || s >= ctx->nstore)
        return fail(ctx, B200TAU_ERR_ARG, "atom %d: store index %d outside tmatStore (%d)", jb.atom,
                    s, ctx->nstore);
  }
  return B200TAU_OK;
}

int solve_impl(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs, int prec, double2 *dev_out,
               bool sync_and_check) {
  if (njobs == 0) return B200TAU_OK;
  int rc = validate_jobs(ctx, jobs, njobs);
  if (rc) return rc;
  std::vector<int> order(njobs);
  for (int j = 0; j < njobs; ++j) order[j] = j;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return ctx->atoms[jobs[a].atom].N > ctx->atoms[jobs[b].atom].N;
  });
  const int maxN = ctx->atoms[jobs[order[0]].atom].N;
  const int ld = round_up(maxN, 64);
  const int slots = choose_slots(ctx, ld, njobs);
  if ((rc = ensure_workspace(ctx, ld, slots))) return rc;
  if ((rc = ensure_jobs(ctx, slots))) return rc;
  ctx->launches = 0;
  std::vector<int> info(slots);
  for (int w0 = 0; w0 < njobs; w0 += slots) {
    const int nw = std::min(slots, njobs - w0);
    if ((rc = run_wave(ctx, jobs, &order[w0], nw, ld, prec, dev_out))) return rc;
    if (sync_and_check || w0 + nw < njobs) {
      CK(cudaMemcpyAsync(info.data(), ctx->d_info, sizeof(int) * nw, cudaMemcpyDeviceToHost,
                         ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      if ((rc = check_info(ctx, info, &order[w0], nw))) return rc;
    }
  }
  return B200TAU_OK;
}

int check_err_flags(b200tau_ctx *ctx) {
  int flags = 0;
  CK(cudaMemcpy(&flags, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flags) {
    cudaMemset(ctx->d_err, 0, sizeof(int));
    return fail(ctx, B200TAU_ERR_TIMEOUT, "a device-side wait exceeded its bound (flags %d)", flags);
  }
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
  AngularTables tab;
  if (build_angular_tables(lmax, &tab)) e = cudaErrorInvalidValue;
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_tables, sizeof(AngularTables));
  if (e == cudaSuccess) e = cudaMemcpy(ctx->d_tables, &tab, sizeof(tab), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_err, 0, sizeof(int));
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
  for (auto &a : ctx->atoms) free_atom(a);
  cudaFree(ctx->d_tables);
  cudaFree(ctx->d_tmat);
  cudaFree(ctx->d_work);
  cudaFree(ctx->d_jobs);
  cudaFree(ctx->d_info);
  cudaFree(ctx->d_err);
  cudaFree(ctx->d_out);
  cudaFree(ctx->d_t0);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char *b200tau_last_error(const b200tau_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void *b200tau_stream(b200tau_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

long b200tau_last_launch_count(const b200tau_ctx *ctx) { return ctx ? ctx->launches : 0; }

int b200tau_gaunt_numbers(int lmax, double *cgnt) {
  if (lmax < 0 || lmax > kMaxLmax || !cgnt) return B200TAU_ERR_ARG;
  gaunt_numbers(lmax, cgnt);
  return B200TAU_OK;
}

int b200tau_upload_tmat(b200tau_ctx *ctx, const double *tmat_store, long ld, int nstore, int blk_size) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (!tmat_store || nstore <= 0 || blk_size != ctx->blk || ld < blk_size || ld % blk_size)
    return fail(ctx, B200TAU_ERR_ARG, "upload_tmat: bad arguments (ld %ld, nstore %d, blk %d, expected blk %d)",
                ld, nstore, blk_size, ctx->blk);
  CK(cudaSetDevice(ctx->device));
  const size_t bytes = sizeof(double2) * (size_t)ld * nstore;
  if (!ctx->d_tmat || (size_t)ctx->tmat_ld * ctx->nstore < (size_t)ld * nstore) {
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->d_tmat);
    ctx->d_tmat = nullptr;
    CK(cudaMalloc(&ctx->d_tmat, bytes));
  }
  CK(cudaMemcpyAsync(ctx->d_tmat, tmat_store, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->tmat_ld = ld;
  ctx->nstore = nstore;
  ctx->group_size = (int)(ld / blk_size);
  return B200TAU_OK;
}

int b200tau_set_atom(b200tau_ctx *ctx, int atom, int num_liz, const double *liz_pos,
                     const int *liz_lmax, const int *liz_store_idx, const double *ubr,
                     const double *ubrd) {
  if (!ctx) return B200TAU_ERR_ARG;
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
  CK(cudaStreamSynchronize(ctx->stream));
  free_atom(a);
  const int L = num_liz;
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
  CK(cudaMalloc(&a.pos, sizeof(double) * 3 * L));
  CK(cudaMalloc(&a.lmax, sizeof(int) * L));
  CK(cudaMalloc(&a.store, sizeof(int) * L));
  CK(cudaMalloc(&a.perm, sizeof(int) * L));
  CK(cudaMalloc(&a.off, sizeof(int) * (L + 1)));
  CK(cudaMemcpy(a.pos, liz_pos, sizeof(double) * 3 * L, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(a.lmax, liz_lmax, sizeof(int) * L, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(a.store, liz_store_idx, sizeof(int) * L, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(a.perm, perm.data(), sizeof(int) * L, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(a.off, off.data(), sizeof(int) * (L + 1), cudaMemcpyHostToDevice));
  a.valid = true;
  return B200TAU_OK;
}

int b200tau_solve(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs, int prec, double *tau00_l) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (njobs < 0 || (njobs > 0 && (!jobs || !tau00_l)))
    return fail(ctx, B200TAU_ERR_ARG, "solve: bad arguments");
  if (prec != B200TAU_PREC_FP64 && prec != B200TAU_PREC_MIXED)
    return fail(ctx, B200TAU_ERR_ARG, "solve: unknown precision %d", prec);
  if (njobs == 0) return B200TAU_OK;
  CK(cudaSetDevice(ctx->device));
  const size_t outn = (size_t)njobs * ctx->b * ctx->b;
  int rc = ensure_out(ctx, outn);
  if (rc) return rc;
  rc = solve_impl(ctx, jobs, njobs, prec, ctx->d_out, true);
  if (rc) return rc;
  CK(cudaMemcpyAsync(tau00_l, ctx->d_out, sizeof(double2) * outn, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return check_err_flags(ctx);
}

int b200tau_solve_device(b200tau_ctx *ctx, const b200tau_job *jobs, int njobs, int prec,
                         double *tau00_l_dev) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (njobs < 0 || (njobs > 0 && (!jobs || !tau00_l_dev)))
    return fail(ctx, B200TAU_ERR_ARG, "solve_device: bad arguments");
  if (prec != B200TAU_PREC_FP64 && prec != B200TAU_PREC_MIXED)
    return fail(ctx, B200TAU_ERR_ARG, "solve_device: unknown precision %d", prec);
  CK(cudaSetDevice(ctx->device));
  return solve_impl(ctx, jobs, njobs, prec, reinterpret_cast<double2 *>(tau00_l_dev), false);
}

int b200tau_sync(b200tau_ctx *ctx) {
  if (!ctx) return B200TAU_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  std::vector<int> info(std::max(ctx->slots, 1));
  if (ctx->d_info && ctx->slots > 0) {
    CK(cudaMemcpy(info.data(), ctx->d_info, sizeof(int) * ctx->slots, cudaMemcpyDeviceToHost));
    for (int w = 0; w < ctx->slots; ++w)
      if (info[w] != 0) {
        cudaMemset(ctx->d_info, 0, sizeof(int) * ctx->slots);
        return fail(ctx, B200TAU_ERR_SINGULAR, "a job of the last wave hit a singular pivot");
      }
  }
  return check_err_flags(ctx);
}

int b200tau_solve_dense(b200tau_ctx *ctx, const double *m, int n, int ldm, const double *t0, int b,
                        int prec, double *tau00) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (!m || !t0 || !tau00 || n < 1 || b < 1 || b > n || b > kMaxB || ldm < n)
    return fail(ctx, B200TAU_ERR_ARG, "solve_dense: bad arguments (n %d, b %d, ldm %d)", n, b, ldm);
  if (prec != B200TAU_PREC_FP64 && prec != B200TAU_PREC_MIXED)
    return fail(ctx, B200TAU_ERR_ARG, "solve_dense: unknown precision %d", prec);
  CK(cudaSetDevice(ctx->device));
  const int ld = round_up(n, 64);
  int rc = ensure_workspace(ctx, ld, std::max(1, ctx->slots));
  if (rc) return rc;
  if ((rc = ensure_jobs(ctx, 1))) return rc;
  if ((rc = ensure_out(ctx, (size_t)b * b))) return rc;
  if (!ctx->d_t0) CK(cudaMalloc(&ctx->d_t0, sizeof(double2) * kMaxB * kMaxB));
  const int r = n - b;  // reorder: central block (first b) goes last
  double2 *W = ctx->d_work;
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
  CK(cudaMemcpyAsync(ctx->d_t0, t0, es * b * b, cudaMemcpyHostToDevice, ctx->stream));
  JobDev J;
  std::memset(&J, 0, sizeof(J));
  J.M = W;
  J.N = n;
  J.n = r;
  J.b = b;
  J.ld = ld;
  J.t0 = ctx->d_t0;
  J.t0_ld = b;
  J.out = ctx->d_out;
  J.out_mode = 1;
  CK(cudaMemcpyAsync(ctx->d_jobs, &J, sizeof(J), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_info, 0, sizeof(int), ctx->stream));
  ctx->launches = 0;
  (void)prec;
  CK(launch_lu_fp64(ctx->d_jobs, 1, r, n, 64, ctx->d_info, ctx->stream, &ctx->launches));
  CK(launch_finalize(ctx->d_jobs, 1, 1, b, ctx->d_info, ctx->stream));
  ctx->launches += 1;
  int info = 0;
  CK(cudaMemcpyAsync(&info, ctx->d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(tau00, ctx->d_out, es * b * b, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (info) return fail(ctx, B200TAU_ERR_SINGULAR, "solve_dense: singular pivot (info %d)", info);
  return B200TAU_OK;
}

int b200tau_build_kkr(b200tau_ctx *ctx, const b200tau_job *job, double *m_out, int n) {
  if (!ctx) return B200TAU_ERR_ARG;
  if (!job || !m_out) return fail(ctx, B200TAU_ERR_ARG, "build_kkr: bad arguments");
  int rc = validate_jobs(ctx, job, 1);
  if (rc) return rc;
  const AtomDev &a = ctx->atoms[job->atom];
  if (n != a.N) return fail(ctx, B200TAU_ERR_ARG, "build_kkr: n %d != N %d", n, a.N);
  CK(cudaSetDevice(ctx->device));
  const int ld = round_up(a.N, 64);
  if ((rc = ensure_workspace(ctx, ld, std::max(1, ctx->slots)))) return rc;
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
  J.M = ctx->d_work;
  J.L = a.L;
  J.N = a.N;
  J.b = a.b;
  J.n = a.N - a.b;
  J.ld = ld;
  J.iie = job->iie;
  J.ispin = job->ispin;
  CK(cudaMemcpyAsync(ctx->d_jobs, &J, sizeof(J), cudaMemcpyHostToDevice, ctx->stream));
  BuildParams bp;
  bp.tables = ctx->d_tables;
  bp.tmat = ctx->d_tmat;
  bp.tmat_ld = ctx->tmat_ld;
  bp.blk = ctx->blk;
  bp.kkrsz = ctx->kkrsz;
  bp.ns = ctx->ns;
  bp.npola = ctx->npola;
  CK(launch_kkr_build(ctx->d_jobs, 1, a.L, bp, ctx->d_err, ctx->stream));
  // undo the central-site-last order: rows/cols [0, r) <-> [b, N), [r, N) <-> [0, b)
  const int r = a.N - a.b, b = a.b;
  const size_t es = sizeof(double2);
  double2 *hm = reinterpret_cast<double2 *>(m_out);
  const double2 *W = ctx->d_work;
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
