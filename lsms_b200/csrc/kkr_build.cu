// KKR matrix build M = 1 - t G0 on the device (FP64).
//
// Restates, for one (atom, energy, spin) job per grid row:
//   buildBGijCPU            src/MultipleScattering/buildKKRMatrix_CPU.cpp:96-176
//     (Hankel :23-40, sin/cos powers :42-59, D_lm :127-140, Gaunt sum :148-176),
//   setBGijCPU / setgij     buildKKRMatrix_CPU.cpp:61-94, setgij.f:29-38 (spin-diagonal G),
//   M_ij = -t_i G_ij        buildKKRMatrix_CPU.cpp:388-412, calculateTauMatrix.cpp:156-183,240-242
//                           (t gathered with the F77 build's per-site lmax semantics).
// The reference's CUDA build (buildGijCudaKernel, buildKKRMatrix_CUDA.cu:215-381) runs one CTA
// per site pair with a serial thread-0 prologue and global read-modify-writes of a second N x N
// matrix.  Here one CTA owns one block column of M (one LIZ site j) for one job: the angular
// gather tables arrive in shared memory by one bulk-async (TMA) copy, each warp builds whole
// -t_i G_ij blocks for a row site i with G held in shared memory, and every store writes
// contiguous 256-byte column segments of M.  No N x N scratch is written besides M itself.
//
// Site order in M: LIZ sites 1..L-1 then the central site 0 (JobDev::perm), so the
// elimination leaves 1 - Delta in the trailing block.

#include <cuda_runtime.h>

#include "common.cuh"

namespace b200 {
namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;

// Per-pair prologue values, one column per pair of the current chunk of row sites: hfn_l (re, im),
// normalised P_lm, cos(m phi), sin(m phi).
constexpr int kProH = 0;                          // 2 (kMaxLend + 1) doubles
constexpr int kProP = kProH + 2 * (kMaxLend + 1);  // kNdlm
constexpr int kProC = kProP + kNdlm;               // kMaxLend + 1
constexpr int kProS = kProC + kMaxLend + 1;        // kMaxLend + 1
constexpr int kProN = kProS + kMaxLend + 1;

constexpr int kChunk = 96;  // row-site pairs per prologue pass of a CTA (two CTAs fit an SM)

struct BuildSmem {
  AngularTables tab;
  double2 D[kWarps][kNdlj];
  double2 G[kWarps][kMaxKK * kMaxKK];  // staged only for a non-diagonal t
  double pro[kProN][kChunk];
  // lmax-3 blocks: gather record of element it of lane L (lm1 = L / 16 + 2 it, lm2 = L % 16):
  // coefficients with the sign of i^rot folded in (negated for rot 2, 3), and the packed D
  // indices (6 bits each) plus the swap flag of an odd rot in bit 24
  double2 gc01[8][32], gc23[8][32];
  unsigned gd[8][32];
  unsigned long long bar;
};
static_assert(sizeof(BuildSmem) <= 113 * 1024, "two build CTAs per SM");

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {  // c + a*b
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(a.y, b.x, c.y);
  return c;
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

// e / kk for the block sizes (l + 1)^2, l <= 3, with constant divisors.
__device__ __forceinline__ int div_kk(int e, int kk) {
  switch (kk) {
    case 16: return e >> 4;
    case 9: return e / 9;
    case 4: return e >> 2;
    default: return e;
  }
}

__device__ __forceinline__ bool table_copy_done(unsigned bar) {
  unsigned done;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
      : "=r"(done)
      : "r"(bar)
      : "memory");
  return done != 0;
}

// Stage the angular tables with one bulk copy (cp.async.bulk, completion on an mbarrier).
// The wait is bounded by `polls` (BuildParams::table_polls); the outcome is made uniform over the
// CTA, and on expiry the CTA records an error and keeps waiting (bounded again, far longer) so
// that it never exits with a copy into its shared memory still in flight.
__device__ bool stage_tables(BuildSmem &sm, const AngularTables *src, int *err, long polls) {
  const unsigned bar = smem_u32(&sm.bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                 "r"((unsigned)sizeof(AngularTables))
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(&sm.tab)),
        "l"(src), "r"((unsigned)sizeof(AngularTables)), "r"(bar)
        : "memory");
  }
  __syncthreads();
  bool ok = false;
  for (long it = 0; it < polls; ++it)
    if (table_copy_done(bar)) {
      ok = true;
      break;
    }
  ok = __syncthreads_and(ok) != 0;
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(err, kErrBuildWait);
    for (long it = 0; it < kDrainPolls; ++it)
      if (table_copy_done(bar)) break;
  }
  return ok;
}

template <int FK>
__global__ void __launch_bounds__(kThreads)
    kkr_build_kernel(const JobDev *__restrict__ jobs, BuildParams p, int *err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BuildSmem &sm = *reinterpret_cast<BuildSmem *>(smem_raw);
  const JobDev &J = jobs[blockIdx.y];
  const int pc = blockIdx.x;
  if (pc >= J.L) return;
  if (!stage_tables(sm, p.tables, err, p.table_polls)) return;
  const AngularTables &T = sm.tab;
  {
    const int it = threadIdx.x >> 5, L = threadIdx.x & 31;
    const int lm1 = (L >> 4) + 2 * it, lm2 = L & 15;
    const int te = lm2 * kMaxKK + lm1;
    const int rot = T.rot[te];
    const double sg = rot >= 2 ? -1.0 : 1.0;
    double c[kMaxTerms];
    unsigned d = (unsigned)(rot & 1) << 24;
#pragma unroll
    for (int q = 0; q < kMaxTerms; ++q) {  // unused terms: coefficient 0, index 0
      const bool on = q < T.nterm[te];
      c[q] = on ? sg * T.coef[te * kMaxTerms + q] : 0.0;
      d |= (unsigned)(on ? T.didx[te * kMaxTerms + q] : 0) << (6 * q);
    }
    sm.gc01[it][L] = make_double2(c[0], c[1]);
    sm.gc23[it][L] = make_double2(c[2], c[3]);
    sm.gd[it][L] = d;
  }
  __syncthreads();

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int ns = p.ns;
  const int kkrsz = p.kkrsz;
  const int bstore = ns * kkrsz;  // leading dimension of a stored t block
  const int j = J.perm[pc];
  const int lj = J.lmax[j];
  const int kkj = (lj + 1) * (lj + 1);
  const int col0 = J.off[pc];
  const int ld = J.ld;
  double2 *__restrict__ M = J.M;
  // second copy for the factorisation when refinement keeps M: FP64 (FK 1) or FP32 (FK 2)
  double2 *__restrict__ F64 = FK == 1 ? static_cast<double2 *>(J.F) : nullptr;
  float2 *__restrict__ F32 = FK == 2 ? static_cast<float2 *>(J.F) : nullptr;
  auto put = [&](size_t idx, double2 v) {
    M[idx] = v;
    if (FK == 1) F64[idx] = v;
    else if (FK == 2) F32[idx] = make_float2((float)v.x, (float)v.y);
  };
  const double2 prel = J.prel;
  // collinear spin-polarised: spin block offset kkrsz^2 * ispin (buildKKRMatrix_CPU.cpp:402)
  const long jsm = (p.npola != p.ns) ? (long)kkrsz * kkrsz * J.ispin : 0;

  // Row sites run in chunks of kChunk.  For a chunk, thread t < 2 kChunk computes one half of the
  // scalar prologue of pair t % kChunk: threads below kChunk the Hankel functions, the others
  // the Legendre functions and cos/sin(m phi), into pro[.][slot]; then the warps build the chunk's
  // blocks, pair pr = base + warp + kWarps q, from those values.
  double(*pro)[kChunk] = sm.pro;
  for (int base = 0; base < J.L; base += kChunk) {
    {
      const int slot = threadIdx.x % kChunk;
      const bool hankel = threadIdx.x < kChunk;
      const int pr = base + slot;
      if (threadIdx.x < 2 * kChunk && pr < J.L && pr != pc) {
        const int i = J.perm[pr];
        const int lend = J.lmax[i] + lj;
        // rij = pos(ir1) - pos(ir2), ir1 = row site (calculateTauMatrix.cpp:206-208)
        const double rx = J.pos[3 * i + 0] - J.pos[3 * j + 0];
        const double ry = J.pos[3 * i + 1] - J.pos[3 * j + 1];
        const double rz = J.pos[3 * i + 2] - J.pos[3 * j + 2];
        const double r = sqrt(rx * rx + ry * ry + rz * rz);
        if (hankel) {
          // spherical Hankel recursion, hfn_l = -i^(l+1) h_l(kR) e^{ikR}/R (:23-40)
          double2 H[kMaxLend + 1];
          const double2 z = make_double2(prel.x * r, prel.y * r);
          const double2 zi = cdiv(make_double2(1.0, 0.0), z);
          H[0] = make_double2(0.0, -1.0);
          {
            const double2 t = cmul(make_double2(0.0, 1.0), zi);
            H[1] = make_double2(-1.0 - t.x, -t.y);
          }
#pragma unroll
          for (int l = 1; l < kMaxLend; ++l) {
            const double2 a = cmul(H[l], zi);
            H[l + 1] = make_double2((2.0 * l + 1.0) * a.x - H[l - 1].x, (2.0 * l + 1.0) * a.y - H[l - 1].y);
          }
          double sn, cs;
          sincos(z.x, &sn, &cs);
          const double e = exp(-z.y) / r;
          const double2 f = make_double2(e * cs, e * sn);  // e^{iz}/r
#pragma unroll
          for (int l = 0; l <= kMaxLend; ++l) {
            if (l > lend) break;
            double2 h = cmul(H[l], f);
            h = cmul(h, make_double2(T.ilp1_re[l], T.ilp1_im[l]));
            pro[kProH + 2 * l][slot] = -h.x;
            pro[kProH + 2 * l + 1][slot] = -h.y;
          }
        } else {
          // normalised P_lm(cos theta) (associatedLegendreFunction.hpp:33-69)
          double P[kNdlm];
          const double x = rz / r;
          const double y = sqrt(1.0 - x * x);
          P[0] = sqrt(1.0 / (4.0 * 3.14159265358979323846));
#pragma unroll
          for (int m = 1; m <= kMaxLend; ++m) {
            const int mm = m * (m + 1) / 2 + m, pm = (m - 1) * m / 2 + (m - 1);
            P[mm] = -T.plm_mm[m] * y * P[pm];
            P[mm - 1] = T.plm_m1[m] * x * P[pm];
          }
#pragma unroll
          for (int m = 0; m < kMaxLend; ++m)
#pragma unroll
            for (int l = m + 2; l <= kMaxLend; ++l) {
              const int k = l * (l + 1) / 2 + m;
              P[k] = T.plm_a[k] * (x * P[(l - 1) * l / 2 + m] - T.plm_b[k] * P[(l - 2) * (l - 1) / 2 + m]);
            }
#pragma unroll
          for (int k = 0; k < kNdlm; ++k) pro[kProP + k][slot] = P[k];
          // cos(m phi), sin(m phi) (:42-59)
          const double pmag = sqrt(rx * rx + ry * ry);
          double c1 = 0.0, s1 = 0.0;
          if (pmag > 1.0e-6) {
            c1 = rx / pmag;
            s1 = ry / pmag;
          }
          double C = 1.0, S = 0.0;
          pro[kProC][slot] = 1.0;
          pro[kProS][slot] = 0.0;
#pragma unroll
          for (int m = 1; m <= kMaxLend; ++m) {
            const double Cm = m == 1 ? c1 : C * c1 - S * s1;
            const double Sm = m == 1 ? s1 : S * c1 + C * s1;
            C = Cm;
            S = Sm;
            pro[kProC + m][slot] = C;
            pro[kProS + m][slot] = S;
          }
        }
      }
    }
    __syncthreads();
    for (int q = 0; base + warp + kWarps * q < min(J.L, base + kChunk); ++q) {
    const int pr = base + warp + kWarps * q;
    const int slot = pr - base;
    const int i = J.perm[pr];
    const int li = J.lmax[i];
    const int kki = (li + 1) * (li + 1);
    const int row0 = J.off[pr];
    const int nr = ns * kki, nc = ns * kkj;
    if (pr == pc) {  // diagonal block: identity (buildKKRMatrix_CPU.cpp:266-268); G_ii = 0
      const double one = p.g_mode ? 0.0 : 1.0;
      for (int c = 0; c < nc; ++c)
        for (int r = lane; r < nr; r += 32)
          put((size_t)(row0 + r) + (size_t)(col0 + c) * ld, make_double2(r == c ? one : 0.0, 0.0));
      continue;
    }
    const int lend = li + lj;
    // D_{l,m} = hfn_l P_l|m| (cos m phi -/+ i sin m phi), (-1)^m for m < 0 (:127-140)
    for (int e = lane; e < (lend + 1) * (lend + 1); e += 32) {
      const int l = (int)sqrtf((float)e);  // exact: e < 64 and squares are exact in FP32
      const int m = e - l * (l + 1);
      const int am = m < 0 ? -m : m;
      const double pl = pro[kProP + l * (l + 1) / 2 + am][slot];
      const double2 h = make_double2(pro[kProH + 2 * l][slot], pro[kProH + 2 * l + 1][slot]);
      const double cm = pro[kProC + am][slot], sm_ = pro[kProS + am][slot];
      double2 f = make_double2(pl * cm, -pl * sm_);
      if (m < 0) {
        const double sg = (am & 1) ? -1.0 : 1.0;
        f = make_double2(sg * pl * cm, sg * pl * sm_);
      }
      sm.D[warp][e] = cmul(h, f);
    }
    __syncwarp();
    // M block = -t_i * diag_s(G): rows (s_r, r'), columns (s_c, c') (setgij.f:29-38)
    const double2 *__restrict__ tb =
        p.tmat + (long)J.store[i] * p.tmat_ld + (long)J.iie * p.blk + jsm;
    const bool tdiag = p.tdiag != nullptr && p.tdiag[((long)J.store[i] * p.group + J.iie) * 2 + J.ispin] != 0;
    // With a diagonal t (spherical scatterer) or for G itself each G element gives its M
    // elements directly; otherwise G is staged for the t G product.
    const bool direct = tdiag || p.g_mode;
    // G(lm2, lm1) = pi4 i^(l2-l1) sum_l3 cgnt(l3/2, lm1, lm2) D(l3, m2-m1) (:148-176); lanes run
    // along lm2 (rows) so that the direct stores are column segments.  When kki divides 32 a
    // lane's row lm2 is the same for all its elements, so the diagonal t values are loaded once.
    const bool lane_row = (32 % kki) == 0;
    double2 tdg0 = make_double2(0.0, 0.0), tdg1 = tdg0;  // spin 0, 1
    if (direct && !p.g_mode && lane_row) {
      const int t0 = lane % kki, t1 = kkrsz + lane % kki;
      tdg0 = __ldg(tb + t0 + (long)t0 * bstore);
      if (ns > 1) tdg1 = __ldg(tb + t1 + (long)t1 * bstore);
    }
    const double2 *Dw = sm.D[warp];
    if (direct && ns == 1 && kki == 16 && kkj == 16 && T.lmax == 3) {
      // -t_rr G for lmax-3 blocks from the per-lane gather records: the same sums, products and
      // roundings as the general loop below (the folded signs are exact)
      const double2 tneg = make_double2(-tdg0.x, -tdg0.y);
      const int lm2 = lane & 15;
#pragma unroll 2
      for (int it = 0; it < 8; ++it) {
        const int lm1 = (lane >> 4) + 2 * it;
        const double2 c01 = sm.gc01[it][lane], c23 = sm.gc23[it][lane];
        const unsigned d = sm.gd[it][lane];
        const double2 d0 = Dw[d & 63], d1 = Dw[(d >> 6) & 63], d2 = Dw[(d >> 12) & 63], d3 = Dw[(d >> 18) & 63];
        double2 acc = make_double2(0.0, 0.0);
        acc.x += c01.x * d0.x;
        acc.y += c01.x * d0.y;
        acc.x += c01.y * d1.x;
        acc.y += c01.y * d1.y;
        acc.x += c23.x * d2.x;
        acc.y += c23.x * d2.y;
        acc.x += c23.y * d3.x;
        acc.y += c23.y * d3.y;
        acc.x *= T.pi4;
        acc.y *= T.pi4;
        const double2 g = (d >> 24) ? make_double2(-acc.y, acc.x) : acc;
        const double2 v = p.g_mode ? g : cfma(tneg, g, make_double2(0.0, 0.0));
        put((size_t)(row0 + lm2) + (size_t)(col0 + lm1) * ld, v);
      }
      continue;
    }
    for (int e = lane; e < kki * kkj; e += 32) {
      const int lm1 = div_kk(e, kki), lm2 = e - lm1 * kki;
      const int te = lm2 * kMaxKK + lm1;
      const int nt = T.nterm[te];
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int q2 = 0; q2 < kMaxTerms; ++q2) {
        if (q2 < nt) {
          const double cg = T.coef[te * kMaxTerms + q2];
          const double2 d = Dw[T.didx[te * kMaxTerms + q2]];
          acc.x += cg * d.x;
          acc.y += cg * d.y;
        }
      }
      acc.x *= T.pi4;
      acc.y *= T.pi4;
      const int rot = T.rot[te];
      double2 g = acc;
      if (rot == 1) g = make_double2(-acc.y, acc.x);
      else if (rot == 2) g = make_double2(-acc.x, -acc.y);
      else if (rot == 3) g = make_double2(acc.y, -acc.x);
      if (!direct) {
        sm.G[warp][lm2 * kMaxKK + lm1] = g;
        continue;
      }
      for (int sr = 0; sr < ns; ++sr) {
        double2 v = g;
        if (!p.g_mode) {  // -t_rr G, rounded as the general path's one nonzero term
          double2 tv = sr == 0 ? tdg0 : tdg1;
          if (!lane_row) {
            const int trow = sr * kkrsz + lm2;
            tv = __ldg(tb + trow + (long)trow * bstore);
          }
          const double2 pr2 = cfma(tv, g, make_double2(0.0, 0.0));
          v = make_double2(-pr2.x, -pr2.y);
        }
        for (int sc = 0; sc < ns; ++sc)
          put((size_t)(row0 + sr * kki + lm2) + (size_t)(col0 + sc * kkj + lm1) * ld,
              sc == sr ? v : make_double2(0.0, 0.0));
      }
    }
    __syncwarp();
    if (direct) continue;
    const int r_lo = lane & 15;
    const int c_par = lane >> 4;
    for (int rr = r_lo; rr < nr; rr += 16) {
      const int trow = (rr / kki) * kkrsz + (rr % kki);
      for (int sc = 0; sc < ns; ++sc) {
        double2 trow_v[kMaxKK];
#pragma unroll
        for (int k = 0; k < kMaxKK; ++k)
          trow_v[k] = (k < kki) ? __ldg(tb + trow + (long)(sc * kkrsz + k) * bstore)
                                : make_double2(0.0, 0.0);
        for (int cp = c_par; cp < kkj; cp += 2) {
          double2 acc = make_double2(0.0, 0.0);
#pragma unroll
          for (int k = 0; k < kMaxKK; ++k)
            if (k < kki) acc = cfma(trow_v[k], sm.G[warp][k * kMaxKK + cp], acc);
          put((size_t)(row0 + rr) + (size_t)(col0 + sc * kkj + cp) * ld, make_double2(-acc.x, -acc.y));
        }
      }
    }
    __syncwarp();
    }
    __syncthreads();  // pro is rewritten by the next chunk's prologue
  }
}

// One warp per (store, energy, spin) t block: is every off-diagonal element exactly zero?
__global__ void tdiag_flags_kernel(const double2 *__restrict__ tmat, long ld, int nstore, int group, int b,
                                   int kkrsz, int colpol, unsigned char *__restrict__ flags) {
  const int f = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (f >= nstore * group * 2) return;
  const int sp = f & 1, ie = (f >> 1) % group, st = (f >> 1) / group;
  if (sp == 1 && !colpol) {
    if (lane == 0) flags[f] = 0;
    return;
  }
  const long blk = (long)(2 * kkrsz) * (2 * kkrsz);
  const double2 *t = tmat + (long)st * ld + (long)ie * blk + (colpol ? (long)kkrsz * kkrsz * sp : 0);
  bool off = false;
  for (int e = lane; e < b * b; e += 32) {
    const int c = e / b, r = e - c * b;
    const double2 v = t[e];
    off |= r != c && (v.x != 0.0 || v.y != 0.0);
  }
  off = __any_sync(0xffffffffu, off);
  if (lane == 0) flags[f] = off ? 0 : 1;
}

}  // namespace

cudaError_t launch_tdiag_flags(const double2 *tmat, long ld, int nstore, int group, int b, int kkrsz, bool colpol,
                               unsigned char *flags, cudaStream_t s) {
  const int n = nstore * group * 2;
  if (n <= 0) return cudaSuccess;
  tdiag_flags_kernel<<<(n + 7) / 8, 256, 0, s>>>(tmat, ld, nstore, group, b, kkrsz, colpol ? 1 : 0, flags);
  return cudaGetLastError();
}

cudaError_t launch_kkr_build(const JobDev *jobs, int njobs, int max_L, const BuildParams &p,
                             int *err_flags, cudaStream_t s, long *launches) {
  const int smem = (int)sizeof(BuildSmem);
  if (p.f_kind < 0 || p.f_kind > 2) return cudaErrorInvalidValue;
  void (*kern)(const JobDev *, BuildParams, int *) =
      p.f_kind == 0 ? kkr_build_kernel<0> : p.f_kind == 1 ? kkr_build_kernel<1> : kkr_build_kernel<2>;
  cudaError_t e = ensure_smem(kern, smem);
  if (e != cudaSuccess) return e;
  dim3 grid(max_L, njobs);
  kern<<<grid, kThreads, smem, s>>>(jobs, p, err_flags);
  if (launches) *launches += 1;
  return cudaGetLastError();
}

}  // namespace b200
