// ORACLE / TEST INFRASTRUCTURE ONLY.  Never linked into the product library.
//
// C++ restatements of the few Fortran routines that the reference's C++
// tau00 path (calculateTauMatrix with build id 0x2000 and solver ids
// 0x2001/0x2002/0x2005/0x2f01) calls.  gfortran is not available, so these are
// written from the cited Fortran sources; everything else in the oracle is the
// reference's own C++ compiled from its source tree (see oracle/Makefile).
//
// Symbols the chosen solver ids never reach (makegij_, setgij_, block_inv_,
// write_kkrmat_, tripmt_, tau_inv_postproc_rel_) abort if called.

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <ctime>

typedef std::complex<double> Cplx;

extern "C" {
void gauss_legendre_points_(double *x1, double *x2, double *x, double *w, int *n);
void plm_normalized_(int *lmax, double *x, double *plm);
void zgetrf_(int *m, int *n, Cplx *a, int *lda, int *ipvt, int *info);
void zgetrs_(const char *t, int *n, int *nrhs, Cplx *a, int *lda, int *ipvt,
             Cplx *b, int *ldb, int *info);
}

double MPI_Wtime() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// src/Misc/gaunt.f:100-119 (defac): sign factor and 0-based packed index of P_l|m|.
static void defac(int l, int m, int &ifac, int &jl) {
  if (m >= 0) {
    ifac = 1;
    jl = l * (l + 1) / 2 + m;
  } else {
    ifac = (std::abs(m) % 2 == 0) ? 1 : -1;
    jl = l * (l + 1) / 2 - m;
  }
}

// src/Misc/gaunt.f:1-97 (gaunt): quadrature of three normalised P_lm over the
// first `ngauss` Gauss-Legendre nodes, zeroed below 1e-14.
static double gaunt(int l1, int m1, int l2, int m2, int l3, int m3, int lmaxp,
                    int ngauss, const double *wg, const double *plmg,
                    const double *clm) {
  const int ldp = (lmaxp + 1) * (lmaxp + 2) / 2;
  const double pi = 3.141592653589793;
  const double fourpi = 4.0 * pi;
  if (l1 > lmaxp || l2 > lmaxp || l3 > lmaxp) {
    fprintf(stderr, "gaunt:: bad parameters\n");
    abort();
  }
  double val = 0.0;
  if ((l1 + l2 + l3) % 2 != 0) return 0.0;
  if (m1 - m2 + m3 != 0) return 0.0;
  if (l1 + l2 < l3 || l2 + l3 < l1 || l3 + l1 < l2) return 0.0;
  int ifac1, jl1, ifac2, jl2, ifac3, jl3;
  defac(l1, m1, ifac1, jl1);
  defac(l2, -m2, ifac2, jl2);
  defac(l3, m3, ifac3, jl3);
  for (int ng = 0; ng < ngauss; ng++)
    val += wg[ng] * plmg[jl1 + ng * ldp] * plmg[jl2 + ng * ldp] *
           plmg[jl3 + ng * ldp];
  if (std::fabs(val) < 1.0e-14) return 0.0;
  const int sgn2 = 1 - 2 * (std::abs(m2) % 2);
  return fourpi * val * ifac1 * clm[jl1] * sgn2 * ifac2 * clm[jl2] * ifac3 *
         clm[jl3];
}

extern "C" {

// src/Misc/cgaunt_c.f90:3-109 (cgaunt).  cgnt is Fortran cgnt(lmax+1,(lmax+1)^2,(lmax+1)^2).
void cgaunt_(int *lmax_p, double *clm, double *plmg, double *tg, double *wg,
             double *cgnt, int *lofk, int *mofk, int *iprint, char *istop) {
  (void)iprint;
  (void)istop;
  const int lmax = *lmax_p;
  int ntot = 2 * (2 * lmax + 1);
  double m1d = -1.0, p1d = 1.0;
  gauss_legendre_points_(&m1d, &p1d, tg, wg, &ntot);
  const int n1 = 2 * lmax + 1;
  const int ldp = (2 * lmax + 1) * (2 * lmax + 2) / 2;
  int l2max = 2 * lmax;
  for (int ng = 0; ng < n1; ng++) plm_normalized_(&l2max, &tg[ng], &plmg[ng * ldp]);
  const int nk = (lmax + 1) * (lmax + 1);
  for (int j2 = 0; j2 < nk; j2++) {
    const int l2 = lofk[j2], m2 = mofk[j2];
    for (int j1 = 0; j1 < nk; j1++) {
      const int l1 = lofk[j1], m1 = mofk[j1];
      const int m3 = m2 - m1;
      const int llow = std::max(std::abs(m3), std::abs(l1 - l2));
      for (int l3 = l1 + l2; l3 >= llow; l3 -= 2) {
        double c = gaunt(l1, m1, l2, m2, l3, m3, 2 * lmax, 2 * lmax + 1, wg,
                         plmg, clm);
        if (std::fabs(c) < 1.0e-14) c = 0.0;
        cgnt[l3 / 2 + (lmax + 1) * (j1 + nk * j2)] = c;
      }
    }
  }
}

// src/Misc/ifacts_c.f:3-72 (ifacts): illp(lm,lmp) = i^(l-lp), ilp1(l) = i^(l+1).
void ifacts_(int *lmax_p, Cplx *illp, Cplx *ilp1, int *iprint, char *istop,
             int istop_len) {
  (void)iprint;
  (void)istop;
  (void)istop_len;
  const int lmax = *lmax_p;
  const Cplx sqrtm1(0.0, 1.0);
  ilp1[0] = Cplx(1.0, 0.0);
  for (int l = 1; l <= 2 * lmax; l++) ilp1[l] = ilp1[l - 1] * sqrtm1;
  const int nk = (lmax + 1) * (lmax + 1);
  for (int l = 0; l <= lmax; l++)
    for (int m = -l; m <= l; m++) {
      const int lm = l * (l + 1) + m;
      for (int lp = 0; lp <= lmax; lp++)
        for (int mp = -lp; mp <= lp; mp++) {
          const int lmp = lp * (lp + 1) + mp;
          illp[lm + nk * lmp] = ilp1[l] / ilp1[lp];
        }
    }
  for (int l = 0; l <= 2 * lmax; l++) ilp1[l] = ilp1[l] * sqrtm1;
}

// src/Misc/spin_trafo.f:1-59: u = spin-space rotation for moment direction evec, ud = u^+.
void spin_trafo_(double *evec, Cplx *u, Cplx *ud) {
  const double tol = 1.0e-8;
  const Cplx sqrtm1(0.0, 1.0);
  u[0] = std::sqrt(0.5 * (1.0 + evec[2]));
  if (std::abs(u[0]) < tol) {
    u[0] = 0.0;
    u[1] = 1.0;
    u[2] = 1.0;
  } else {
    u[1] = -0.5 * (evec[0] + sqrtm1 * evec[1]) / u[0];
    u[2] = 0.5 * (evec[0] - sqrtm1 * evec[1]) / u[0];
  }
  u[3] = u[0];
  ud[0] = std::conj(u[0]);
  ud[1] = std::conj(u[2]);
  ud[2] = std::conj(u[1]);
  ud[3] = std::conj(u[3]);
}

// src/MultipleScattering/trgtol.f:3-110: ml(:,:,k) = (u * mg * ud) spin block k
// (k in column-major order of the 2x2 spin matrix).
void trgtol_(int *nr_p, int *nc_p, Cplx *u, Cplx *ud, Cplx *mg, Cplx *ml) {
  const int nr = *nr_p, nc = *nc_p;
  const int ldg = 2 * nr;
  for (int i = 0; i < 4 * nr * nc; i++) ml[i] = 0.0;
  // (row-spin of u, column-spin of ud) for output block k = 0..3
  const int ia[4] = {0, 1, 0, 1};  // u(ia, .)
  const int jb[4] = {0, 0, 1, 1};  // ud(., jb)
  for (int k = 0; k < 4; k++) {
    Cplx *out = ml + (size_t)k * nr * nc;
    for (int q = 0; q < 2; q++)        // column spin of mg
      for (int p = 0; p < 2; p++) {    // row spin of mg
        // u is column-major 2x2: u(r,c) = u[r + 2c]
        const Cplx f = u[ia[k] + 2 * p] * ud[q + 2 * jb[k]];
        for (int j = 0; j < nc; j++)
          for (int i = 0; i < nr; i++)
            out[i + nr * j] += f * mg[(p * nr + i) + ldg * (q * nc + j)];
      }
  }
}

// src/MultipleScattering/tau_inv_postproc.f:1-77: tau00 = (1-delta)^-1 t,
// output delta*tau00 (= tau00 - t), rotated for n_spin_cant = 2.
void tau_inv_postproc_nrel_(int *kkrsz_ns_p, int *n_spin_cant, Cplx *wbig,
                            Cplx *delta, Cplx *tmat, int *ipvt, Cplx *tau00,
                            Cplx *ubr, Cplx *ubrd, Cplx *tau00_l) {
  int n = *kkrsz_ns_p;
  const int nn = n * n;
  for (int i = 0; i < nn; i++) wbig[i] = 0.0;
  for (int i = 0; i < n; i++) wbig[i + n * i] = 1.0;
  for (int i = 0; i < nn; i++) wbig[i] -= delta[i];
  int info;
  zgetrf_(&n, &n, wbig, &n, ipvt, &info);
  for (int i = 0; i < nn; i++) tau00[i] = tmat[i];
  zgetrs_("n", &n, &n, wbig, &n, ipvt, tau00, &n, &info);
  Cplx *tmp = new Cplx[nn];
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      Cplx s = 0.0;
      for (int k = 0; k < n; k++) s += delta[i + n * k] * tau00[k + n * j];
      tmp[i + n * j] = s;
    }
  if (*n_spin_cant == 2) {
    int kk = n / 2;
    trgtol_(&kk, &kk, ubr, ubrd, tmp, tau00_l);
  } else {
    for (int i = 0; i < nn; i++) tau00_l[i] = tmp[i];
  }
  delete[] tmp;
}

static void unreachable(const char *name) {
  fprintf(stderr, "oracle: %s is not reachable with the configured solver id\n", name);
  abort();
}
void makegij_() { unreachable("makegij_"); }
void setgij_() { unreachable("setgij_"); }
void block_inv_() { unreachable("block_inv_"); }
void write_kkrmat_() { unreachable("write_kkrmat_"); }
void tripmt_() { unreachable("tripmt_"); }
void tau_inv_postproc_rel_() { unreachable("tau_inv_postproc_rel_"); }

}  // extern "C"
