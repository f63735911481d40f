// Angular-momentum tables for the G0 build, computed on the host once per context.
//
// What the reference computes at start-up (src/Main/lsms.cpp:244-248):
//   AngularMomentumIndices (src/Misc/Indices.hpp:136-170): lofk/mofk up to 2 lmax,
//   Gaunt numbers cgnt(l3/2, L1, L2) = int Y_L1 Y*_L2 Y_L3 (src/Misc/cgaunt_c.f90:3-109,
//     src/Misc/gaunt.f:1-119): Gauss-Legendre quadrature of normalised P_lm,
//   i-factors illp = i^(l-l'), ilp1 = i^(l+1) (src/Misc/ifacts_c.f:3-72).
// Here the same quantities are produced by this file's own quadrature (Newton
// iteration for the Legendre roots, exact for the polynomial integrands up to
// degree 4 (2 lmax + 1) - 1) and folded into a gather list per G element.

#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace b200 {
namespace {

// Gauss-Legendre nodes/weights on [-1, 1] by Newton iteration on P_n.
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  const double pi = std::acos(-1.0);
  for (int i = 0; i < n; i++) {
    double z = std::cos(pi * (i + 0.75) / (n + 0.5));
    double dp = 1.0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = 0.0;
      for (int k = 1; k <= n; k++) {
        double p2 = p1;
        p1 = p0;
        p0 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p2) / k;
      }
      dp = n * (z * p0 - p1) / (z * z - 1.0);
      double dz = p0 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = 0.0;
    for (int k = 1; k <= n; k++) {
      double p2 = p1;
      p1 = p0;
      p0 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p2) / k;
    }
    dp = n * (z * p0 - p1) / (z * z - 1.0);
    x[i] = -z;
    w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

inline int pidx(int l, int m) { return l * (l + 1) / 2 + m; }

// Normalised associated Legendre functions (Y_lm = Pbar_lm(cos t) e^{i m phi},
// Condon-Shortley phase included), all l <= lmax, index l(l+1)/2 + m.
void plm_normalised(double x, int lmax, double *p) {
  const double pi = std::acos(-1.0);
  const double y = std::sqrt(1.0 - x * x);
  p[0] = std::sqrt(1.0 / (4.0 * pi));
  for (int m = 1; m <= lmax; m++) {
    p[pidx(m, m)] = -std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * y * p[pidx(m - 1, m - 1)];
    p[pidx(m, m - 1)] = std::sqrt(2.0 * m + 1.0) * x * p[pidx(m - 1, m - 1)];
  }
  for (int m = 0; m < lmax; m++)
    for (int l = m + 2; l <= lmax; l++) {
      double a = std::sqrt((4.0 * l * l - 1.0) / (double(l * l) - double(m * m)));
      double b = std::sqrt((double((l - 1) * (l - 1)) - double(m * m)) /
                           (4.0 * (l - 1) * (l - 1) - 1.0));
      p[pidx(l, m)] = a * (x * p[pidx(l - 1, m)] - b * p[pidx(l - 2, m)]);
    }
}

}  // namespace

// cgnt[l3/2 + (lmax+1)*(j1 + kk*j2)] = int Y_L1 Y*_L2 Y_L3 dOmega, L3 = (l3, m2 - m1),
// for |l1-l2| <= l3 <= l1+l2 with l1+l2+l3 even; |c| < 1e-14 flushed to 0.
void gaunt_numbers(int lmax, double *cgnt) {
  const int kk = (lmax + 1) * (lmax + 1);
  const int lp = 2 * lmax;
  const int ng = 2 * (2 * lmax + 1);
  std::vector<double> x, w;
  gauss_legendre(ng, x, w);
  const int nd = (lp + 1) * (lp + 2) / 2;
  std::vector<double> plm((size_t)ng * nd);
  for (int g = 0; g < ng; g++) plm_normalised(x[g], lp, &plm[(size_t)g * nd]);
  std::vector<int> lofk, mofk;
  for (int l = 0; l <= lp; l++)
    for (int m = -l; m <= l; m++) {
      lofk.push_back(l);
      mofk.push_back(m);
    }
  const double twopi = 2.0 * std::acos(-1.0);
  std::memset(cgnt, 0, sizeof(double) * (lmax + 1) * kk * kk);
  auto pl = [&](int g, int l, int m, int &sgn) {
    sgn = 1;
    if (m < 0) {
      m = -m;
      if (m & 1) sgn = -1;
    }
    return plm[(size_t)g * nd + pidx(l, m)];
  };
  for (int j2 = 0; j2 < kk; j2++)
    for (int j1 = 0; j1 < kk; j1++) {
      const int l1 = lofk[j1], m1 = mofk[j1], l2 = lofk[j2], m2 = mofk[j2];
      const int m3 = m2 - m1;
      const int llow = std::max(std::abs(m3), std::abs(l1 - l2));
      for (int l3 = l1 + l2; l3 >= llow; l3 -= 2) {
        double s = 0.0;
        int s1 = 1, s2 = 1, s3 = 1;
        for (int g = 0; g < ng; g++)
          s += w[g] * pl(g, l1, m1, s1) * pl(g, l2, -m2, s2) * pl(g, l3, m3, s3);
        double c = 0.0;
        if (std::fabs(s) >= 1e-14) {
          // Y*_{l2 m2} = (-1)^m2 Y_{l2,-m2}; the phi integral gives 2 pi.
          const int cs = (std::abs(m2) & 1) ? -1 : 1;
          c = twopi * s * s1 * s2 * s3 * cs;
        }
        if (std::fabs(c) < 1e-14) c = 0.0;
        cgnt[l3 / 2 + (lmax + 1) * (j1 + kk * j2)] = c;
      }
    }
}

int build_angular_tables(int lmax, AngularTables *t) {
  if (lmax < 0 || lmax > kMaxLmax) return 1;
  std::memset(t, 0, sizeof(*t));
  t->lmax = lmax;
  const int kk = (lmax + 1) * (lmax + 1);
  std::vector<double> cg((size_t)(lmax + 1) * kk * kk);
  gaunt_numbers(lmax, cg.data());
  std::vector<int> lofk, mofk;
  for (int l = 0; l <= lmax; l++)
    for (int m = -l; m <= l; m++) {
      lofk.push_back(l);
      mofk.push_back(m);
    }
  // Gather list in the reference's order: l3 from l1+l2 down to llow
  // (buildKKRMatrix_CPU.cpp:148-175).  Row lm2 belongs to site i, column lm1 to site j.
  for (int lm2 = 0; lm2 < kk; lm2++)
    for (int lm1 = 0; lm1 < kk; lm1++) {
      const int e = lm2 * kMaxKK + lm1;
      const int l1 = lofk[lm1], m1 = mofk[lm1], l2 = lofk[lm2], m2 = mofk[lm2];
      const int m3 = m2 - m1;
      const int llow = std::max(std::abs(m3), std::abs(l1 - l2));
      int q = 0;
      for (int l3 = l1 + l2; l3 >= llow; l3 -= 2) {
        t->coef[e * kMaxTerms + q] = cg[l3 / 2 + (lmax + 1) * (lm1 + kk * lm2)];
        t->didx[e * kMaxTerms + q] = l3 * (l3 + 1) + m3;
        q++;
      }
      t->nterm[e] = q;
      t->rot[e] = (((l2 - l1) % 4) + 4) % 4;
    }
  // i^(l+1)
  for (int l = 0; l <= 2 * lmax; l++) {
    const int r = (l + 1) % 4;
    t->ilp1_re[l] = (r == 0) ? 1.0 : (r == 2 ? -1.0 : 0.0);
    t->ilp1_im[l] = (r == 1) ? 1.0 : (r == 3 ? -1.0 : 0.0);
  }
  const int lp = 2 * lmax;
  for (int m = 1; m <= lp; m++) {
    t->plm_mm[m] = std::sqrt((2.0 * m + 1.0) / (2.0 * m));
    t->plm_m1[m] = std::sqrt(2.0 * m + 1.0);
  }
  for (int m = 0; m < lp; m++)
    for (int l = m + 2; l <= lp; l++) {
      t->plm_a[pidx(l, m)] = std::sqrt((4.0 * l * l - 1.0) / (double(l * l) - double(m * m)));
      t->plm_b[pidx(l, m)] = std::sqrt((double((l - 1) * (l - 1)) - double(m * m)) /
                                       (4.0 * (l - 1) * (l - 1) - 1.0));
    }
  t->pi4 = 4.0 * 2.0 * std::asin(1.0);
  return 0;
}

}  // namespace b200
