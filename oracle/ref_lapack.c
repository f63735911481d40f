/* ORACLE / TEST INFRASTRUCTURE ONLY.
 * The reference calls Fortran-style BLAS/LAPACK symbols (zgemm_, zgetrf_, ...).
 * No system BLAS is installed; scipy ships an LP64 OpenBLAS whose exports carry a
 * "scipy_" prefix.  These one-line forwarders bind the reference's calls to it. */
#include <complex.h>
typedef double _Complex zc;

void scipy_zgemm_(const char*, const char*, int*, int*, int*, const zc*, const zc*, int*,
                  const zc*, int*, const zc*, zc*, int*);
void scipy_zcopy_(int*, const zc*, int*, zc*, int*);
void scipy_zgetrf_(int*, int*, zc*, int*, int*, int*);
void scipy_zgetrs_(const char*, int*, int*, zc*, int*, int*, zc*, int*, int*);
void scipy_zgesv_(int*, int*, zc*, int*, int*, zc*, int*, int*);
void scipy_zcgesv_(int*, int*, zc*, int*, int*, zc*, int*, zc*, int*, zc*, float _Complex*,
                   double*, int*, int*);
void scipy_openblas_set_num_threads(int);

void zgemm_(const char* ta, const char* tb, int* m, int* n, int* k, const zc* al, const zc* a,
            int* lda, const zc* b, int* ldb, const zc* be, zc* c, int* ldc) {
  scipy_zgemm_(ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc);
}
void zcopy_(int* n, const zc* x, int* ix, zc* y, int* iy) { scipy_zcopy_(n, x, ix, y, iy); }
int zgetrf_(int* m, int* n, zc* a, int* lda, int* ipiv, int* info) {
  scipy_zgetrf_(m, n, a, lda, ipiv, info);
  return 0;
}
int zgetrs_(const char* t, int* n, int* nrhs, zc* a, int* lda, int* ipiv, zc* b, int* ldb,
            int* info) {
  scipy_zgetrs_(t, n, nrhs, a, lda, ipiv, b, ldb, info);
  return 0;
}
void zgesv_(int* n, int* nrhs, zc* a, int* lda, int* ipiv, zc* b, int* ldb, int* info) {
  scipy_zgesv_(n, nrhs, a, lda, ipiv, b, ldb, info);
}
void zcgesv_(int* n, int* nrhs, zc* a, int* lda, int* ipiv, zc* b, int* ldb, zc* x, int* ldx,
             zc* work, float _Complex* swork, double* rwork, int* iter, int* info) {
  scipy_zcgesv_(n, nrhs, a, lda, ipiv, b, ldb, x, ldx, work, swork, rwork, iter, info);
}
void tauref_set_num_threads(int n) { scipy_openblas_set_num_threads(n); }
