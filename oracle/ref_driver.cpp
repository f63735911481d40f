// ORACLE / TEST INFRASTRUCTURE ONLY.  Never linked into the product library.
//
// Plain-pointer entry points around the reference's own C++ tau00 path, so the
// Python tests and the CPU baseline can call it through ctypes.  Each function
// fills the reference's boundary types (LSMSSystemParameters, LocalTypeInfo,
// AtomData, Matrix<Complex>) the way src/Main/lsms.cpp:244-248 and
// src/Main/buildLIZandCommLists.cpp:377-410,552-555 do, then calls
//   calculateTauMatrix   (src/MultipleScattering/calculateTauMatrix.cpp:320-837)
//   buildKKRMatrixCPU    (src/MultipleScattering/buildKKRMatrix_CPU.cpp:621-646)
// compiled from the reference source tree by oracle/Makefile.

#include <cstring>
#include <vector>

#include "Complex.hpp"
#include "Main/SystemParameters.hpp"
#include "Matrix.hpp"
#include "Misc/Coeficients.hpp"
#include "Misc/Indices.hpp"
#include "PhysicalConstants.hpp"

void calculateTauMatrix(LSMSSystemParameters &lsms, LocalTypeInfo &local,
                        AtomData &atom, int localAtomIndex, int ispin,
                        Complex energy, Complex prel, Complex *tau00_l,
                        Matrix<Complex> &m, int iie);
void buildKKRMatrixCPU(LSMSSystemParameters &lsms, LocalTypeInfo &local,
                       AtomData &atom, int ispin, int iie, Complex energy,
                       Complex prel, Matrix<Complex> &m);
void solveTauFullzgetrf(LSMSSystemParameters &lsms, LocalTypeInfo &local, AtomData &atom, Matrix<Complex> &m,
                        Matrix<Complex> &tau, int ispin);

namespace {

int g_tables_lmax = -1;

void init_tables(LSMSSystemParameters &lsms, int lmax) {
  if (g_tables_lmax == lmax) return;
  // src/Main/lsms.cpp:244-248
  AngularMomentumIndices::init(2 * lmax);
  SphericalHarmonicsCoeficients::init(2 * lmax);
  GauntCoeficients::init(lsms);
  IFactors::init(lsms, lmax);
  g_tables_lmax = lmax;
}

struct RefProblem {
  LSMSSystemParameters lsms;
  LocalTypeInfo local;
};

void setup(RefProblem &p, int lmax, int n_spin_cant, int n_spin_pola,
           unsigned solver, int numLIZ, const double *pos, const int *lizlmax,
           const int *storeIdx, int nstore, int group_size, const double *tmat,
           const double *ubr, const double *ubrd) {
  LSMSSystemParameters &lsms = p.lsms;
  lsms.lsmsMode = LSMSMode::main;
  lsms.rank = 0;
  lsms.relativity = scalar;
  lsms.n_spin_cant = n_spin_cant;
  lsms.n_spin_pola = n_spin_pola;
  lsms.maxlmax = lmax;
  lsms.zblockLUSize = 0;
  lsms.global.iprint = -1;
  lsms.global.GPUThreads = 1;
  lsms.global.linearSolver = solver;
  lsms.global.setIstop("main");
  init_tables(lsms, lmax);

  LocalTypeInfo &local = p.local;
  local.setNumLocal(1);
  const int kkrsz = (lmax + 1) * (lmax + 1);
  const int kkrsz2 = 2 * kkrsz;
  local.blkSizeTmatStore = kkrsz2 * kkrsz2;  // buildLIZandCommLists.cpp:552-555
  local.lDimTmatStore = local.blkSizeTmatStore * group_size;
  local.tmatStore.resize(local.lDimTmatStore, nstore);
  std::memcpy(&local.tmatStore(0, 0), tmat,
              sizeof(Complex) * (size_t)local.lDimTmatStore * nstore);

  AtomData &atom = local.atom[0];
  atom.lmax = lmax;
  atom.kkrsz = kkrsz;
  atom.numLIZ = numLIZ;
  atom.LIZStoreIdx.resize(numLIZ);
  atom.LIZlmax.resize(numLIZ);
  atom.LIZPos.resize(3, numLIZ);
  atom.nrmat = 0;
  for (int j = 0; j < numLIZ; j++) {
    atom.LIZStoreIdx[j] = storeIdx[j];
    atom.LIZlmax[j] = lizlmax[j];
    for (int c = 0; c < 3; c++) atom.LIZPos(c, j) = pos[3 * j + c];
    atom.nrmat += (lizlmax[j] + 1) * (lizlmax[j] + 1);
  }
  for (int k = 0; k < 4; k++) {
    atom.ubr[k] = Complex(ubr ? ubr[2 * k] : 0.0, ubr ? ubr[2 * k + 1] : 0.0);
    atom.ubrd[k] = Complex(ubrd ? ubrd[2 * k] : 0.0, ubrd ? ubrd[2 * k + 1] : 0.0);
  }
}

}  // namespace

extern "C" {

void tauref_set_num_threads(int n);

// tau00_l for one (atom, energy, spin): the reference's calculateTauMatrix.
// prel = sqrt(E (1 + E c2inv)) as in calculateTauMatrix.cpp:846.
int tauref_calculate(int lmax, int n_spin_cant, int n_spin_pola, unsigned solver,
                     int numLIZ, const double *pos, const int *lizlmax,
                     const int *storeIdx, int nstore, int group_size,
                     const double *tmat, int iie, int ispin, double e_re,
                     double e_im, const double *ubr, const double *ubrd,
                     double *tau00_l) {
  RefProblem p;
  setup(p, lmax, n_spin_cant, n_spin_pola, solver, numLIZ, pos, lizlmax,
        storeIdx, nstore, group_size, tmat, ubr, ubrd);
  AtomData &atom = p.local.atom[0];
  const Complex energy(e_re, e_im);
  const Complex prel = std::sqrt(energy * (1.0 + energy * c2inv));
  const int nrmat_ns = n_spin_cant * atom.nrmat;
  Matrix<Complex> m(nrmat_ns, nrmat_ns);
  calculateTauMatrix(p.lsms, p.local, atom, 0, ispin, energy, prel,
                     reinterpret_cast<Complex *>(tau00_l), m, iie);
  return 0;
}

// The KKR matrix M = 1 - t G exactly as the reference's C++ build leaves it.
int tauref_build_kkr(int lmax, int n_spin_cant, int n_spin_pola, int numLIZ,
                     const double *pos, const int *lizlmax, const int *storeIdx,
                     int nstore, int group_size, const double *tmat, int iie,
                     int ispin, double e_re, double e_im, double *m_out) {
  RefProblem p;
  setup(p, lmax, n_spin_cant, n_spin_pola, 0x2000, numLIZ, pos, lizlmax,
        storeIdx, nstore, group_size, tmat, nullptr, nullptr);
  AtomData &atom = p.local.atom[0];
  const Complex energy(e_re, e_im);
  const Complex prel = std::sqrt(energy * (1.0 + energy * c2inv));
  const int nrmat_ns = n_spin_cant * atom.nrmat;
  Matrix<Complex> m(nrmat_ns, nrmat_ns);
  buildKKRMatrixCPU(p.lsms, p.local, atom, ispin, iie, energy, prel, m);
  for (int j = 0; j < nrmat_ns; j++)
    for (int i = 0; i < nrmat_ns; i++) {
      m_out[2 * ((size_t)i + (size_t)nrmat_ns * j)] = m(i, j).real();
      m_out[2 * ((size_t)i + (size_t)nrmat_ns * j) + 1] = m(i, j).imag();
    }
  return nrmat_ns;
}

// Full tau = M^-1 T: the reference's C++ build followed by its solveTauFullzgetrf
// (src/MultipleScattering/linearSolvers_CPU.cpp:125-144), as src/Kubo/CurrentMatrix.cpp:184-190
// calls them.
int tauref_tau_full(int lmax, int n_spin_cant, int n_spin_pola, int numLIZ, const double *pos,
                    const int *lizlmax, const int *storeIdx, int nstore, int group_size,
                    const double *tmat, int iie, int ispin, double e_re, double e_im,
                    double *tau_out) {
  RefProblem p;
  setup(p, lmax, n_spin_cant, n_spin_pola, 0x2000, numLIZ, pos, lizlmax,
        storeIdx, nstore, group_size, tmat, nullptr, nullptr);
  AtomData &atom = p.local.atom[0];
  const Complex energy(e_re, e_im);
  const Complex prel = std::sqrt(energy * (1.0 + energy * c2inv));
  const int nrmat_ns = n_spin_cant * atom.nrmat;
  Matrix<Complex> m(nrmat_ns, nrmat_ns), tau(nrmat_ns, nrmat_ns);
  buildKKRMatrixCPU(p.lsms, p.local, atom, ispin, iie, energy, prel, m);
  solveTauFullzgetrf(p.lsms, p.local, atom, m, tau, ispin);
  for (int j = 0; j < nrmat_ns; j++)
    for (int i = 0; i < nrmat_ns; i++) {
      tau_out[2 * ((size_t)i + (size_t)nrmat_ns * j)] = tau(i, j).real();
      tau_out[2 * ((size_t)i + (size_t)nrmat_ns * j) + 1] = tau(i, j).imag();
    }
  return nrmat_ns;
}

// The angular tables after the reference's init: cgnt (lmax+1, kkrsz, kkrsz)
// Fortran order, illp (kkrsz, kkrsz) column-major complex, ilp1 (2 lmax + 1).
int tauref_tables(int lmax, double *cgnt, double *illp, double *ilp1) {
  LSMSSystemParameters lsms;
  lsms.global.iprint = -1;
  lsms.global.setIstop("main");
  lsms.maxlmax = lmax;
  init_tables(lsms, lmax);
  const int kkrsz = (lmax + 1) * (lmax + 1);
  for (int k = 0; k < kkrsz; k++)
    for (int j = 0; j < kkrsz; j++)
      for (int l = 0; l <= lmax; l++)
        cgnt[l + (lmax + 1) * (j + kkrsz * k)] = GauntCoeficients::cgnt(l, j, k);
  for (int j = 0; j < kkrsz; j++)
    for (int i = 0; i < kkrsz; i++) {
      illp[2 * (i + kkrsz * j)] = IFactors::illp(i, j).real();
      illp[2 * (i + kkrsz * j) + 1] = IFactors::illp(i, j).imag();
    }
  for (int l = 0; l <= 2 * lmax; l++) {
    ilp1[2 * l] = IFactors::ilp1[l].real();
    ilp1[2 * l + 1] = IFactors::ilp1[l].imag();
  }
  return 0;
}

}  // extern "C"
