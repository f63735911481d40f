// C++ adapter: the reference's tau00 call surface on top of the b200tau C ABI.
//
// Header-only; the LSMS types are template parameters, so this file compiles inside the LSMS
// tree against the reference's own headers (src/Main/SystemParameters.hpp, src/SingleSite/
// AtomData.hpp, include/Matrix.hpp, include/Complex.hpp) without this library depending on them.
//
//   uploadTmatStore_b200   <- DeviceStorage::copyTmatStoreToDevice
//                             (src/Accelerator/DeviceStorage.cu:284-303; called where
//                             src/Main/energyContourIntegration.cpp:462-474 uploads the store)
//   setAtoms_b200          <- DeviceAtom::copyFromAtom (DeviceStorage.cu:341-404)
//   calculateTauMatrix_b200 <- calculateTauMatrix (src/MultipleScattering/calculateTauMatrix.cpp:320-323),
//                             identical argument list
//   calculateAllTauMatrices_b200 <- calculateAllTauMatrices (calculateTauMatrix.cpp:841-945),
//                             all local atoms (and both spins when collinear-polarised) in one batch
//
// Contexts: one per host thread and LSMS instance (the reference keeps one DeviceStorage per
// OpenMP thread, DeviceStorage.hpp:102-140); created lazily on the thread's current CUDA device.
// Errors are returned as b200tau status codes; the message is b200tau_last_error(context()).
#ifndef B200TAU_LSMS_ADAPTER_HPP
#define B200TAU_LSMS_ADAPTER_HPP

#include <cmath>
#include <complex>
#include <vector>

#include "b200tau.h"

namespace b200tau_lsms {

// The precision used by the adapter (B200TAU_PREC_*); the linearSolver id that selects this
// build path (a new id in the reference's linearSolver bitfield) is decoded by the caller.
inline int &precision() {
  static thread_local int prec = B200TAU_PREC_MIXED;
  return prec;
}

inline b200tau_ctx *&context_slot() {
  static thread_local b200tau_ctx *ctx = nullptr;
  return ctx;
}

// The calling thread's context for (maxlmax, n_spin_cant, n_spin_pola), created on first use.
template <class SystemParameters>
inline b200tau_ctx *context(SystemParameters &lsms, int device = 0) {
  b200tau_ctx *&ctx = context_slot();
  if (!ctx) {
    if (b200tau_create(&ctx, device, lsms.maxlmax, lsms.n_spin_cant, lsms.n_spin_pola) != B200TAU_OK)
      ctx = nullptr;
  }
  return ctx;
}

inline void release() {
  b200tau_destroy(context_slot());
  context_slot() = nullptr;
}

// LocalTypeInfo::tmatStore (SystemParameters.hpp:260-262) -> device, once per energy group.
template <class SystemParameters, class LocalTypeInfo>
int uploadTmatStore_b200(SystemParameters &lsms, LocalTypeInfo &local) {
  b200tau_ctx *ctx = context(lsms);
  if (!ctx) return B200TAU_ERR_CUDA;
  return b200tau_upload_tmat(ctx, reinterpret_cast<const double *>(&local.tmatStore(0, 0)),
                             (long)local.lDimTmatStore, (int)local.tmatStore.n_col(),
                             local.blkSizeTmatStore);
}

// AtomData LIZ (AtomData.hpp:440-445) and spin frame (ubr/ubrd, AtomData.hpp:466) of every
// local atom -> device, once per SCF iteration (the LIZ does not change within it).
template <class SystemParameters, class LocalTypeInfo>
int setAtoms_b200(SystemParameters &lsms, LocalTypeInfo &local) {
  b200tau_ctx *ctx = context(lsms);
  if (!ctx) return B200TAU_ERR_CUDA;
  for (int i = 0; i < local.num_local; i++) {
    auto &atom = local.atom[i];
    int rc = b200tau_set_atom(ctx, i, atom.numLIZ, &atom.LIZPos(0, 0), atom.LIZlmax.data(),
                              atom.LIZStoreIdx.data(), reinterpret_cast<const double *>(atom.ubr),
                              reinterpret_cast<const double *>(atom.ubrd));
    if (rc != B200TAU_OK) return rc;
  }
  return B200TAU_OK;
}

// Same arguments as calculateTauMatrix (calculateTauMatrix.cpp:320-323).  `m` is not needed
// (the KKR matrix lives in device memory) and is left untouched.
template <class SystemParameters, class LocalTypeInfo, class AtomData, class ComplexT, class MatrixT>
int calculateTauMatrix_b200(SystemParameters &lsms, LocalTypeInfo &local, AtomData &atom, int localAtomIndex,
                            int ispin, ComplexT energy, ComplexT prel, ComplexT *tau00_l, MatrixT &m, int iie) {
  (void)local;
  (void)atom;
  (void)m;
  b200tau_ctx *ctx = context(lsms);
  if (!ctx) return B200TAU_ERR_CUDA;
  b200tau_job job{};
  job.atom = localAtomIndex;
  job.iie = iie;
  job.ispin = ispin;
  job.energy[0] = std::real(energy);
  job.energy[1] = std::imag(energy);
  job.prel[0] = std::real(prel);
  job.prel[1] = std::imag(prel);
  return b200tau_solve(ctx, &job, 1, precision(), reinterpret_cast<double *>(tau00_l));
}

// calculateAllTauMatrices without the per-atom loop: every local atom (and the second spin when
// n_spin_pola != n_spin_cant, written to column i + num_local as calculateTauMatrix.cpp:914-916
// does) in one batched solve.  tau00_l is Matrix<Complex>(kkrsz_ns^2, num_local[*2]).
template <class SystemParameters, class LocalTypeInfo, class ComplexT, class MatrixT>
int calculateAllTauMatrices_b200(SystemParameters &lsms, LocalTypeInfo &local, ComplexT energy, int iie,
                                 MatrixT &tau00_l, double c2inv) {
  b200tau_ctx *ctx = context(lsms);
  if (!ctx) return B200TAU_ERR_CUDA;
  const ComplexT prel = std::sqrt(energy * (1.0 + energy * c2inv));  // calculateTauMatrix.cpp:846
  const int nspin = (lsms.n_spin_pola != lsms.n_spin_cant) ? 2 : 1;
  std::vector<b200tau_job> jobs;
  for (int s = 0; s < nspin; s++)
    for (int i = 0; i < local.num_local; i++) {
      b200tau_job j{};
      j.atom = i;
      j.iie = iie;
      j.ispin = s;
      j.energy[0] = std::real(energy);
      j.energy[1] = std::imag(energy);
      j.prel[0] = std::real(prel);
      j.prel[1] = std::imag(prel);
      jobs.push_back(j);
    }
  // job order (spin-major, then atom) matches the columns of tau00_l
  return b200tau_solve(ctx, jobs.data(), (int)jobs.size(), precision(),
                       reinterpret_cast<double *>(&tau00_l(0, 0)));
}

}  // namespace b200tau_lsms

#endif  // B200TAU_LSMS_ADAPTER_HPP
