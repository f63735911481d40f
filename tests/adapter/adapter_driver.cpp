// Exercises include/b200tau_lsms_adapter.hpp with the stand-in types: reads a problem written by
// the Python test (binary, see tests/test_adapter.py), runs calculateTauMatrix_b200 for every
// energy and calculateAllTauMatrices_b200 for energy 0, and writes tau00_l back.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "b200tau_lsms_adapter.hpp"
#include "mock_lsms.hpp"

static void rd(FILE *f, void *p, size_t n) {
  if (fread(p, 1, n, f) != n) { fprintf(stderr, "short read\n"); exit(2); }
}

int main(int argc, char **argv) {
  if (argc != 3) return 2;
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 2;
  int hdr[6];  // lmax, ns, npola, L, nstore, ngroup
  rd(f, hdr, sizeof(hdr));
  LSMSSystemParameters lsms;
  lsms.maxlmax = hdr[0];
  lsms.n_spin_cant = hdr[1];
  lsms.n_spin_pola = hdr[2];
  const int L = hdr[3], nstore = hdr[4], ngroup = hdr[5];
  const int kk = (hdr[0] + 1) * (hdr[0] + 1), b = hdr[1] * kk, blk = 4 * kk * kk;
  LocalTypeInfo local;
  local.num_local = 1;
  local.atom.resize(1);
  AtomData &atom = local.atom[0];
  atom.numLIZ = L;
  atom.LIZPos.resize(3, L);
  atom.LIZlmax.resize(L);
  atom.LIZStoreIdx.resize(L);
  rd(f, atom.LIZPos.data.data(), sizeof(double) * 3 * L);
  rd(f, atom.LIZlmax.data(), sizeof(int) * L);
  rd(f, atom.LIZStoreIdx.data(), sizeof(int) * L);
  rd(f, atom.ubr, sizeof(atom.ubr));
  rd(f, atom.ubrd, sizeof(atom.ubrd));
  local.blkSizeTmatStore = blk;
  local.lDimTmatStore = blk * ngroup;
  local.tmatStore.resize(local.lDimTmatStore, nstore);
  rd(f, local.tmatStore.data.data(), sizeof(Complex) * local.tmatStore.data.size());
  std::vector<Complex> energies(ngroup);
  rd(f, energies.data(), sizeof(Complex) * ngroup);
  fclose(f);

  const double c2inv = 1.0 / (274.071998412 * 274.071998412);
  b200tau_lsms::precision() = B200TAU_PREC_FP64;
  if (b200tau_lsms::uploadTmatStore_b200(lsms, local) != B200TAU_OK) return 3;
  if (b200tau_lsms::setAtoms_b200(lsms, local) != B200TAU_OK) return 4;
  std::vector<Complex> out((size_t)ngroup * b * b + b * b);
  Matrix<Complex> m;
  for (int ie = 0; ie < ngroup; ie++) {
    const Complex prel = std::sqrt(energies[ie] * (1.0 + energies[ie] * c2inv));
    int rc = b200tau_lsms::calculateTauMatrix_b200(lsms, local, atom, 0, 0, energies[ie], prel,
                                                   &out[(size_t)ie * b * b], m, ie);
    if (rc != B200TAU_OK) {
      fprintf(stderr, "calculateTauMatrix_b200: %s\n", b200tau_last_error(b200tau_lsms::context(lsms)));
      return 5;
    }
  }
  Matrix<Complex> all(b * b, 1);
  if (b200tau_lsms::calculateAllTauMatrices_b200(lsms, local, energies[0], 0, all, c2inv) != B200TAU_OK) return 6;
  for (int e = 0; e < b * b; e++) out[(size_t)ngroup * b * b + e] = all(e, 0);
  b200tau_lsms::release();
  FILE *o = fopen(argv[2], "wb");
  fwrite(out.data(), sizeof(Complex), out.size(), o);
  fclose(o);
  return 0;
}
