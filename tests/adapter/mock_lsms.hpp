// Minimal stand-ins for the LSMS boundary types (field names and layouts of
// src/Main/SystemParameters.hpp, src/SingleSite/AtomData.hpp, include/Matrix.hpp) so the adapter
// can be compiled and exercised without the reference tree.
#pragma once
#include <complex>
#include <vector>

typedef std::complex<double> Complex;

template <class T>
struct Matrix {  // column-major, operator()(i, j) = data[i + j * lDim] (Matrix.hpp:126-148)
  int lDim = 0, nCol = 0;
  std::vector<T> data;
  Matrix() = default;
  Matrix(int m, int n) { resize(m, n); }
  void resize(int m, int n) { lDim = m; nCol = n; data.assign((size_t)m * n, T()); }
  T &operator()(int i, int j) { return data[i + (size_t)j * lDim]; }
  int n_col() const { return nCol; }
};

struct LSMSSystemParameters {
  int maxlmax = 3, n_spin_cant = 1, n_spin_pola = 1;
};

struct AtomData {
  int numLIZ = 0;
  std::vector<int> LIZStoreIdx, LIZlmax;
  Matrix<double> LIZPos;
  Complex ubr[4], ubrd[4];
};

struct LocalTypeInfo {
  int num_local = 0;
  std::vector<AtomData> atom;
  int lDimTmatStore = 0, blkSizeTmatStore = 0;
  Matrix<Complex> tmatStore;
};
