// Host matrix containers: reading through libcgb200's MatrixMarket reader
// and the CRS / ELL builds (stable bucketing of COO entries by row, so every
// row keeps file order, as the reference's conversions do:
// Matrix.cpp:203-228 and 339-361).
#include "Matrix.h"

#include <cstdlib>
#include <cstring>
#include <iostream>
#include <vector>

#include "cgx.h"

MatrixCOO::MatrixCOO(const char *file) {
  int n = 0, z = 0;
  int *i = nullptr, *j = nullptr;
  double *v = nullptr;
  cgx_status st = cgx_mtx_read(file, &n, &z, &i, &j, &v);
  if (st != CGX_SUCCESS) {
    std::cerr << cgx_last_error() << std::endl;
    std::exit(1);
  }
  N = n;
  nz = z;
  I.reset(new int[nz > 0 ? nz : 1]);
  J.reset(new int[nz > 0 ? nz : 1]);
  V.reset(new floatType[nz > 0 ? nz : 1]);
  nzPerRow.reset(new int[N > 0 ? N : 1]());
  if (nz > 0) {
    std::memcpy(I.get(), i, sizeof(int) * (size_t)nz);
    std::memcpy(J.get(), j, sizeof(int) * (size_t)nz);
    std::memcpy(V.get(), v, sizeof(double) * (size_t)nz);
  }
  cgx_free(i);
  cgx_free(j);
  cgx_free(v);
  for (int e = 0; e < nz; e++) nzPerRow[I[e]]++;
}

int MatrixCOO::getMaxNz() const {
  int m = 0;
  for (int r = 0; r < N; r++) m = nzPerRow[r] > m ? nzPerRow[r] : m;
  return m;
}

void MatrixDataCRS::allocatePtr(int rows) { ptr = new int[rows + 1]; }
void MatrixDataCRS::deallocatePtr() {
  delete[] ptr;
  ptr = nullptr;
}
void MatrixDataCRS::allocateIndexAndValue(int values) {
  index = new int[values > 0 ? values : 1];
  value = new floatType[values > 0 ? values : 1];
}
void MatrixDataCRS::deallocateIndexAndValue() {
  delete[] index;
  delete[] value;
  index = nullptr;
  value = nullptr;
}

void MatrixDataELL::allocateLength(int rows) { length = new int[rows]; }
void MatrixDataELL::deallocateLength() {
  delete[] length;
  length = nullptr;
}
void MatrixDataELL::allocateIndexAndData() {
  index = new int[elements > 0 ? elements : 1]();
  data = new floatType[elements > 0 ? elements : 1]();
}
void MatrixDataELL::deallocateIndexAndData() {
  delete[] index;
  delete[] data;
  index = nullptr;
  data = nullptr;
}

template <> void DataMatrix<MatrixDataCRS>::convert(const MatrixCOO &coo) {
  N = coo.N;
  nz = coo.nz;
  allocatePtr(N);
  ptr[0] = 0;
  for (int r = 0; r < N; r++) ptr[r + 1] = ptr[r] + coo.nzPerRow[r];
  allocateIndexAndValue(nz);
  std::vector<int> next(ptr, ptr + N);
  for (int e = 0; e < nz; e++) {
    int slot = next[coo.I[e]]++;
    index[slot] = coo.J[e];
    value[slot] = coo.V[e];
  }
}

template <> void DataMatrix<MatrixDataELL>::convert(const MatrixCOO &coo) {
  N = coo.N;
  nz = coo.nz;
  maxNz = coo.getMaxNz();
  const long long slots = (long long)maxNz * N;
  if (slots > 0x7fffffffLL) {
    std::cerr << "ELL matrix too large for this interface!" << std::endl;
    std::exit(1);
  }
  elements = (int)slots;
  allocateLength(N);
  std::memcpy(length, coo.nzPerRow.get(), sizeof(int) * (size_t)N);
  allocateIndexAndData();
  std::vector<int> fill((size_t)N, 0);
  for (int e = 0; e < nz; e++) {
    const int r = coo.I[e];
    const size_t k = (size_t)fill[r]++ * (size_t)N + (size_t)r;
    index[k] = coo.J[e];
    data[k] = coo.V[e];
  }
}

void Jacobi::allocateC(int N) { C = new floatType[N](); }
void Jacobi::deallocateC() {
  delete[] C;
  C = nullptr;
}
void Jacobi::init(const MatrixCOO &coo) {
  allocateC(coo.N);
  // The last diagonal entry in file order wins (Preconditioner.cpp:13-23).
  for (int e = 0; e < coo.nz; e++)
    if (coo.I[e] == coo.J[e]) C[coo.I[e]] = 1 / coo.V[e];
}
