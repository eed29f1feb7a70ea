// Sparse matrix containers of the cg_b200 host program.
//
// The field names and layouts are the reference's (Matrix.h:14-103) because
// they are part of the interface a CG backend programs against: COO arrays
// I/J/V plus nzPerRow; CRS ptr/index/value; column-major padded ELL with
// maxNz, elements, length, index, data and element (i, j) at j*N + i.
// Allocation goes through virtual hooks so that a backend can place the
// arrays in pinned memory (the reference's Matrix.h:58-65, 90-97).
#ifndef CGB200_MATRIX_H
#define CGB200_MATRIX_H

#include <memory>

using floatType = double;

struct Matrix {
  int N = 0;
  int nz = 0;
};

struct MatrixCOO : Matrix {
  std::unique_ptr<int[]> I;
  std::unique_ptr<int[]> J;
  std::unique_ptr<floatType[]> V;
  std::unique_ptr<int[]> nzPerRow;

  MatrixCOO() = delete;
  // Reads a MatrixMarket file (parallel reader of libcgb200, cgx_mtx_read).
  // Prints the reference's message and exits with status 1 on errors.
  explicit MatrixCOO(const char *file);

  int getMaxNz() const;
};

struct MatrixDataCRS {
  int *ptr = nullptr;
  int *index = nullptr;
  floatType *value = nullptr;

  virtual ~MatrixDataCRS() {}
  virtual void allocatePtr(int rows);
  virtual void deallocatePtr();
  virtual void allocateIndexAndValue(int values);
  virtual void deallocateIndexAndValue();
  void deallocate() {
    deallocatePtr();
    deallocateIndexAndValue();
  }
};

struct MatrixDataELL {
  int maxNz = 0;
  int elements = 0;  // kept as int for interface compatibility
  int *length = nullptr;
  int *index = nullptr;
  floatType *data = nullptr;

  virtual ~MatrixDataELL() {}
  virtual void allocateLength(int rows);
  virtual void deallocateLength();
  virtual void allocateIndexAndData();
  virtual void deallocateIndexAndData();
  void deallocate() {
    deallocateLength();
    deallocateIndexAndData();
  }
};

template <class Data> struct DataMatrix : Matrix, Data {
  // Converts keeping each row's entries in COO (file) order.
  void convert(const MatrixCOO &coo);
};
using MatrixCRS = DataMatrix<MatrixDataCRS>;
using MatrixELL = DataMatrix<MatrixDataELL>;

// Jacobi preconditioner: C = 1 / diag(A) (the reference's Preconditioner.h).
struct Jacobi {
  floatType *C = nullptr;
  virtual ~Jacobi() {}
  void init(const MatrixCOO &coo);
  virtual void allocateC(int N);
  virtual void deallocateC();
};

#endif
