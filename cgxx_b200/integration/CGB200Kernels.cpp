// CGB200Kernels: a plug-in for the reference's own CG class (hahnjo/CGxx
// CG.h:19-293) that runs every kernel on a B200 through libcgb200's C ABI.
//
// This file is compiled against the UNMODIFIED reference headers and sources
// (oracle/Makefile target `adapter`), exactly as a maintainer would add a new
// programming model next to cuda/CGCUDA.cu: the reference's CG::solve
// (CG.cpp:284-385) drives the loop and receives every dot product on the
// host, so the iteration is the reference's own. It shows that the C ABI is a
// drop-in for the per-kernel interface; the fused device solve (cgx_solve)
// is the fast path and is what cg_b200 uses.
#include <cstdlib>
#include <iostream>

#include "CG.h"
#include "cgx.h"

namespace {
void ok(cgx_status s) {
  if (s != CGX_SUCCESS) {
    // The reference's error convention (cuda/utils.h:10-15).
    std::cerr << cgx_last_error() << std::endl;
    std::exit(1);
  }
}
}  // namespace

class CGB200Kernels : public CG {
  cgx_handle *h = nullptr;

  static cgx_vector v(Vector x) { return (cgx_vector)x; }

  bool supportsMatrixFormat(MatrixFormat f) override {
    return f == MatrixFormatCRS || f == MatrixFormatELL || f == MatrixFormatCOO;
  }
  bool supportsPreconditioner(Preconditioner p) override {
    return p == PreconditionerJacobi;
  }

  void init(const char *matrixFile) override {
    ok(cgx_create(&h, 0));
    CG::init(matrixFile);
  }

  void allocateX() override {
    ok(cgx_host_alloc((void **)&x, sizeof(floatType) * N));
  }
  void deallocateX() override { cgx_host_free(x); }

  bool needsTransfer() override { return true; }

  void doTransferTo() override {
    switch (matrixFormat) {
    case MatrixFormatCRS:
      ok(cgx_upload_crs(h, N, nz, matrixCRS->ptr, matrixCRS->index,
                        matrixCRS->value));
      break;
    case MatrixFormatELL:
      // The reference's conversion sets `elements` (= N * max row length)
      // but never `maxNz` (Matrix.cpp:339-361), so the width comes from it.
      ok(cgx_upload_ell(h, N, nz, N > 0 ? matrixELL->elements / N : 0,
                        matrixELL->length, matrixELL->index,
                        matrixELL->data));
      break;
    case MatrixFormatCOO:
      ok(cgx_upload_coo(h, N, nz, matrixCOO->I.get(), matrixCOO->J.get(),
                        matrixCOO->V.get()));
      break;
    }
    if (preconditioner == PreconditionerJacobi)
      ok(cgx_upload_jacobi(h, jacobi->C));
    ok(cgx_set_vector(h, CGX_VECTOR_K, k));
    ok(cgx_set_vector(h, CGX_VECTOR_X, x));
    ok(cgx_synchronize(h));
  }

  void doTransferFrom() override { ok(cgx_get_vector(h, CGX_VECTOR_X, x)); }

  void cpy(Vector dst, Vector src) override {
    ok(cgx_copy(h, v(dst), v(src)));
    ok(cgx_synchronize(h));
  }
  void matvecKernel(Vector x_, Vector y_) override {
    ok(cgx_matvec(h, v(x_), v(y_)));
    ok(cgx_synchronize(h));
  }
  void axpyKernel(floatType a, Vector x_, Vector y_) override {
    ok(cgx_axpy(h, a, v(x_), v(y_)));
    ok(cgx_synchronize(h));
  }
  void xpayKernel(Vector x_, floatType a, Vector y_) override {
    ok(cgx_xpay(h, v(x_), a, v(y_)));
    ok(cgx_synchronize(h));
  }
  floatType vectorDotKernel(Vector a, Vector b) override {
    double r = 0;
    ok(cgx_dot(h, v(a), v(b), &r));
    return r;
  }
  void applyPreconditionerKernel(Vector x_, Vector y_) override {
    ok(cgx_apply_jacobi(h, v(x_), v(y_)));
    ok(cgx_synchronize(h));
  }

public:
  CGB200Kernels() : CG(MatrixFormatCRS, PreconditionerJacobi) {}

  void cleanup() override {
    CG::cleanup();
    if (h) cgx_destroy(h);
    h = nullptr;
  }
};

CG *CG::getInstance() { return new CGB200Kernels; }
