// The CG class of cg_b200: the reference's solver surface (CG.h:19-293 of
// hahnjo/CGxx) -- same public methods, the same protected per-kernel virtual
// interface, the same CG_* environment switches, right-hand side, check and
// summary output -- so that a backend written for the reference's CG ports by
// recompiling, and tools that parse its output keep working.
//
// One addition: solve() first offers the whole solve to the backend through
// the virtual fusedSolve(); a backend that runs the iteration on the device
// (CGB200) returns true and never receives the per-kernel calls. Backends
// without it fall back to the reference's algorithm, driven kernel by kernel.
#ifndef CGB200_CG_H
#define CGB200_CG_H

#include <cassert>
#include <chrono>
#include <memory>
#include <string>

#include "Matrix.h"

class CG {
public:
  enum Vector { VectorK, VectorX, VectorP, VectorQ, VectorR, VectorZ };
  enum MatrixFormat { MatrixFormatCOO, MatrixFormatCRS, MatrixFormatELL };
  enum Preconditioner { PreconditionerNone, PreconditionerJacobi };
  enum WorkDistributionCalc { WorkDistributionByRow, WorkDistributionByNz };

private:
  struct Timing {
    using clock = std::chrono::steady_clock;
    using duration = std::chrono::duration<double>;
    duration io{0}, converting{0}, transferTo{0}, transferFrom{0}, check{0};
    duration solve{0}, matvec{0}, axpy{0}, xpay{0}, vectorDot{0},
        preconditioner{0};
  };
  using time_point = Timing::clock::time_point;
  time_point now() const { return Timing::clock::now(); }

  // Timed wrappers around the per-kernel interface.
  void matvec(Vector in, Vector out);
  void axpy(floatType a, Vector x, Vector y);
  void xpay(Vector x, floatType a, Vector y);
  floatType vectorDot(Vector a, Vector b);
  void applyPreconditioner(Vector x, Vector y);

  // The reference's PCG, one virtual kernel call at a time.
  void genericSolve();

protected:
  int iteration = 0;
  int maxIterations = 1000;
  floatType residual = 0;
  floatType tolerance = 1e-9;
  floatType checkTolerance = 1e-5;
  Timing timing;

  int N = 0;
  int nz = 0;

  // Accepted for compatibility; a single device has no work distribution.
  WorkDistributionCalc workDistributionCalc = WorkDistributionByRow;
  bool overlappedGather = false;

  MatrixFormat matrixFormat;
  std::unique_ptr<MatrixCOO> matrixCOO;
  std::unique_ptr<MatrixCRS> matrixCRS;
  std::unique_ptr<MatrixELL> matrixELL;

  Preconditioner preconditioner;
  std::unique_ptr<Jacobi> jacobi;

  floatType *k = nullptr;
  floatType *x = nullptr;

  CG(MatrixFormat defaultMatrixFormat,
     Preconditioner defaultPreconditioner = PreconditionerNone)
      : matrixFormat(defaultMatrixFormat),
        preconditioner(defaultPreconditioner) {}

  virtual bool supportsMatrixFormat(MatrixFormat format) = 0;
  virtual bool supportsPreconditioner(Preconditioner) { return false; }
  virtual int getNumberOfChunks() { return -1; }
  virtual bool supportsOverlappedGather() { return false; }

  virtual void allocateMatrixCRS();
  virtual void allocateMatrixELL();
  virtual void allocateJacobi();
  virtual void allocateK();
  virtual void deallocateK();
  virtual void allocateX();
  virtual void deallocateX();

  virtual void doTransferTo() {}
  virtual void doTransferFrom() {}

  virtual void cpy(Vector dst, Vector src) = 0;
  virtual void matvecKernel(Vector x, Vector y) = 0;
  virtual void axpyKernel(floatType a, Vector x, Vector y) = 0;
  virtual void xpayKernel(Vector x, floatType a, Vector y) = 0;
  virtual floatType vectorDotKernel(Vector a, Vector b) = 0;
  virtual void applyPreconditionerKernel(Vector, Vector) {
    assert(0 && "Preconditioner not implemented!");
  }

  // Whole-solve hook: return true after solving (x, iteration and residual
  // set), false to let solve() run the per-kernel algorithm.
  virtual bool fusedSolve() { return false; }
  // A backend that builds the CRS/ELL layout on its device from the COO
  // entries it uploads returns true; init() then keeps the COO and skips the
  // host conversion (the conversion time moves into "Transfer to time").
  virtual bool convertsOnDevice() { return false; }
  // Lets a fused backend report device-measured per-kernel times (seconds).
  void setKernelTimes(double matvecS, double axpyS, double xpayS, double dotS,
                      double precondS);

  static void printPadded(const char *label, const std::string &value);

public:
  virtual ~CG() {}

  virtual void parseEnvironment();
  virtual void init(const char *matrixFile);

  void resetX();
  void resetNonInitTimings() {
    Timing old = timing;
    timing = Timing{};
    timing.io = old.io;
    timing.converting = old.converting;
  }

  virtual bool needsTransfer() { return false; }
  void transferTo() {
    auto start = now();
    doTransferTo();
    timing.transferTo = now() - start;
  }
  void solve();
  void transferFrom() {
    auto start = now();
    doTransferFrom();
    timing.transferFrom = now() - start;
  }

  virtual void printSummary();
  bool check();
  virtual void cleanup();

  static CG *getInstance();
};

#endif
