// CG base class of cg_b200 and the program's main(). Reproduces the
// reference's observable behaviour (hahnjo/CGxx CG.cpp): environment
// switches and their error messages / exit status, the right-hand side
// k = A * 1, x0 = 0, the solution check and the labelled summary.
#include "CG.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>

namespace {

[[noreturn]] void die(const std::string &msg) {
  std::cerr << msg << std::endl;
  std::exit(1);
}

// Non-empty value of an environment variable, or nullptr.
const char *envValue(const char *name) {
  const char *v = std::getenv(name);
  return (v != nullptr && *v != 0) ? v : nullptr;
}

// strtol/strtod accept the value only if the whole string converts without a
// range error (the reference's checks, CG.cpp:39-74).
bool wholeLong(const char *s, long &out) {
  char *end = nullptr;
  errno = 0;
  out = std::strtol(s, &end, 0);
  return errno == 0 && *end == 0;
}

bool wholeDouble(const char *s, double &out) {
  char *end = nullptr;
  errno = 0;
  out = std::strtod(s, &end);
  return errno == 0 && *end == 0;
}

std::string upper(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), ::toupper);
  return s;
}

std::string lower(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), ::tolower);
  return s;
}

}  // namespace

// --- environment -------------------------------------------------------------

void CG::parseEnvironment() {
  if (const char *v = envValue("CG_MAX_ITER")) {
    long n;
    int asInt = wholeLong(v, n) ? (int)n : 0;
    if (!wholeLong(v, n) || asInt <= 0) die("Invalid value for CG_MAX_ITER!");
    maxIterations = asInt;
  }
  if (const char *v = envValue("CG_TOLERANCE")) {
    double t;
    if (!wholeDouble(v, t) || !(t > 0)) die("Invalid value for CG_TOLERANCE!");
    tolerance = t;
  }
  if (const char *v = envValue("CG_CHECK_TOLERANCE")) {
    double t;
    // As in the reference (CG.cpp:67), the value is accepted whenever it
    // parses and the *convergence* tolerance is positive.
    if (!wholeDouble(v, t) || !(tolerance > 0))
      die("Invalid value for CG_CHECK_TOLERANCE!");
    checkTolerance = t;
  }
  if (const char *v = envValue("CG_MATRIX_FORMAT")) {
    const std::string f = upper(v);
    if (f == "COO")
      matrixFormat = MatrixFormatCOO;
    else if (f == "CRS")
      matrixFormat = MatrixFormatCRS;
    else if (f == "ELL")
      matrixFormat = MatrixFormatELL;
    else
      die("Invalid value for CG_MATRIX_FORMAT! (COO, CRS, or ELL)");
    if (!supportsMatrixFormat(matrixFormat))
      die("No support for this matrix format!");
  }
  if (const char *v = envValue("CG_PRECONDITIONER")) {
    const std::string p = lower(v);
    if (p == "none")
      preconditioner = PreconditionerNone;
    else if (p == "jacobi")
      preconditioner = PreconditionerJacobi;
    else
      die("Invalid value for CG_PRECONDITIONER! (none, or jacobi)");
    if (preconditioner != PreconditionerNone &&
        !supportsPreconditioner(preconditioner))
      die("No support for this preconditioner!");
  }
  if (const char *v = envValue("CG_WORK_DISTRIBUTION")) {
    const std::string w = lower(v);
    if (w == "row")
      workDistributionCalc = WorkDistributionByRow;
    else if (w == "nz")
      workDistributionCalc = WorkDistributionByNz;
    else
      die("Invalid value for CG_WORK_DISTRIBUTION! (row, or nz)");
  }
  if (const char *v = envValue("CG_OVERLAPPED_GATHER")) {
    overlappedGather = std::string(v) != "0";
    if (overlappedGather &&
        (getNumberOfChunks() == -1 || !supportsOverlappedGather()))
      die("No support for overlapped gather!");
  }
}

// --- allocation hooks ----------------------------------------------------------

void CG::allocateMatrixCRS() { matrixCRS.reset(new MatrixCRS); }
void CG::allocateMatrixELL() { matrixELL.reset(new MatrixELL); }
void CG::allocateJacobi() { jacobi.reset(new Jacobi); }
void CG::allocateK() { k = new floatType[N]; }
void CG::deallocateK() {
  delete[] k;
  k = nullptr;
}
void CG::allocateX() { x = new floatType[N]; }
void CG::deallocateX() {
  delete[] x;
  x = nullptr;
}

// --- set-up ----------------------------------------------------------------------

void CG::init(const char *matrixFile) {
  std::cout << "Reading matrix from " << matrixFile << "..." << std::endl;
  const auto startIO = now();
  matrixCOO.reset(new MatrixCOO(matrixFile));
  N = matrixCOO->N;
  nz = matrixCOO->nz;
  const auto startConverting = now();

  const bool onDevice = convertsOnDevice();
  if (matrixFormat == MatrixFormatCRS) {
    std::cout << "Converting matrix to CRS format..." << std::endl;
    if (!onDevice) {
      allocateMatrixCRS();
      matrixCRS->convert(*matrixCOO);
    }
  } else if (matrixFormat == MatrixFormatELL) {
    std::cout << "Converting matrix to ELL format..." << std::endl;
    if (!onDevice) {
      allocateMatrixELL();
      matrixELL->convert(*matrixCOO);
    }
  }
  if (preconditioner == PreconditionerJacobi) {
    std::cout << "Initializing Jacobi preconditioner..." << std::endl;
    allocateJacobi();
    jacobi->init(*matrixCOO);
  }
  timing.converting = now() - startConverting;
  timing.io = now() - startIO;

  // Right-hand side with the exact solution (1, ..., 1): row sums in COO
  // order (CG.cpp:256-261).
  allocateK();
  std::fill(k, k + N, 0.0);
  for (int e = 0; e < nz; e++) k[matrixCOO->I[e]] += matrixCOO->V[e];

  allocateX();
  resetX();

  if (matrixFormat != MatrixFormatCOO && !onDevice) matrixCOO.reset();
}

void CG::resetX() { std::fill(x, x + N, 0.0); }

// --- timed kernel wrappers -------------------------------------------------------

void CG::matvec(Vector in, Vector out) {
  auto t = now();
  matvecKernel(in, out);
  timing.matvec += now() - t;
}
void CG::axpy(floatType a, Vector xv, Vector yv) {
  auto t = now();
  axpyKernel(a, xv, yv);
  timing.axpy += now() - t;
}
void CG::xpay(Vector xv, floatType a, Vector yv) {
  auto t = now();
  xpayKernel(xv, a, yv);
  timing.xpay += now() - t;
}
floatType CG::vectorDot(Vector a, Vector b) {
  auto t = now();
  floatType r = vectorDotKernel(a, b);
  timing.vectorDot += now() - t;
  return r;
}
void CG::applyPreconditioner(Vector xv, Vector yv) {
  auto t = now();
  applyPreconditionerKernel(xv, yv);
  timing.preconditioner += now() - t;
}

void CG::setKernelTimes(double matvecS, double axpyS, double xpayS,
                        double dotS, double precondS) {
  timing.matvec = Timing::duration(matvecS);
  timing.axpy = Timing::duration(axpyS);
  timing.xpay = Timing::duration(xpayS);
  timing.vectorDot = Timing::duration(dotS);
  timing.preconditioner = Timing::duration(precondS);
}

// --- solve ---------------------------------------------------------------------------

void CG::solve() {
  std::cout << "Solving..." << std::endl;
  const auto start = now();
  if (!fusedSolve()) genericSolve();
  timing.solve = now() - start;
}

// Hestenes-Stiefel PCG as the reference runs it (CG.cpp:284-385): the
// convergence test is on the recurrence residual relative to ||r0||, and the
// iteration that meets it is counted.
void CG::genericSolve() {
  const bool pc = preconditioner != PreconditionerNone;
  matvec(VectorX, VectorR);
  xpay(VectorK, -1.0, VectorR);
  if (pc)
    applyPreconditioner(VectorR, VectorP);
  else
    cpy(VectorP, VectorR);
  floatType r2 = vectorDot(VectorR, VectorR);
  const floatType nrm0 = std::sqrt(r2);
  floatType rho = pc ? vectorDot(VectorP, VectorR) : r2;

  for (iteration = 0; iteration < maxIterations; iteration++) {
    matvec(VectorP, VectorQ);
    const floatType a = rho / vectorDot(VectorP, VectorQ);
    axpy(a, VectorP, VectorX);
    axpy(-a, VectorQ, VectorR);
    r2 = vectorDot(VectorR, VectorR);
    residual = std::sqrt(r2) / nrm0;
    if (residual <= tolerance) {
      iteration++;
      break;
    }
    const floatType rhoOld = rho;
    if (pc) {
      applyPreconditioner(VectorR, VectorZ);
      rho = vectorDot(VectorR, VectorZ);
    } else {
      rho = r2;
    }
    xpay(pc ? VectorZ : VectorR, rho / rhoOld, VectorP);
  }
}

// --- check and summary -------------------------------------------------------------

bool CG::check() {
  std::cout << "Checking solution..." << std::endl;
  const auto start = now();
  int errors = 0;
  for (int i = 0; i < N; i++)
    if (std::abs(x[i] - 1.0) > checkTolerance) errors++;
  timing.check = now() - start;
  if (errors == 0)
    std::cout << "Solution is correct!" << std::endl;
  else
    std::cout << errors << " elements are incorrect!" << std::endl;
  return errors == 0;
}

void CG::printPadded(const char *label, const std::string &value) {
  std::cout << std::left << std::setw(25) << label << value << std::endl;
}

void CG::printSummary() {
  std::cout << std::endl << "x = [ ";
  for (int i = 0; i < 10 && i < N; i++) std::cout << x[i] << " ";
  std::cout << "]" << std::endl;

  printPadded("Iterations:", std::to_string(iteration));
  std::ostringstream res;
  res << std::scientific << residual;
  printPadded("Residual:", res.str());
  printPadded("# rows / # nonzeros:",
              std::to_string(N) + " / " + std::to_string(nz));
  static const char *formats[] = {"COO", "CRS", "ELL"};
  printPadded("Matrix format:", formats[matrixFormat]);
  printPadded("Preconditioner:",
              preconditioner == PreconditionerNone ? "None" : "Jacobi");

  std::cout << std::endl;
  printPadded("IO time:", std::to_string(timing.io.count()));
  double total = 0;
  if (matrixFormat != MatrixFormatCOO || preconditioner != PreconditionerNone) {
    printPadded("Converting time:", std::to_string(timing.converting.count()));
    total += timing.converting.count();
  }
  if (needsTransfer()) {
    printPadded("Transfer to time:", std::to_string(timing.transferTo.count()));
    total += timing.transferTo.count();
  }
  printPadded("Solve time:", std::to_string(timing.solve.count()));
  total += timing.solve.count();
  if (needsTransfer()) {
    printPadded("Transfer from time:",
                std::to_string(timing.transferFrom.count()));
    total += timing.transferFrom.count();
  }
  printPadded("Check time:", std::to_string(timing.check.count()));
  total += timing.check.count();
  printPadded("Total time (excl. IO):", std::to_string(total));

  std::cout << std::endl;
  const double mv = timing.matvec.count();
  printPadded("MatVec time:", std::to_string(mv));
  // The first product (r = k - A x0) counts too (CG.cpp:509-511).
  const double flops = 2.0 * (iteration + 1) * nz;
  printPadded("MatVec GFLOP/s:", std::to_string(flops / 1e9 / mv));
  printPadded("axpy time:", std::to_string(timing.axpy.count()));
  printPadded("xpay time:", std::to_string(timing.xpay.count()));
  printPadded("vectorDot time:", std::to_string(timing.vectorDot.count()));
  if (preconditioner != PreconditionerNone)
    printPadded("Preconditioner time:",
                std::to_string(timing.preconditioner.count()));
}

void CG::cleanup() {
  deallocateK();
  deallocateX();
  if (matrixCRS) matrixCRS->deallocate();
  if (matrixELL) matrixELL->deallocate();
  if (jacobi) jacobi->deallocateC();
}

// --- program ----------------------------------------------------------------------------

int main(int argc, char *argv[]) {
  if (argc != 2 && argc != 3) {
    std::cerr << "Usage: " << argv[0] << " <matrix.mtx> [<repetitions>]"
              << std::endl;
    std::exit(1);
  }
  int repetitions = 1;
  if (argc > 2) {
    long r;
    if (wholeLong(argv[2], r) && (int)r > 0)
      repetitions = (int)r;
    else
      std::cerr << "Invalid value for repetitions! Disabling..." << std::endl;
  }

  std::unique_ptr<CG> cg(CG::getInstance());
  cg->parseEnvironment();
  cg->init(argv[1]);
  for (int i = 0; i < repetitions; i++) {
    if (i != 0) std::cout << std::endl;
    if (cg->needsTransfer()) cg->transferTo();
    cg->solve();
    if (cg->needsTransfer()) cg->transferFrom();
    cg->check();
    cg->printSummary();
    cg->resetX();
    cg->resetNonInitTimings();
  }
  cg->cleanup();
  return EXIT_SUCCESS;
}
