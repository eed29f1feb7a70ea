// In-process driver for the reference's own CG -- TEST INFRASTRUCTURE ONLY.
//
// Linked by oracle/Makefile against the unmodified reference sources
// (CG.cpp compiled with -Dmain=cg_reference_main, Matrix.cpp,
// Preconditioner.cpp, WorkDistribution.cpp and one backend such as
// serial/SerialCG.cpp or openmp/CGOpenMP.cpp). It runs the same sequence as
// the reference's main() (CG.cpp:539-591) but can replace the right-hand side
// k (protected member, CG.h:167) before solving and writes the solution x to
// a binary file, so that tests can compare the reference's x with ours.
//
// usage: ref_harness <matrix.mtx> [--rhs k.bin] [--x-out x.bin] [--reps n]
//   k.bin / x.bin hold N little-endian doubles and nothing else.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <memory>
#include <vector>

#include "CG.h"

namespace {
// Forming &Peek::k inside a class derived from CG yields a floatType*CG::*
// that may be applied to any CG object -- the one portable way to reach a
// protected member of an object whose dynamic type is another subclass.
struct Peek : CG {
  static floatType *CG::*kMember() { return &Peek::k; }
  static floatType *CG::*xMember() { return &Peek::x; }
  static int CG::*nMember() { return &Peek::N; }
};
}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) {
    std::cerr << "usage: " << argv[0]
              << " <matrix.mtx> [--rhs k.bin] [--x-out x.bin] [--reps n]"
              << std::endl;
    return 2;
  }
  const char *mtx = argv[1];
  const char *rhs = nullptr, *xout = nullptr;
  int reps = 1;
  for (int a = 2; a < argc; a++) {
    if (!std::strcmp(argv[a], "--rhs") && a + 1 < argc)
      rhs = argv[++a];
    else if (!std::strcmp(argv[a], "--x-out") && a + 1 < argc)
      xout = argv[++a];
    else if (!std::strcmp(argv[a], "--reps") && a + 1 < argc)
      reps = std::atoi(argv[++a]);
    else {
      std::cerr << "bad argument " << argv[a] << std::endl;
      return 2;
    }
  }

  std::unique_ptr<CG> cg(CG::getInstance());
  cg->parseEnvironment();
  cg->init(mtx);
  int N = (*cg).*Peek::nMember();

  if (rhs) {
    FILE *f = std::fopen(rhs, "rb");
    if (!f) {
      std::cerr << "cannot open " << rhs << std::endl;
      return 2;
    }
    floatType *k = (*cg).*Peek::kMember();
    size_t got = std::fread(k, sizeof(floatType), (size_t)N, f);
    std::fclose(f);
    if (got != (size_t)N) {
      std::cerr << "short rhs file" << std::endl;
      return 2;
    }
  }

  for (int i = 0; i < reps; i++) {
    if (i != 0) std::cout << std::endl;
    if (cg->needsTransfer()) cg->transferTo();
    cg->solve();
    if (cg->needsTransfer()) cg->transferFrom();
    cg->check();
    cg->printSummary();
    if (i + 1 == reps && xout) {
      FILE *f = std::fopen(xout, "wb");
      floatType *x = (*cg).*Peek::xMember();
      std::fwrite(x, sizeof(floatType), (size_t)N, f);
      std::fclose(f);
    }
    cg->resetX();
    cg->resetNonInitTimings();
  }
  cg->cleanup();
  return 0;
}
